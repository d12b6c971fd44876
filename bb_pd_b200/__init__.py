"""bb_pd_b200: BB_PD's bond-force + explicit/ADR time-step hot path on B200.

The numerical work runs in libbbpd (CUDA, sm_100a; C ABI in include/bbpd.h).
This package is the host-side mirror of the reference's MATLAB calls:

    routines   the reference MEX routines under their own names (in place)
    Solver     the fused time loop, state resident on the GPU
    beam       synthetic beams like the reference's input scripts
"""
from . import _native, beam, routines
from ._native import BBPDError, device_count
from .solver import Solver, make_params

__all__ = ["Solver", "make_params", "beam", "routines", "BBPDError", "device_count", "_native"]
