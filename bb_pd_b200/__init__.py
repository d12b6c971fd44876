"""bb_pd_b200: BB_PD's bond-force + explicit/ADR time-step hot path on B200.

The numerical work runs in libbbpd (CUDA, sm_100a; C ABI in include/bbpd.h).
This package is the host-side mirror of the reference's MATLAB calls:

    routines   the reference MEX routines under their own names (in place)
    Solver     the fused time loop, state resident on the GPU
    Batch      many solvers stepped by one persistent launch (batching form)
    serving    continuous batching of beam solves under an HBM budget
    beam       synthetic beams like the reference's input scripts
    builder    the reference's input module (horizons, notch, bond data) on the GPU
    static     the static (implicit) Newton-Raphson solver and the stiffness triplets
"""
from . import _native, beam, builder, routines, serving, static
from ._native import BBPDError, device_count
from .batch import Batch
from .solver import Solver, make_params

__all__ = ["Solver", "Batch", "make_params", "beam", "builder", "routines", "static", "serving", "BBPDError", "device_count",
           "_native"]
