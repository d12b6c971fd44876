"""ctypes binding of libbbpd (include/bbpd.h).

The library is the product: every numerical call below runs CUDA kernels. If
the shared object is missing, or no GPU is visible, calls raise; there is no
Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("BBPD_LIB") or os.path.join(HERE, "lib", "libbbpd.so")
MEX_DIR = os.path.join(HERE, "mex")

# status codes (bbpd_status)
OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_NONFINITE, ERR_UNSUPPORTED, ERR_NO_DEVICE = range(8)
LAW_LINEAR, LAW_BILINEAR, LAW_TRILINEAR, LAW_EXPONENTIAL = range(4)
SCHEME_EULERCROMER, SCHEME_ADR = range(2)
PREC_FP64, PREC_FP32 = range(2)
AMP_LINEAR, AMP_SMOOTHSTEP = range(2)
ORDER_INPUT, ORDER_MORTON, ORDER_TILED, ORDER_LATTICE = range(4)
FIELD = {"displacement": 0, "velocity": 1, "force": 2, "deformed": 3, "force_prev": 4,
         "acceleration": 5, "bsf": 16, "flag": 17, "fail": 18, "damage_energy": 19}
LAWS = {"linear": LAW_LINEAR, "bilinear": LAW_BILINEAR, "trilinear": LAW_TRILINEAR,
        "exponential": LAW_EXPONENTIAL}


class BBPDError(RuntimeError):
    """A libbbpd call returned a non-zero bbpd_status."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("law", C.c_int32), ("scheme", C.c_int32), ("precision", C.c_int32),
        ("n_chunks", C.c_int32), ("amplitude", C.c_int32), ("node_order", C.c_int32),
        ("cell_volume", C.c_double), ("dt", C.c_double), ("damping", C.c_double),
        ("s0", C.c_double), ("s1", C.c_double), ("sc", C.c_double), ("sc_steel", C.c_double),
        ("k_exp", C.c_double), ("alpha_exp", C.c_double), ("beta_tri", C.c_double),
        ("failure_functionality", C.c_double), ("rate", C.c_double),
        ("applied_final", C.c_double), ("n_time_steps", C.c_int64),
        ("guard_band", C.c_double), ("barrier_timeout_s", C.c_double),
    ]


_P = C.POINTER(C.c_double)


class Problem(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64), ("n_bonds", C.c_int64),
        ("undeformed_coordinates", _P), ("bondlist", _P), ("undeformed_length", _P),
        ("bond_stiffness", _P), ("volume_correction", _P), ("bond_type", _P), ("fail", _P),
        ("stretch_plastic", _P), ("s0", _P), ("s1", _P), ("sc", _P), ("density", _P),
        ("mass", _P), ("constraint_flag", _P), ("prescribed_flag", _P),
    ]


class Info(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64), ("n_bonds", C.c_int64), ("n_entries", C.c_int64),
        ("n_slices", C.c_int64), ("grid_blocks", C.c_int32), ("block_threads", C.c_int32),
        ("device_bytes", C.c_int64), ("bytes_per_step", C.c_double), ("layout", C.c_int32),
        ("reserved", C.c_int32),
    ]


class Penetrator(C.Structure):
    _fields_ = [("centre_x", C.c_double), ("centre_z", C.c_double), ("radius", C.c_double),
                ("increment", C.c_double), ("family", _P), ("n_family", C.c_int64),
                ("reaction", C.c_int32), ("reserved", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [
        ("n_members", C.c_int32), ("blocks_per_sm", C.c_int32), ("grab", C.c_int32),
        ("graph", C.c_int32), ("n_classes", C.c_int32), ("reserved", C.c_int32),
        ("total_slices", C.c_int64), ("device_bytes", C.c_int64),
    ]


class BeamSpec(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("dx", C.c_double),
        ("horizon_factor", C.c_double), ("E", C.c_double), ("stiffness_factor", C.c_double),
        ("density", C.c_double), ("support_x", C.c_double * 2), ("n_supports", C.c_int32),
        ("load_midspan_top", C.c_int32), ("notch", C.c_int32), ("sc_lognormal", C.c_int32),
        ("notch_x", C.c_double), ("notch_depth", C.c_double), ("sc_mean", C.c_double),
        ("sc_cov", C.c_double), ("seed", C.c_uint64),
    ]


class BeamScalars(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64), ("n_bonds", C.c_int64), ("horizon", C.c_double),
        ("cell_volume", C.c_double), ("bond_stiffness_concrete", C.c_double),
        ("dt", C.c_double), ("n_supported", C.c_int64), ("n_prescribed", C.c_int64),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load libbbpd.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m bb_pd_b200.build` "
                               "(libbbpd has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.bbpd_last_error.restype = C.c_char_p
        L.bbpd_status_string.restype = C.c_char_p
        L.bbpd_params_default.restype = None
        L.bbpd_create.argtypes = [C.POINTER(Problem), C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]
        for name in ("bbpd_step", "bbpd_step_async"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_int64]
        for name in ("bbpd_sync", "bbpd_destroy"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.bbpd_get.argtypes = [C.c_void_p, C.c_int, _P]
        L.bbpd_set.argtypes = [C.c_void_p, C.c_int, _P]
        L.bbpd_get_step.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.bbpd_set_step.argtypes = [C.c_void_p, C.c_int64, C.c_double]
        L.bbpd_get_info.argtypes = [C.c_void_p, C.POINTER(Info)]
        L.bbpd_last_kernel_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
        L.bbpd_selftest_wait_timeout.argtypes = [C.c_double]
        L.bbpd_selftest_division.argtypes = [C.c_int64, C.c_uint64] + [C.POINTER(C.c_int64)] * 3 + [_P]
        L.bbpd_selftest_fp64_peak.argtypes = [C.c_double, _P]
        L.bbpd_selftest_exp.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_uint64, C.POINTER(C.c_int64),
                                        C.POINTER(C.c_uint64)]
        L.bbpd_get_reaction.argtypes = [C.c_void_p, C.c_int64, _P]
        L.bbpd_track_damage_energy.argtypes = [C.c_void_p]
        L.bbpd_set_contact.argtypes = [C.c_void_p, C.c_int, C.POINTER(Penetrator)]
        L.bbpd_set_probes.argtypes = [C.c_void_p, C.c_int, _P, C.POINTER(C.c_int32)]
        L.bbpd_get_probes.argtypes = [C.c_void_p, C.c_int64, _P]
        L.bbpd_batch_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        for name in ("bbpd_batch_destroy",):
            getattr(L, name).argtypes = [C.c_void_p]
        for name in ("bbpd_batch_add", "bbpd_batch_remove"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_void_p]
        L.bbpd_batch_step.argtypes = [C.c_void_p, C.c_int64]
        L.bbpd_batch_tune.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.bbpd_batch_set_schedule.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.bbpd_batch_set_mixing.argtypes = [C.c_void_p, C.c_int]
        L.bbpd_batch_get_info.argtypes = [C.c_void_p, C.POINTER(BatchInfo)]
        L.bbpd_batch_last_kernel_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
        L.bbpd_beam_count.argtypes = [C.POINTER(BeamSpec), C.POINTER(BeamScalars)]
        L.bbpd_beam_build.argtypes = [C.POINTER(BeamSpec)] + [_P] * 11
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        L = lib()
        msg = L.bbpd_last_error().decode(errors="replace")
        raise BBPDError(status, f"libbbpd: {L.bbpd_status_string(status).decode()}: {msg}")


def ptr(a: np.ndarray | None):
    """Pointer to a contiguous float64 array (or NULL)."""
    if a is None:
        return None
    if a.dtype != np.float64 or not (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]):
        raise TypeError("expected a contiguous float64 array")
    return a.ctypes.data_as(_P)


def device_count() -> int:
    return int(lib().bbpd_device_count())
