"""Call mexFunction gateways from Python with the stub mxArray layout of
bb_pd_b200/csrc/mexstub/mex.h ({rows, cols, double *pr})."""
import ctypes as C
import os

import numpy as np

from bb_pd_b200 import _native as N


class MxArray(C.Structure):
    _fields_ = [("m", C.c_size_t), ("n", C.c_size_t), ("pr", C.POINTER(C.c_double))]


def _mx(a, keep):
    if np.isscalar(a):
        a = np.array([[float(a)]], order="F")
    assert isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
    keep.append(a)
    m = a.shape[0]
    n = a.shape[1] if a.ndim == 2 else 1
    return MxArray(m, n, a.ctypes.data_as(C.POINTER(C.c_double)))


def _call(fn, args):
    keep = []
    arr = (MxArray * max(len(args), 1))(*[_mx(a, keep) for a in args])
    ptrs = (C.POINTER(MxArray) * max(len(args), 1))(*[C.pointer(arr[i]) for i in range(len(args))])
    fn.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    fn.restype = None
    fn(0, None, len(args), ptrs)


_gw = {}


def gateway(name):
    if name not in _gw:
        so = C.CDLL(os.path.join(N.MEX_DIR, name + ".mexa64"))
        so.mexstub_error_message.restype = C.c_char_p
        _gw[name] = so
    return _gw[name]


def call_gateway(name, args):
    """Run our gateway; returns (errors raised by this call, last message)."""
    so = gateway(name)
    before = so.mexstub_error_count()
    _call(so.mexFunction, args)
    return so.mexstub_error_count() - before, so.mexstub_error_message().decode()


def call_ref_gateway(ref_lib, symbol, args):
    """Run one of the reference's own gateways (compiled with the same stub)."""
    _call(getattr(ref_lib, symbol), args)
