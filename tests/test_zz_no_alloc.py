"""GPU test of bbpd_dev_calculatedampingcoefficient_noalloc, the damping
coefficient with fixed in-library scratch and the result in device memory.

It must agree with bbpd_dev_calculatedampingcoefficient (the allocating
routine) on two calls in a row with different inputs; both reduce in the same
32-ary tree order, so the test tolerance is exact equality. Sizes beyond the
static scratch are rejected before anything is launched. Edge sizes (empty,
one slice, exactly one group of 32 slices), the clamp branch and a small call
made right after the largest one are compared the same way. This file is named to
be collected last, so it also runs after every other GPU test in one process;
it passes alone as well (the first call does the per-device set-up)."""
import ctypes as C

import numpy as np
import pytest
import torch

from bb_pd_b200 import _native as N

pytestmark = pytest.mark.gpu

MAX_NODES = 16777216   # BBPD_DAMPING_NOALLOC_MAX_NODES
RTOL = 0.0             # same summation order: identical results expected


def _lib():
    L = N.lib()
    sig = [C.c_void_p] * 3 + [C.c_double] + [C.c_void_p] * 2 + [C.c_int64, C.c_void_p, C.c_void_p]
    L.bbpd_dev_calculatedampingcoefficient.argtypes = sig
    L.bbpd_dev_calculatedampingcoefficient_noalloc.argtypes = sig
    return L


def _inputs(nN, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    dev = torch.device("cuda")

    def col(scale):   # node-major nN x 3 (x of node k at [k], y at [k + nN], ...)
        return (torch.randn(3 * nN, generator=g, device=dev, dtype=torch.float64) * scale).contiguous()

    F, Fp, vhp, u = col(1e6), col(1e6), col(1e-3), col(1e-4)
    vhp[torch.rand(3 * nN, generator=g, device=dev) < 0.1] = 0.0   # skipped terms
    m = torch.rand(nN, generator=g, device=dev, dtype=torch.float64) * 9e4 + 1e4
    return F, m, Fp, vhp, u


def _args(t, dt, nN):
    F, m, Fp, vhp, u = t
    return (F.data_ptr(), m.data_ptr(), Fp.data_ptr(), dt, vhp.data_ptr(), u.data_ptr(), nN)


def test_noalloc_matches_allocating_routine_twice():
    L = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    dt = 1e-6
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    cases = [(70001, 11), (MAX_NODES, 12)]
    inputs = [_inputs(nN, seed) for nN, seed in cases]
    torch.cuda.synchronize()
    # two calls in a row, each into its own device slot
    for k, ((nN, _), t) in enumerate(zip(cases, inputs)):
        N.check(L.bbpd_dev_calculatedampingcoefficient_noalloc(
            *_args(t, dt, nN), C.c_void_p(out.data_ptr() + 8 * k), C.c_void_p(stream)))
    got = out.cpu().numpy()
    for k, ((nN, _), t) in enumerate(zip(cases, inputs)):
        ref = C.c_double(-2.0)
        N.check(L.bbpd_dev_calculatedampingcoefficient(
            *_args(t, dt, nN), C.cast(C.pointer(ref), C.c_void_p), C.c_void_p(stream)))
        np.testing.assert_allclose(got[k], ref.value, rtol=RTOL, atol=0.0)
        assert 0.0 <= got[k] <= 2.0


def _compare(L, cases, dt=1e-6):
    """Each case in turn through the no-allocation entry (results kept in
    device memory), then each through the allocating routine: equal bit for bit."""
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((len(cases),), -1.0, dtype=torch.float64, device="cuda")
    for k, (nN, t) in enumerate(cases):
        N.check(L.bbpd_dev_calculatedampingcoefficient_noalloc(
            *_args(t, dt, nN), C.c_void_p(out.data_ptr() + 8 * k), C.c_void_p(stream)))
    got = out.cpu().numpy()
    for k, (nN, t) in enumerate(cases):
        ref = C.c_double(-2.0)
        N.check(L.bbpd_dev_calculatedampingcoefficient(
            *_args(t, dt, nN), C.cast(C.pointer(ref), C.c_void_p), C.c_void_p(stream)))
        assert got[k] == ref.value, (nN, got[k], ref.value)
    return got


def test_noalloc_small_after_large():
    """A small case right after the largest one: the scratch then holds the
    large call's partials beyond the small call's range, which it must not read."""
    L = _lib()
    cases = [(MAX_NODES, _inputs(MAX_NODES, 21)), (70001, _inputs(70001, 22)), (1025, _inputs(1025, 23))]
    _compare(L, cases)


def test_noalloc_edge_sizes():
    """nNodes 0 (no slices), 1 and 32 (one slice), 1024 (exactly one group of
    32 slices: the top kernel reads the two partials directly) and 1025."""
    L = _lib()
    cases = [(n, _inputs(max(n, 1), 30 + n % 7)) for n in (0, 1, 32, 1024, 1025)]
    got = _compare(L, cases)
    assert got[0] == 0.0                       # empty sums: cn = 0


def test_noalloc_clamp_and_zero_branches():
    """cn > 2 is replaced by 1.9 (calculatedampingcoefficient.m:107-110), a
    non-positive quotient gives 0 and u = 0 gives 0 (cn2 = 0)."""
    L = _lib()
    dev = torch.device("cuda")
    nN = 2000
    m = torch.full((nN,), 2.0, dtype=torch.float64, device=dev)
    one = torch.ones(3 * nN, dtype=torch.float64, device=dev)
    zero = torch.zeros(3 * nN, dtype=torch.float64, device=dev)
    # (F/m - Fp/m) / (dt vh) = -10 for every DOF: cn1 / cn2 = 10, 2 sqrt(10) > 2
    clamp = (zero, m, (one * 20.0).contiguous(), one, one)
    # the same with the sign turned: cn1 / cn2 < 0
    negative = ((one * 20.0).contiguous(), m, zero, one, one)
    still = (one, m, zero, one, zero)          # u = 0
    got = _compare(L, [(nN, clamp), (nN, negative), (nN, still)], dt=1.0)
    assert got.tolist() == [1.9, 0.0, 0.0]


def test_noalloc_rejects_sizes_beyond_scratch():
    L = _lib()
    t = _inputs(32, 3)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.bbpd_dev_calculatedampingcoefficient_noalloc(
        *_args(t, 1e-6, MAX_NODES + 1), C.c_void_p(out.data_ptr()), None)
    assert rc == N.ERR_ARG
    assert "limit" in N.lib().bbpd_last_error().decode()
