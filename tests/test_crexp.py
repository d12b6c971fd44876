"""The correctly rounded exp of the exponential law (bb_pd_b200/csrc/crexp.cuh),
compiled for the host from the same source as the device code.

The reference's law calls libm's exp (calculatebsfexponentialMex.c:43); the
device replaces CUDA's exp with this one so that the law rounds exp(x) the
way a correctly rounded libm does. These tests pin the host build:
  * against exp(x) correctly rounded from an 80-digit decimal evaluation,
    on the law's argument range -25 .. 0, over the whole double range and at
    the ends (overflow, subnormal results, tiny arguments);
  * the fast double-double step against the 128-bit accurate step;
  * against glibc's exp, which is not correctly rounded everywhere: the
    disagreements are counted (reported), never more than one unit in the
    last place.
The GPU test (test_gpu_routines.py) checks that the device build returns the
same bits as this host build."""
import ctypes as C
import os
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "bb_pd_b200", "csrc")


def build_host_harness(out: str) -> C.CDLL:
    subprocess.run(["g++", "-O2", "-fopenmp", "-ffp-contract=off", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(HERE, "crexp_host.cpp"), "-o", out, "-lm"], check=True)
    L = C.CDLL(out)
    for f in ("crexp_many", "crexp_accurate_many", "glibc_exp_many"):
        getattr(L, f).argtypes = [C.c_void_p, C.c_void_p, C.c_long]
    L.crexp_survey.argtypes = [C.c_double, C.c_double, C.c_long, C.c_uint64] + [C.POINTER(C.c_long)] * 3
    L.crexp_bits_sum.argtypes = [C.c_double, C.c_double, C.c_long, C.c_uint64]
    L.crexp_bits_sum.restype = C.c_uint64
    return L


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    return build_host_harness(str(tmp_path_factory.mktemp("crexp") / "libcrexp_host.so"))


def run(L, fn, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    getattr(L, fn)(x.ctypes.data, y.ctypes.data, len(x))
    return y


def correctly_rounded(xs):
    getcontext().prec = 80
    return np.array([float(str(Decimal(float(x)).exp())) for x in xs])


EDGES = [0.0, -0.0, 1.0, -1.0, 0.5, -0.5, 100.0, -100.0, 709.78, 709.782712893384, 709.7827128933841,
         709.79, 710.0, -708.39, -708.4, -720.0, -744.4, -745.1, -745.13, -745.1332, -745.14, -746.0,
         2.0 ** -54, -2.0 ** -54, 2.0 ** -53, -2.0 ** -53, 2.0 ** -60, -2.0 ** -61, 1e-10, -1e-10,
         -25.0, -24.999999999999996, -1e-300, float("inf"), float("-inf")]


def test_edges(lib):
    x = np.array(EDGES)
    got = run(lib, "crexp_many", x)
    ref = correctly_rounded(x)
    for a, b, xi in zip(got, ref, x):
        assert a == b and np.signbit(a) == np.signbit(b), (xi, a, b)
    assert np.isnan(run(lib, "crexp_many", np.array([np.nan]))[0])


@pytest.mark.parametrize("lo,hi,n", [(-25.0, 0.0, 3000), (-745.0, 709.7, 3000), (-1e-3, 1e-3, 500),
                                     (-745.13, -708.0, 500)])
def test_against_decimal(lib, lo, hi, n):
    x = np.random.default_rng(int(1000 * abs(lo)) + n).uniform(lo, hi, n)
    got = run(lib, "crexp_many", x)
    ref = correctly_rounded(x)
    bad = np.nonzero(got.view(np.int64) != ref.view(np.int64))[0]
    assert len(bad) == 0, [(x[i], got[i], ref[i]) for i in bad[:5]]
    m = np.abs(x) >= 2.0 ** -60
    acc = run(lib, "crexp_accurate_many", x[m])
    assert np.array_equal(acc.view(np.int64), ref[m].view(np.int64))


def test_near_table_points(lib):
    """Arguments next to the reduction's multiples of ln2/256, where r is tiny
    and cancels most of x."""
    base = np.arange(-6000, 6000, 7, dtype=np.float64) * (np.log(2.0) / 256)
    x = np.concatenate([base, np.nextafter(base, np.inf), np.nextafter(base, -np.inf)])
    got = run(lib, "crexp_many", x)
    ref = correctly_rounded(x)
    bad = np.nonzero(got.view(np.int64) != ref.view(np.int64))[0]
    assert len(bad) == 0, [(x[i], got[i], ref[i]) for i in bad[:5]]


@pytest.mark.parametrize("lo,hi", [(-25.0, 0.0), (-745.0, 709.0)])
def test_survey_against_glibc_and_accurate_step(lib, lo, hi):
    n = 4_000_000
    dg, dg1, da = C.c_long(), C.c_long(), C.c_long()
    lib.crexp_survey(lo, hi, n, 12345, C.byref(dg), C.byref(dg1), C.byref(da))
    assert da.value == 0            # fast step == accurate step whenever it answers
    assert dg1.value == 0           # glibc is never more than one ulp away
    assert dg.value < n * 2e-3      # glibc's misrounding rate (about 8 in 10^4 here)
    print(f"[{lo}, {hi}): {dg.value} of {n} differ from glibc by one ulp")
