"""GPU parity of the per-routine entry points (one per reference MEX routine)
against the golden vectors of the reference's compiled MEX code and against the
oracle restatement. Bar: bit-identical (up to the sign of zero); the
exponential law within 1e-12 relative (CUDA's exp may differ from glibc's in
the last bit)."""
import os

import numpy as np
import pytest

import bb_pd_b200 as bb
from bb_pd_b200 import routines as R
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
P = po.P
EXP_RTOL = 1e-12


def gold(name):
    return {k: (np.asfortranarray(v) if isinstance(v, np.ndarray) and v.ndim == 2 else v)
            for k, v in np.load(os.path.join(GOLD, name + ".npz")).items()}


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def test_deformedlength_golden():
    g = gold("deformedlength")
    nB = len(g["L0"])
    o = {k: np.zeros(nB) for k in ("L", "dX", "dY", "dZ", "s")}
    R.calculatedeformedlengthMex(g["x"], g["bl"], g["L0"], o["L"], o["dX"], o["dY"], o["dZ"], o["s"])
    for k in o:
        assert same(o[k], g[k]), k


def test_bsfexponential_golden():
    g = gold("bsfexponential")
    n = len(g["s"])
    bsf, BSF, flag = np.zeros(n), g["BSF0"].copy(), g["flag0"].copy()
    R.calculatebsfexponentialMex(g["s"], g["s0"], g["sc"], float(g["k"]), float(g["alpha"]), bsf, BSF, g["BT"], flag)
    assert same(flag, g["flag"])
    np.testing.assert_allclose(BSF, g["BSF"], rtol=EXP_RTOL, atol=0)
    np.testing.assert_allclose(bsf, g["bsf"], rtol=EXP_RTOL, atol=0)
    assert np.array_equal(BSF == 1, g["BSF"] == 1)        # broken set identical
    # the device exp is correctly rounded; glibc's misrounds about 8 in 10^4
    # arguments, so nearly every value is bit-identical
    differ = int(np.sum(bsf.view(np.int64) != g["bsf"].view(np.int64)))
    print(f"bsf values differing from the compiled reference: {differ} of {n}")
    assert differ <= max(2, n // 200)


def test_bondforces_golden():
    g = gold("bondforces")
    n = len(g["s"])
    f = {k: np.zeros(n) for k in ("fX", "fY", "fZ")}
    R.calculatebondforcesMex(f["fX"], f["fY"], f["fZ"], g["fail"], g["dX"], g["dY"], g["dZ"], g["L"], g["s"],
                             g["sp"], g["BS"], float(g["V"]), g["VCF"], g["BSF"])
    for k in f:
        assert same(f[k], g[k]), k


@pytest.mark.parametrize("fn,key", [("calculatenodalforcesopenmpMex", "F_omp"), ("calculatenodalforcesMex", "F_serial")])
def test_nodalforces_golden(fn, key):
    g = gold("nodalforces")
    nN = int(g["nN"])
    F = np.zeros((nN, 3), order="F")
    getattr(R, fn)(g["bl"], F, g["fX"], g["fY"], g["fZ"])
    assert same(F, g[key])
    # accumulates into the existing nodalForce like the reference (+=)
    F2 = np.asfortranarray(np.ones((nN, 3)))
    Fo = F2.copy(order="F")
    po.lib().orc_nodalforces_chunked(len(g["fX"]), nN, P(g["bl"]), P(Fo), P(g["fX"]), P(g["fY"]), P(g["fZ"]),
                                     8 if key == "F_omp" else 1)
    getattr(R, fn)(g["bl"], F2, g["fX"], g["fY"], g["fZ"])
    assert same(F2, Fo)


def test_nodalforces_large_random():
    """A bond list much larger than the chunk count, in a shuffled order."""
    inp = bb.beam.build(bb.beam.small(nx=30, ny=6, nz=6))
    rng = np.random.default_rng(5)
    perm = rng.permutation(inp["nBonds"])
    bl = np.asfortranarray(inp["BONDLIST"][perm])
    nB, nN = inp["nBonds"], inp["nNodes"]
    fX, fY, fZ = (rng.normal(0, 1e6, nB) for _ in range(3))
    for T, fn in ((8, R.calculatenodalforcesopenmpMex), (1, R.calculatenodalforcesMex)):
        F = np.zeros((nN, 3), order="F")
        Fo = np.zeros((nN, 3), order="F")
        fn(bl, F, fX, fY, fZ)
        po.lib().orc_nodalforces_chunked(nB, nN, P(bl), P(Fo), P(fX), P(fY), P(fZ), T)
        assert same(F, Fo)


def test_eulercromer_golden():
    g = gold("eulercromer")
    nN = g["F"].shape[0]
    a = np.zeros((nN, 3), order="F")
    v, u = g["v0"].copy(order="F"), g["u0"].copy(order="F")
    x = np.zeros((nN, 3), order="F")
    R.timeintegrationeulercromerMex(a, g["F"], float(g["D"]), v, g["rho"], g["CF"], float(g["dt"]), u, x, g["X"])
    for k, arr in (("a", a), ("v", v), ("u", u), ("x", x)):
        assert same(arr, g[k]), k


@pytest.mark.parametrize("ff", [0, 1])
def test_bondfailure_golden(ff):
    g = gold("bondfailure")
    f = g["fail0"].copy()
    R.calculatebondfailureMex(f, float(ff), g["BT"], g["s"], float(g["sc"]), float(g["scSteel"]))
    assert same(f, g[f"fail_ff{ff}"])


def _stretches(n, rng):
    from tests.golden.make_golden import stretch_sample
    return stretch_sample(rng, n, 1e-4, 2e-3)


def test_trilinear_vs_oracle():
    rng = np.random.default_rng(7)
    n = 5000
    s = np.concatenate([_stretches(n - 3, rng), [3e-4, np.nextafter(3e-4, 1), np.nextafter(3e-4, 0)]])
    BT = rng.choice([0.0, 1.0], n, p=[0.9, 0.1])
    B0 = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
    f0 = (rng.random(n) < 0.2).astype(np.float64)
    B, f = B0.copy(), f0.copy()
    R.calculatebsftrilinear(s, 1e-4, 3e-4, 2e-3, B, BT, f)
    Bo, fo = B0.copy(), f0.copy()
    po.lib().orc_bsf_trilinear(P(s), P(np.array([1e-4])), 0, P(np.array([3e-4])), 0, P(np.array([2e-3])), 0, 0.25,
                               P(Bo), P(BT), P(fo), n)
    assert same(B, Bo) and same(f, fo)


def test_bilinear_vs_oracle():
    rng = np.random.default_rng(8)
    n = 5000
    s = _stretches(n, rng)
    BT = rng.choice([0.0, 2.0], n, p=[0.9, 0.1])
    B0 = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
    f0 = (rng.random(n) < 0.2).astype(np.float64)
    B, f = B0.copy(), f0.copy()
    R.calculatebondsofteningfactor(s, 1e-4, 2e-3, f, B, BT)
    Bo, fo = B0.copy(), f0.copy()
    po.lib().orc_bsf_bilinear(P(s), P(np.array([1e-4])), 0, P(np.array([2e-3])), 0, P(Bo), P(BT), P(fo), n)
    assert same(B, Bo) and same(f, fo)


@pytest.mark.parametrize("nN", [1, 33, 5000, 70001])
def test_damping_coefficient_vs_oracle(nN):
    rng = np.random.default_rng(nN)
    F, Fp, vhp, u = (np.asfortranarray(rng.normal(0, s, (nN, 3))) for s in (1e6, 1e6, 1e-3, 1e-4))
    vhp[rng.random((nN, 3)) < 0.1] = 0.0           # skipped terms
    m = rng.uniform(1e4, 1e5, nN)
    dt = 1e-6
    cn = R.calculatedampingcoefficient(F, m, Fp, dt, vhp, u)
    cno = po.lib().orc_damping_coefficient_tree(P(F), P(m), P(Fp), dt, P(vhp), P(u), nN)
    assert cn == cno
    cns = po.lib().orc_damping_coefficient_seq(P(F), P(m), P(Fp), dt, P(vhp), P(u), nN)
    assert abs(cn - cns) <= 1e-12 * max(abs(cns), 1e-300) or (cn == 0 and cns == 0) or (cn == 1.9 and cns == 1.9)


@pytest.mark.parametrize("it", [1, 7])
def test_adr_integrate_vs_oracle(it):
    rng = np.random.default_rng(it)
    nN = 3000
    F, vhp, u0 = (np.asfortranarray(rng.normal(0, s, (nN, 3))) for s in (1e6, 1e-3, 1e-4))
    m = rng.uniform(1e4, 1e5, nN)
    CF = np.asfortranarray((rng.random((nN, 3)) < 0.05).astype(np.float64))
    vh, u = np.zeros((nN, 3), order="F"), u0.copy(order="F")
    R.timeintegrationADR(it, 1e-6, vh, F, m, 0.37, vhp, u, CF)
    vho, uo = np.zeros((nN, 3), order="F"), u0.copy(order="F")
    po.lib().orc_adr_integrate(it, 1e-6, P(vho), P(F), P(m), 0.37, P(vhp), P(uo), P(CF), nN)
    assert same(vh, vho) and same(u, uo)


def test_bad_bondlist_rejected():
    g = gold("nodalforces")
    bl = g["bl"].copy(order="F")
    bl[3, 1] = 0.0          # node id 0 does not exist (1-based)
    F = np.zeros((int(g["nN"]), 3), order="F")
    with pytest.raises(bb.BBPDError) as e:
        R.calculatenodalforcesopenmpMex(bl, F, g["fX"], g["fY"], g["fZ"])
    assert e.value.status == bb._native.ERR_ARG


def test_wait_timeout_selftest():
    """A device-side wait on a flag nothing sets expires and reports, without hanging."""
    import time
    t = time.time()
    rc = bb._native.lib().bbpd_selftest_wait_timeout(0.2)
    assert rc == bb._native.ERR_TIMEOUT
    assert time.time() - t < 10


def test_division_selftest():
    """The kernels' division by a shared divisor (Markstein) equals IEEE
    division bit for bit on 2e8 seeded samples, hard rounding cases included."""
    import ctypes as C
    rb, qb, n = C.c_int64(), C.c_int64(), C.c_int64()
    err = C.c_double()
    bb._native.check(bb._native.lib().bbpd_selftest_division(200_000_000, 20261203, C.byref(rb), C.byref(qb),
                                                              C.byref(n), C.byref(err)))
    print(f"samples {n.value}, rcp.approx max rel err {err.value:.3e}")
    assert n.value > 150_000_000
    assert rb.value == 0 and qb.value == 0, (rb.value, qb.value)


def test_damage_vs_oracle():
    inp = bb.beam.build(bb.beam.small(nx=20, ny=4, nz=6))
    bl, nfam = inp["BONDLIST"], inp["nFAMILYMEMBERS"]
    rng = np.random.default_rng(5)
    fail = (rng.random(inp["nBonds"]) > 0.3).astype(np.float64)
    d = R.calculatedamage(bl, fail, nfam)
    do = np.zeros(inp["nNodes"])
    po.lib().orc_damage(P(bl), P(fail), P(nfam), inp["nBonds"], inp["nNodes"], P(do))
    assert same(d, do)
    assert same(R.calculatedamage(bl, np.ones(inp["nBonds"]), nfam), np.zeros(inp["nNodes"]))
    bad = np.asfortranarray(bl.copy())
    bad[0, 0] = inp["nNodes"] + 1
    with pytest.raises(bb.BBPDError) as e:
        R.calculatedamage(bad, fail, nfam)
    assert e.value.status == bb._native.ERR_ARG


def test_damageenergy_vs_oracle():
    """calculatedamageenergy.m on the GPU, bit for bit with the oracle over
    stretches on both sides of s0 and sc (and on them), over repeated steps."""
    rng = np.random.default_rng(9)
    n = 200_003
    bs = rng.uniform(1e18, 4e18, n)
    L0 = rng.uniform(1e-3, 4e-3, n)
    s0 = np.full(n, 1e-4)
    sc = np.exp(rng.normal(np.log(2e-3), 0.1, n))
    e_gpu, e_orc = np.zeros(n), np.zeros(n)
    for step in range(4):
        st = rng.uniform(-1e-3, 4e-3, n)
        st[:1000] = s0[:1000]
        st[1000:2000] = sc[1000:2000]
        st[2000:2100] = np.nan
        R.calculatedamageenergy(bs, s0, sc, L0, st, 25, 0.25, 1.5625e-8, e_gpu)
        po.lib().orc_damageenergy(P(bs), P(s0), P(sc), P(L0), P(st), 25.0, 0.25, 1.5625e-8, P(e_orc), n)
        assert same(e_gpu, e_orc), step
    assert (e_gpu > 0).mean() > 0.5


def test_crexp_device_matches_host_build(tmp_path):
    """The device's correctly rounded exp (crexp.cuh) returns the same bits as
    the host build of the same code, which test_crexp.py pins against an
    80-digit evaluation: 10^8 arguments of the exponential law's range and
    2 * 10^7 over the whole double range; its fast step never disagrees with
    its accurate step."""
    import ctypes as C
    from test_crexp import build_host_harness
    H = build_host_harness(str(tmp_path / "libcrexp_host.so"))
    for lo, hi, n, seed in ((-25.0, 0.0, 100_000_000, 11), (-745.0, 709.7, 20_000_000, 12)):
        fv, bs = C.c_int64(), C.c_uint64()
        bb._native.check(bb._native.lib().bbpd_selftest_exp(lo, hi, n, seed, C.byref(fv), C.byref(bs)))
        assert fv.value == 0, (lo, hi, fv.value)
        assert bs.value == H.crexp_bits_sum(lo, hi, n, seed), (lo, hi)
