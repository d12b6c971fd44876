"""CPU tests of the oracle (the checker): the C restatement against the golden
vectors made by the reference's compiled MEX routines, against the compiled
routines themselves, and against known answers derived from the formulas."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLD = os.path.join(os.path.dirname(__file__), "golden")
P = po.P


def gold(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def same(a, b):
    """Bitwise equality up to the sign of zero."""
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


# ---------------------------------------------------------------- golden vectors

def test_golden_deformedlength():
    g = gold("deformedlength")
    nB, nN = len(g["L0"]), g["x"].shape[0]
    out = {k: np.zeros(nB) for k in ("L", "dX", "dY", "dZ", "s")}
    po.lib().orc_deformedlength(P(np.asfortranarray(g["x"])), P(np.asfortranarray(g["bl"])), P(g["L0"]),
                                nB, nN, P(out["L"]), P(out["dX"]), P(out["dY"]), P(out["dZ"]), P(out["s"]))
    for k in out:
        assert same(out[k], g[k]), k


def test_golden_bsfexponential():
    g = gold("bsfexponential")
    n = len(g["s"])
    bsf, BSF, flag = np.zeros(n), g["BSF0"].copy(), g["flag0"].copy()
    po.lib().orc_bsf_exponential(P(g["s"]), P(g["s0"]), 1, P(g["sc"]), 1, float(g["k"]), float(g["alpha"]),
                                 P(bsf), P(BSF), P(g["BT"]), P(flag), n)
    assert same(bsf, g["bsf"]) and same(BSF, g["BSF"]) and same(flag, g["flag"])
    # the vectors exercise every branch
    s, s0, sc, BT = g["s"], g["s0"], g["sc"], g["BT"]
    assert ((BT == 0) & (s > s0) & (s <= sc)).sum() > 100
    assert ((BT == 0) & (s > sc)).sum() > 100
    assert ((BT != 0)).sum() > 100


def test_golden_bondforces():
    g = gold("bondforces")
    n = len(g["s"])
    f = {k: np.zeros(n) for k in ("fX", "fY", "fZ")}
    po.lib().orc_bondforces(P(f["fX"]), P(f["fY"]), P(f["fZ"]), P(g["fail"]), P(g["dX"]), P(g["dY"]),
                            P(g["dZ"]), P(g["L"]), P(g["s"]), P(g["sp"]), P(g["BS"]), float(g["V"]),
                            P(g["VCF"]), P(g["BSF"]), n)
    for k in f:
        assert same(f[k], g[k]), k
    assert np.all(g["fX"][:3] == 0)   # NaN guard exercised


@pytest.mark.parametrize("chunks,key", [(8, "F_omp"), (1, "F_serial")])
def test_golden_nodalforces(chunks, key):
    g = gold("nodalforces")
    nN, nB = int(g["nN"]), len(g["fX"])
    F = np.zeros((nN, 3), order="F")
    po.lib().orc_nodalforces_chunked(nB, nN, P(np.asfortranarray(g["bl"])), P(F), P(g["fX"]), P(g["fY"]),
                                     P(g["fZ"]), chunks)
    assert same(F, g[key])


def test_golden_nodalforces_order_matters():
    """The 8-chunk order differs from the serial order in the last bits: the
    vectors do pin the summation order, not just the sum."""
    g = gold("nodalforces")
    assert not np.array_equal(g["F_omp"], g["F_serial"])
    np.testing.assert_allclose(g["F_omp"], g["F_serial"], rtol=1e-9, atol=1e-3)


def test_golden_eulercromer():
    g = gold("eulercromer")
    nN = g["F"].shape[0]
    a = np.zeros((nN, 3), order="F")
    v, u, x = (np.asfortranarray(g[k]).copy(order="F") for k in ("v0", "u0", "u0"))
    x[:] = 0
    po.lib().orc_eulercromer(P(a), P(np.asfortranarray(g["F"])), float(g["D"]), P(v), P(g["rho"]),
                             P(np.asfortranarray(g["CF"])), float(g["dt"]), P(u), P(x),
                             P(np.asfortranarray(g["X"])), nN, 3)
    assert same(a, g["a"]) and same(v, g["v"]) and same(u, g["u"]) and same(x, g["x"])


@pytest.mark.parametrize("ff", [0, 1])
def test_golden_bondfailure(ff):
    g = gold("bondfailure")
    n = len(g["s"])
    f = g["fail0"].copy()
    po.lib().orc_bondfailure(P(f), float(ff), P(g["BT"]), P(g["s"]), P(np.array([float(g["sc"])])), 0,
                             float(g["scSteel"]), n)
    assert same(f, g[f"fail_ff{ff}"])


def _loop_input(g):
    keys = ("undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH", "BONDSTIFFNESS",
            "VOLUMECORRECTIONFACTORS", "DENSITY", "massVector", "CONSTRAINTFLAG", "BODYFORCEFLAG")
    inp = {k: np.asfortranarray(g[k]) for k in keys}
    inp.update(nNodes=int(g["nNodes"]), nBonds=int(g["nBonds"]), DT=float(g["DT"]),
               cellVolume=float(g["cellVolume"]))
    return inp


def test_golden_loop_restated():
    g = gold("loop_ec_exponential")
    r = po.Run(_loop_input(g), kernels="restated", law="exponential", scheme="eulercromer",
               rate=float(g["rate"]), sc=2e-3, s0=1e-4)
    r.step(int(g["steps"]))
    for f in ("displacement", "velocity", "force", "deformed", "acceleration", "bsf", "flag", "fail"):
        assert same(r.get(f), g["out_" + f]), f
    assert g["out_flag"].sum() > 0 and (g["out_bsf"] == 1).sum() > 0, "fixture should soften and break bonds"


# ------------------------------------------------ restatement vs compiled reference

needs_ref = pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built (reference tree absent)")


@needs_ref
@pytest.mark.parametrize("law", ["exponential", "linear"])
def test_loop_restated_equals_reference_mex(law):
    from bb_pd_b200 import beam
    inp = beam.build(beam.small(nx=16, ny=4, nz=5))
    kw = dict(law=law, scheme="eulercromer", rate=-3e-6, sc=1.5e-3)
    a, b = po.Run(inp, kernels="restated", **kw), po.Run(inp, kernels="reference", **kw)
    a.step(120)
    b.step(120)
    for f in ("displacement", "force", "bsf", "flag", "fail", "velocity"):
        assert same(a.get(f), b.get(f)), f


# ---------------------------------------------------------------- known answers

def _bonds(nx=5, ny=4, nz=4, dx=1e-3):
    from tests.golden.make_golden import lattice
    X, bl = lattice(nx, ny, nz, dx)
    i, j = bl[:, 0].astype(int) - 1, bl[:, 1].astype(int) - 1
    L0 = np.sqrt(((X[i] - X[j]) ** 2).sum(1))
    return X, bl, L0


def test_kat_uniform_stretch():
    """Affine stretch x = (1 + e) X: every bond has stretch e, force c V VCF e d/L."""
    X, bl, L0 = _bonds()
    e = 1e-4
    x = np.asfortranarray(X * (1 + e))
    nB, nN = len(bl), len(X)
    o = {k: np.zeros(nB) for k in ("L", "dX", "dY", "dZ", "s")}
    po.lib().orc_deformedlength(P(x), P(bl), P(L0), nB, nN, *(P(o[k]) for k in ("L", "dX", "dY", "dZ", "s")))
    np.testing.assert_allclose(o["s"], e, rtol=1e-9)
    c, V = 3e18, 1e-9
    f = {k: np.zeros(nB) for k in ("fX", "fY", "fZ")}
    ones, zeros = np.ones(nB), np.zeros(nB)
    po.lib().orc_bondforces(P(f["fX"]), P(f["fY"]), P(f["fZ"]), P(ones), P(o["dX"]), P(o["dY"]), P(o["dZ"]),
                            P(o["L"]), P(o["s"]), P(zeros), P(np.full(nB, c)), V, P(ones), P(zeros), nB)
    np.testing.assert_allclose(f["fX"], c * V * o["s"] * o["dX"] / o["L"], rtol=1e-12)


def _trilinear(s, s0=1e-4, s1=3e-4, sc=2e-3, BSF=None):
    n = len(s)
    s = np.asarray(s, dtype=np.float64)
    B = np.zeros(n) if BSF is None else BSF.copy()
    flag = np.zeros(n)
    po.lib().orc_bsf_trilinear(P(s), P(np.array([s0])), 0, P(np.array([s1])), 0, P(np.array([sc])), 0, 0.25,
                               P(B), P(np.zeros(n)), P(flag), n)
    return B, flag


def test_kat_trilinear_continuity():
    s0, s1, sc, beta = 1e-4, 3e-4, 2e-3, 0.25
    eps = 1e-12
    B, flag = _trilinear([s0 + eps, s1, s1 + eps, sc, sc + eps, s0 - eps])
    assert abs(B[0]) < 1e-6 and flag[0] == 1          # 0 at the elastic limit
    assert abs(B[1] - (1 - beta * s0 / s1)) < 1e-12    # both branches meet 1 - beta s0/s1 at s1
    assert abs(B[2] - (1 - beta * s0 / s1)) < 1e-8
    assert abs(B[3] - 1) < 1e-12 and B[4] == 1          # reaches 1 at sc, 1 beyond
    assert B[5] == 0 and flag[5] == 0


def test_kat_exponential_endpoints():
    n = 3
    s = np.array([1e-4 + 1e-13, 2e-3, 2e-3 + 1e-9])
    bsf, B, flag = np.zeros(n), np.zeros(n), np.zeros(n)
    po.lib().orc_bsf_exponential(P(s), P(np.array([1e-4])), 0, P(np.array([2e-3])), 0, 25.0, 0.25, P(bsf), P(B),
                                 P(np.zeros(n)), P(flag), n)
    assert abs(B[0]) < 1e-8 and abs(B[1] - 1) < 1e-9 and B[2] == 1


def test_kat_irreversible():
    """Loading into softening then unloading never lowers the damage."""
    s_hist = [5e-4, 1e-3, 2e-4, 0.0, -1e-4, 8e-4]
    B = np.zeros(1)
    seen = 0.0
    for s in s_hist:
        B, _ = _trilinear([s], BSF=B)
        assert B[0] >= seen
        seen = B[0]
    assert seen > 0.5


def test_kat_smoothstep():
    L = po.lib()
    assert L.orc_smoothstep(1, 1, 100, 0.0, -1e-3) == 0.0
    assert abs(L.orc_smoothstep(100, 1, 100, 0.0, -1e-3) + 1e-3) < 1e-18
    h = 1e-6
    for t in (1.0, 100.0):
        slope = (L.orc_smoothstep(t + h, 1, 100, 0, 1) - L.orc_smoothstep(t - h, 1, 100, 0, 1)) / (2 * h)
        assert abs(slope) < 1e-6


def test_kat_newton_third_law():
    """Sum of nodal forces of a free body is zero (to rounding)."""
    X, bl, L0 = _bonds()
    rng = np.random.default_rng(1)
    x = np.asfortranarray(X + rng.normal(0, 1e-6, X.shape))
    nB, nN = len(bl), len(X)
    o = {k: np.zeros(nB) for k in ("L", "dX", "dY", "dZ", "s")}
    po.lib().orc_deformedlength(P(x), P(bl), P(L0), nB, nN, *(P(o[k]) for k in ("L", "dX", "dY", "dZ", "s")))
    f = {k: np.zeros(nB) for k in ("fX", "fY", "fZ")}
    ones, zeros = np.ones(nB), np.zeros(nB)
    po.lib().orc_bondforces(P(f["fX"]), P(f["fY"]), P(f["fZ"]), P(ones), P(o["dX"]), P(o["dY"]), P(o["dZ"]),
                            P(o["L"]), P(o["s"]), P(zeros), P(np.full(nB, 3e18)), 1e-9, P(ones), P(zeros), nB)
    F = np.zeros((nN, 3), order="F")
    po.lib().orc_nodalforces_chunked(nB, nN, P(bl), P(F), P(f["fX"]), P(f["fY"]), P(f["fZ"]), 8)
    scale = np.abs(F).max()
    assert np.all(np.abs(F.sum(0)) < 1e-9 * scale * nN)


def test_kat_eulercromer_two_nodes():
    F = np.asfortranarray([[2.0, 0, 0], [-2.0, 0, 0]])
    v = np.zeros((2, 3), order="F")
    u = np.zeros((2, 3), order="F")
    a = np.zeros((2, 3), order="F")
    X = np.asfortranarray([[0.0, 0, 0], [1.0, 0, 0]])
    x = np.zeros((2, 3), order="F")
    CF = np.asfortranarray([[0.0, 0, 0], [1.0, 0, 0]])
    po.lib().orc_eulercromer(P(a), P(F), 0.0, P(v), P(np.array([2.0, 2.0])), P(CF), 0.5, P(u), P(x), P(X), 2, 3)
    assert a[0, 0] == 1.0 and v[0, 0] == 0.5 and u[0, 0] == 0.25 and x[0, 0] == 0.25
    assert a[1, 0] == 0 and u[1, 0] == 0 and x[1, 0] == 1.0


def test_kat_adr_damping():
    nN = 64
    z = np.zeros((nN, 3), order="F")
    m = np.ones(nN)
    rng = np.random.default_rng(2)
    F = np.asfortranarray(rng.normal(size=(nN, 3)))
    L = po.lib()
    assert L.orc_damping_coefficient_tree(P(F), P(m), P(z), 1.0, P(z), P(z), nN) == 0.0  # u = 0 -> cn = 0
    assert L.orc_cn_from_sums(4.0, 1.0) == 1.9        # 2 sqrt(4) = 4 > 2 -> 1.9
    assert L.orc_cn_from_sums(0.25, 1.0) == 1.0
    assert L.orc_cn_from_sums(-1.0, 1.0) == 0.0


def test_tree_sum_order():
    """orc_tree_sum follows its documented pairing (restated here in numpy)."""
    rng = np.random.default_rng(3)

    def level(x):
        m = -(-len(x) // 32)
        v = np.zeros(m * 32)
        v[:len(x)] = x
        v = v.reshape(m, 32)
        for off in (16, 8, 4, 2, 1):
            v = v + v[:, np.arange(32) ^ off]
        return v[:, 0]

    for n in (1, 31, 32, 33, 1000, 1025, 40000, 70001, 1280000):
        t = rng.normal(size=n) * 10.0 ** rng.integers(-8, 8, n)
        p = level(t)
        while len(p) > 1:
            p = level(p)
        assert po.tree_sum(t) == p[0]
        assert abs(p[0] - t.sum()) <= 1e-12 * np.abs(t).sum()


def test_chunk_rule_matches_libgomp(tmp_path):
    """The static-schedule rule used for the nodal-force order equals what
    libgomp does (the reference forces 8 threads)."""
    src = tmp_path / "probe.c"
    src.write_text(r'''
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
int main(int c, char **v) { int n = atoi(v[1]); int lo[8], hi[8];
 for (int i = 0; i < 8; i++) lo[i] = hi[i] = -1;
 omp_set_num_threads(8);
#pragma omp parallel
 { int id = omp_get_thread_num();
#pragma omp for
   for (int k = 0; k < n; k++) { if (lo[id] < 0) lo[id] = k; hi[id] = k + 1; } }
 for (int i = 0; i < 8; i++) printf("%d %d\n", lo[i], hi[i]); return 0; }''')
    import subprocess
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-fopenmp", "-O1", str(src), "-o", str(exe)], check=True)
    for n in (7, 8, 17, 1000, 1005544):
        out = subprocess.run([str(exe), str(n)], check=True, capture_output=True, text=True).stdout.split()
        got = [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(8)]
        for c in range(8):
            lo, hi = po.chunk_range(n, 8, c)
            if lo == hi:
                assert got[c] == (-1, -1)
            else:
                assert got[c] == (lo, hi)


def test_damage_known_answers():
    """calculatedamage.m:29-45: 1 - (intact bonds) / family size; a family
    counted before bonds were removed (a notch) leaves damage where no bond
    ever broke."""
    bl = np.asfortranarray(np.array([[1, 2], [1, 3], [2, 3], [3, 4]], dtype=np.float64))
    fail = np.array([1.0, 0.0, 1.0, 1.0])
    nfam = np.array([2.0, 2.0, 3.0, 2.0])          # node 4 lost one bond to a notch
    dmg = np.zeros(4)
    po.lib().orc_damage(po.P(bl), po.P(fail), po.P(nfam), 4, 4, po.P(dmg))
    assert list(dmg) == [0.5, 0.0, 1 - 2 / 3, 0.5]


def _energy_formula(bs, s0, sc, L0, s, k, alpha, V):
    """calculatedamageenergy.m:36-55 for one bond, written out again."""
    den = 2 * k * (np.exp(k) - 1) * (1 + alpha)
    shape = (2 * k) - (2 * np.exp(k)) + (alpha * k) - (alpha * k * np.exp(k)) + 2
    if s0 < s <= sc:
        return (bs * s0 * L0 * (s0 - s) * shape / den) * V ** 2
    if s > sc:
        return (bs * s0 * L0 * (s0 - sc) * shape / den) * V ** 2
    return 0.0


def test_damageenergy_known_answers():
    """calculatedamageenergy.m:34-62: nothing below s0, growing with the
    stretch in the softening range, the value at sc above it, and never
    lower than the energy already dissipated (unloading keeps it; a NaN
    stretch adds nothing)."""
    k, alpha, V = 25.0, 0.25, 1.25e-7
    s0, sc = 1e-4, 2e-3
    s = np.array([0.0, 1e-4, 1.5e-4, 1e-3, 2e-3, 5e-3, np.nan])
    n = s.size
    bs, L0 = np.full(n, 3.1e18), np.full(n, 2.5e-3)
    S0, SC = np.full(n, s0), np.full(n, sc)
    e = np.zeros(n)
    po.lib().orc_damageenergy(po.P(bs), po.P(S0), po.P(SC), po.P(L0), po.P(s), k, alpha, V, po.P(e), n)
    want = [_energy_formula(bs[0], s0, sc, L0[0], x, k, alpha, V) for x in s]
    np.testing.assert_allclose(e, want, rtol=1e-14, atol=0)
    assert e[0] == 0 and e[1] == 0 and e[6] == 0
    assert 0 < e[2] < e[3] < e[4] and e[4] == e[5]
    # unloading: a smaller stretch leaves the dissipated energy unchanged
    before = e.copy()
    s2 = np.full(n, 1.2e-4)
    po.lib().orc_damageenergy(po.P(bs), po.P(S0), po.P(SC), po.P(L0), po.P(s2), k, alpha, V, po.P(e), n)
    assert np.array_equal(e[:6], np.maximum(before[:6], e[:6])) and np.array_equal(e[3:6], before[3:6])
    assert e[0] > 0 and e[0] == e[1] == e[6]


def _builder_case(**kw):
    from bb_pd_b200 import beam
    return beam.build(beam.small(nx=12, ny=4, nz=5, **kw))


def test_builder_oracle_matches_lattice_builder():
    """The brute-force restatement of buildhorizons.m, the volume correction,
    buildbonddata.m and buildmassmatrix.m gives the lattice builder's arrays
    bit for bit (both list families by node id)."""
    inp = _builder_case()
    X, n, nb = inp["undeformedCoordinates"], inp["nNodes"], inp["nBonds"]
    L = po.lib()
    fam, fptr = np.zeros(n), np.zeros(n)
    assert L.orc_buildhorizons(po.P(X), n, inp["horizon"], 0, po.P(fam), po.P(fptr), None, None, None) == nb
    bl, L0, family = np.zeros((nb, 2), order="F"), np.zeros(nb), np.zeros(2 * nb)
    assert L.orc_buildhorizons(po.P(X), n, inp["horizon"], nb, po.P(fam), po.P(fptr), po.P(family),
                               po.P(bl), po.P(L0)) == nb
    assert np.array_equal(bl, inp["BONDLIST"]) and np.array_equal(L0, inp["UNDEFORMEDLENGTH"])
    assert np.array_equal(fam, inp["nFAMILYMEMBERS"])
    assert fptr[0] == 1 and np.array_equal(np.diff(fptr), fam[:-1])
    for i in (0, n // 2, n - 1):                  # families by ascending node id, bonds both ways
        f = family[int(fptr[i]) - 1:int(fptr[i] + fam[i]) - 1]
        assert np.all(np.diff(f) > 0)
        mine = np.concatenate([bl[bl[:, 0] == i + 1, 1], bl[bl[:, 1] == i + 1, 0]])
        assert np.array_equal(np.sort(mine), f)
    vcf = np.zeros(nb)
    L.orc_volumecorrection(po.P(L0), nb, inp["horizon"], 5e-3 / 2, po.P(vcf))
    assert np.array_equal(vcf, inp["VOLUMECORRECTIONFACTORS"])
    VH = (4.0 / 3.0) * np.pi * inp["horizon"] ** 3
    bs, bt, bfm, sf = (np.zeros(nb) for _ in range(4))
    assert L.orc_bonddata(po.P(bl), nb, po.P(fam), None, inp["bondStiffnessConcrete"], 0.0, inp["cellVolume"],
                          VH, po.P(bs), po.P(bt), po.P(bfm), po.P(sf)) == 0
    assert np.array_equal(bs, inp["BONDSTIFFNESS"]) and not bt.any() and np.all(bfm == 1)
    mass = np.zeros(n)
    L.orc_massmatrix(n, 5e-3, inp["bondStiffnessConcrete"], inp["DT"], po.P(fam), po.P(mass))
    assert np.array_equal(mass, inp["massVector"])


def test_builder_oracle_bond_types_and_notch():
    """buildbonddata.m's material table (concrete, interface x3, steel) and
    buildnotch.m's removal of the bonds crossing the notch rectangle, checked
    against the lattice builder's notch and a direct segment test."""
    L = po.lib()
    inp = _builder_case()
    X, n, nb, bl = inp["undeformedCoordinates"], inp["nNodes"], inp["nBonds"], inp["BONDLIST"]
    fam = inp["nFAMILYMEMBERS"]
    mat = (X[:, 2] > 0.016).astype(np.float64)
    bs, bt, bfm, sf = (np.zeros(nb) for _ in range(4))
    assert L.orc_bonddata(po.P(bl), nb, po.P(fam), po.P(mat), 2.0, 7.0, 1.0, 1.0, po.P(bs), po.P(bt),
                          po.P(bfm), po.P(sf)) == 0
    mi, mj = mat[bl[:, 0].astype(int) - 1], mat[bl[:, 1].astype(int) - 1]
    assert np.array_equal(bt, mi + mj) and np.array_equal(bfm, np.where(bt == 1, 3.0, 1.0))
    assert np.array_equal(bs, sf * np.where(bt == 2, 7.0, 2.0))
    bad = mat.copy()
    bad[3] = 0.5
    assert L.orc_bonddata(po.P(bl), nb, po.P(fam), po.P(bad), 2.0, 7.0, 1.0, 1.0, po.P(bs), po.P(bt),
                          po.P(bfm), po.P(sf)) == -1
    # notch at x = 6.5 dx, 2.3 dx deep: the lattice builder's rectangle runs
    # from the bottom node layer (z = dx) to dx/2 + depth
    dx = 5e-3
    notched = _builder_case(notch_x=6.5 * dx, notch_depth=1.8 * dx)
    blo, L0o = np.zeros((nb, 2), order="F"), np.zeros(nb)
    famo, fptr, family = np.zeros(n), np.zeros(n), np.zeros(2 * nb)
    m = L.orc_buildnotch(po.P(X), n, po.P(bl), po.P(inp["UNDEFORMEDLENGTH"]), nb, dx, 6.5, 2.3,
                         po.P(blo), po.P(L0o), po.P(famo), po.P(fptr), po.P(family))
    assert m == notched["nBonds"] < nb
    assert np.array_equal(blo.ravel(order="F")[:2 * m], notched["BONDLIST"].ravel(order="F"))
    assert np.array_equal(L0o[:m], notched["UNDEFORMEDLENGTH"])
    assert np.array_equal(famo, notched["nFAMILYMEMBERS"])
    i0 = int(np.argmax(famo))                       # family of a node in bond order of the reduced list
    f = family[int(fptr[i0]) - 1:int(fptr[i0] + famo[i0]) - 1]
    blm = np.asfortranarray(blo.ravel(order="F")[:2 * m].reshape((m, 2), order="F"))
    want = [b if a == i0 + 1 else a for a, b in blm if a == i0 + 1 or b == i0 + 1]
    assert list(f) == want
