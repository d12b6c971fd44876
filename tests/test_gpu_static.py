"""GPU static (implicit) solver against the oracle's restatement of the
reference's displacement-controlled Newton-Raphson (oracle/static_oracle.py,
direct sparse solves). The GPU solves each linear system by a preconditioned
conjugate gradient to a relative residual of 1e-13, so displacements agree to a
tolerance: 1e-8 of the largest displacement while the beam is elastic, 1e-6
through softening, with identical softening and broken-bond sets."""
import numpy as np
import pytest

import bb_pd_b200 as bb
from bb_pd_b200.static import StaticSolver
from oracle.static_oracle import StaticOracle

pytestmark = pytest.mark.gpu
CG = dict(cg_tol=1e-13, max_cg=200000)


def test_static_elastic_vs_oracle():
    inp = bb.beam.build(bb.beam.small(nx=20, ny=4, nz=6))
    g = StaticSolver(inp, law="linear", sc=1.0)
    o = StaticOracle(inp, law="linear", sc=1.0)
    for step in range(3):
        sg = g.step(-1e-6, tol=1e-9, **CG)
        so = o.step(-1e-6, tol=1e-9)
        assert sg.converged and so["converged"], (step, sg.residual, sg.reaction)
        ug, uo = g.get("displacement"), o.get("displacement")
        scale = np.abs(uo).max()
        assert np.abs(ug - uo).max() <= 1e-8 * scale, step
        np.testing.assert_allclose(sg.reaction, so["reaction"], rtol=1e-6)
    # equilibrium: no net force on the free DOFs, the held DOFs carry the load
    F = g.get("force")
    assert abs(F[:, 2].sum()) <= 1e-9 * np.abs(F).max()
    assert same_flags(g.get("fail"), np.ones(inp["nBonds"]))
    g.close()


def same_flags(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


def test_static_softening_vs_oracle():
    """Notched beam, bilinear law (the reference's static driver uses
    calculatebondsofteningfactor with sc = 25 s0): five load steps take it into
    softening and the first bond failures."""
    dx = 5e-3
    inp = bb.beam.build(bb.beam.small(nx=24, ny=4, nz=8, notch_x=12.5 * dx, notch_depth=3.2 * dx))
    kw = dict(law="bilinear", s0=1e-4, sc=2.5e-3)
    g = StaticSolver(inp, **kw)
    o = StaticOracle(inp, **kw)
    for step in range(6):
        sg = g.step(-1e-5, tol=1e-6, max_newton=60, **CG)
        so = o.step(-1e-5, tol=1e-6, max_newton=60)
        assert sg.converged and so["converged"], step
        ug, uo = g.get("displacement"), o.get("displacement")
        assert np.abs(ug - uo).max() <= 1e-6 * np.abs(uo).max(), step
        assert same_flags(g.get("flag"), o.get("flag")), step
        assert same_flags(g.get("fail"), o.get("fail")), step
        np.testing.assert_allclose(g.get("bsf"), o.get("bsf"), rtol=0, atol=1e-6)
    assert g.get("flag").sum() > 100 and (g.get("fail") == 0).any()
    g.close()


def test_static_linearity_and_validation():
    inp = bb.beam.build(bb.beam.small(nx=16, ny=4, nz=5))
    a = StaticSolver(inp, law="linear", sc=1.0)
    b = StaticSolver(inp, law="linear", sc=1.0)
    a.step(-1e-7, tol=1e-10, **CG)
    b.step(-2e-7, tol=1e-10, **CG)
    ua, ub = a.get("displacement"), b.get("displacement")
    assert np.abs(ub - 2 * ua).max() <= 1e-5 * np.abs(ub).max()
    with pytest.raises(bb.BBPDError):
        a.step(-1e-7, tol=0.0)
    with pytest.raises(bb.BBPDError):
        a.get("velocity")
    bad_inp = dict(inp)
    bad_inp["BONDTYPE"] = np.full(inp["nBonds"], 4.0)
    with pytest.raises(bb.BBPDError):
        StaticSolver(bad_inp, law="linear", sc=1.0)
    a.close()
    b.close()


@pytest.mark.parametrize("nod", [3, 2])
def test_stiffness_triplets_vs_oracle(nod):
    """buildstiffnessmatrixCSCformat.m on the GPU: triplets (find order, failed
    bonds skipped, exact zeros dropped) and massVector bit-identical to the
    oracle's literal restatement, on deformed coordinates with damaged,
    interface and broken bonds."""
    from oracle import pyoracle as po
    P = po.P
    inp = bb.beam.build(bb.beam.small(nx=18, ny=4, nz=5))
    rng = np.random.default_rng(4)
    n, nB = inp["nNodes"], inp["nBonds"]
    X = np.asfortranarray(inp["undeformedCoordinates"][:, :nod] + rng.normal(0, 1e-5, (n, nod)))
    bl = inp["BONDLIST"]
    fail = (rng.random(nB) > 0.1).astype(np.float64)
    bsf = np.where(rng.random(nB) < 0.3, rng.random(nB), 0.0)
    bfm = np.where(rng.random(nB) < 0.2, 3.0, 1.0)
    vcf, bs, V = inp["VOLUMECORRECTIONFACTORS"], inp["BONDSTIFFNESS"], inp["cellVolume"]
    from bb_pd_b200.static import buildstiffnessmatrixCSCformat
    r, c, v, m = buildstiffnessmatrixCSCformat(X, bl, vcf, V, bs, bfm, fail, bsf, inp["UNDEFORMEDLENGTH"])
    L = po.lib()
    tot = L.orc_stiffness_coo(P(X), n, nod, P(bl), P(vcf), V, P(bs), P(bfm), P(fail), P(bsf), nB, 0, None, None,
                              None, None)
    orr, occ, ov, om = np.zeros(tot), np.zeros(tot), np.zeros(tot), np.zeros(n)
    L.orc_stiffness_coo(P(X), n, nod, P(bl), P(vcf), V, P(bs), P(bfm), P(fail), P(bsf), nB, tot, P(orr), P(occ),
                        P(ov), P(om))
    assert r.size == tot > 0
    for a, b in ((r, orr), (c, occ), (v, ov), (m, om)):
        assert np.array_equal(a, b)
    assert r.size <= (2 * nod) ** 2 * int(fail.sum())


@pytest.mark.parametrize("law,steps", [("trilinear", 4), ("exponential", 3)])
def test_static_other_laws_vs_oracle(law, steps):
    """The static solver with the trilinear and exponential laws against the
    oracle (its C law routines inside the restated Newton loop)."""
    dx = 5e-3
    inp = bb.beam.build(bb.beam.small(nx=24, ny=4, nz=8, notch_x=12.5 * dx, notch_depth=3.2 * dx))
    kw = dict(law=law, s0=1e-4, sc=2e-3)
    g = StaticSolver(inp, **kw)
    o = StaticOracle(inp, **kw)
    for step in range(steps):
        sg = g.step(-1e-5, tol=1e-6, max_newton=60, **CG)
        so = o.step(-1e-5, tol=1e-6, max_newton=60)
        assert sg.converged and so["converged"], step
        ug, uo = g.get("displacement"), o.get("displacement")
        assert np.abs(ug - uo).max() <= 1e-6 * np.abs(uo).max(), step
        assert same_flags(g.get("flag"), o.get("flag")), step
        assert same_flags(g.get("fail"), o.get("fail")), step
    assert g.get("flag").sum() > 100
    g.close()
