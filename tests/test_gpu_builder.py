"""GPU input builder (builder.cu) against the oracle's brute-force restatement
of the reference's input module and against the lattice builder: bit-identical
families, bond lists, lengths, volume corrections, bond data and masses, on
lattices (with and without a notch) and on irregular point clouds."""
import numpy as np
import pytest

import bb_pd_b200 as bb
from bb_pd_b200 import builder as G
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
P = po.P


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.array_equal(a, b))


def oracle_horizons(X, r):
    X = np.asfortranarray(X, dtype=np.float64)
    n = X.shape[0]
    L = po.lib()
    nfam, fptr = np.zeros(n), np.zeros(n)
    nb = L.orc_buildhorizons(P(X), n, r, 0, P(nfam), P(fptr), None, None, None)
    fam, bl, L0 = np.zeros(2 * nb), np.zeros((nb, 2), order="F"), np.zeros(nb)
    L.orc_buildhorizons(P(X), n, r, nb, P(nfam), P(fptr), P(fam), P(bl), P(L0))
    return nfam, fptr, fam, bl, L0


@pytest.mark.parametrize("cloud", ["jittered", "uniform", "clustered"])
def test_horizons_vs_oracle_point_clouds(cloud):
    rng = np.random.default_rng({"jittered": 1, "uniform": 2, "clustered": 3}[cloud])
    if cloud == "jittered":
        g = np.stack(np.meshgrid(np.arange(18), np.arange(9), np.arange(11), indexing="ij"), -1).reshape(-1, 3)
        X = (g + rng.uniform(-0.3, 0.3, g.shape)) * 2.5e-3
        r = 3.015 * 2.5e-3
    elif cloud == "uniform":
        X = rng.uniform(0, 1, (2500, 3)) * [2.0, 0.5, 1.0]
        r = 0.17
    else:
        c = rng.uniform(-5, 5, (12, 3))
        X = c[rng.integers(0, 12, 3000)] + rng.normal(0, 0.4, (3000, 3))
        r = 0.35
    got = G.buildhorizons(X, r)
    want = oracle_horizons(X, r)
    for name, a, b in zip(("nFAMILYMEMBERS", "NODEFAMILYPOINTERS", "NODEFAMILY", "BONDLIST", "UNDEFORMEDLENGTH"),
                          got, want):
        assert same(a, b), name
    assert got[3].shape[0] > 1000


def test_horizons_match_lattice_builder():
    """20 000 nodes, 1.0M bonds (the 100 x 10 x 20 beam): bit-identical with the
    lattice builder; the arrays cross the host boundary in staged chunks."""
    inp = bb.beam.build(bb.beam.config1())
    nfam, fptr, fam, bl, L0 = G.buildhorizons(inp["undeformedCoordinates"], inp["horizon"])
    assert same(bl, inp["BONDLIST"]) and same(L0, inp["UNDEFORMEDLENGTH"]) and same(nfam, inp["nFAMILYMEMBERS"])
    assert fptr[0] == 1 and same(np.diff(fptr), nfam[:-1]) and fam.size == 2 * bl.shape[0]
    dx = 5e-3
    vcf = G.calculatevolumecorrectionfactors(L0, inp["horizon"], dx / 2)
    assert same(vcf, inp["VOLUMECORRECTIONFACTORS"])
    VH = (4.0 / 3.0) * np.pi * inp["horizon"] ** 3
    bs, bt, bfm, sf = G.buildbonddata(bl, nfam, None, inp["bondStiffnessConcrete"], 0.0, inp["cellVolume"], VH)
    assert same(bs, inp["BONDSTIFFNESS"]) and not bt.any() and np.all(bfm == 1)
    mass = G.buildmassmatrix(inp["nNodes"], dx, inp["bondStiffnessConcrete"], inp["DT"], nfam)
    assert same(mass, inp["massVector"])


def test_notch_vs_oracle_and_lattice_builder():
    dx = 5e-3
    inp = bb.beam.build(bb.beam.small(nx=30, ny=5, nz=8))
    notched = bb.beam.build(bb.beam.small(nx=30, ny=5, nz=8, notch_x=15.5 * dx, notch_depth=3.2 * dx))
    X, bl, L0 = inp["undeformedCoordinates"], inp["BONDLIST"], inp["UNDEFORMEDLENGTH"]
    blo, L0o, nfam, fptr, fam = G.buildnotch(X, bl, L0, dx, 15.5, 3.7)
    n, nb = inp["nNodes"], inp["nBonds"]
    ob, oL, onf, ofp, ofam = np.zeros(2 * nb), np.zeros(nb), np.zeros(n), np.zeros(n), np.zeros(2 * nb)
    m = po.lib().orc_buildnotch(P(X), n, P(bl), P(L0), nb, dx, 15.5, 3.7, P(ob), P(oL), P(onf), P(ofp), P(ofam))
    assert blo.shape == (m, 2) and m < nb
    assert same(blo.ravel(order="F"), ob[:2 * m]) and same(L0o, oL[:m])
    assert same(nfam, onf) and same(fptr, ofp) and same(fam, ofam[:2 * m])
    assert same(blo, notched["BONDLIST"]) and same(nfam, notched["nFAMILYMEMBERS"])


def test_bonddata_material_table_vs_oracle():
    inp = bb.beam.build(bb.beam.small(nx=16, ny=5, nz=6))
    X, bl, nfam = inp["undeformedCoordinates"], inp["BONDLIST"], inp["nFAMILYMEMBERS"]
    nb = inp["nBonds"]
    mat = (X[:, 2] < 0.012).astype(np.float64)          # a steel layer at the bottom
    bs, bt, bfm, sf = G.buildbonddata(bl, nfam, mat, 3.1e18, 2.2e19, 1.25e-7, 1.3e-5)
    o = [np.zeros(nb) for _ in range(4)]
    assert po.lib().orc_bonddata(P(bl), nb, P(nfam), P(mat), 3.1e18, 2.2e19, 1.25e-7, 1.3e-5, *map(P, o)) == 0
    for a, b in zip((bs, bt, bfm, sf), o):
        assert same(a, b)
    assert set(np.unique(bt)) == {0.0, 1.0, 2.0}
    bad = mat.copy()
    bad[7] = 2.0
    with pytest.raises(bb.BBPDError):
        G.buildbonddata(bl, nfam, bad, 3.1e18, 2.2e19, 1.25e-7, 1.3e-5)


def test_builder_edge_cases():
    nfam, fptr, fam, bl, L0 = G.buildhorizons(np.zeros((1, 3)), 1.0)
    assert bl.shape == (0, 2) and same(nfam, [0.0]) and same(fptr, [1.0])
    nfam, fptr, fam, bl, L0 = G.buildhorizons(np.array([[0.0, 0, 0], [1.0, 0, 0], [3.0, 0, 0]]), 1.0)
    assert same(bl, np.array([[1.0, 2.0]])) and same(L0, [1.0]) and same(nfam, [1.0, 1.0, 0.0])
    for r in (0.0, -1.0, np.inf, np.nan):
        with pytest.raises(bb.BBPDError):
            G.buildhorizons(np.zeros((4, 3)), r)
    with pytest.raises(bb.BBPDError):
        G.buildhorizons(np.array([[0.0, 0, 0], [np.nan, 0, 0]]), 1.0)


def test_gpu_built_inputs_drive_the_solver():
    """Inputs from the GPU builder run the fused solver to the same state as the
    lattice builder's (they are the same arrays)."""
    inp = bb.beam.build(bb.beam.small(nx=20, ny=4, nz=6))
    nfam, _, _, bl, L0 = G.buildhorizons(inp["undeformedCoordinates"], inp["horizon"])
    vcf = G.calculatevolumecorrectionfactors(L0, inp["horizon"], 5e-3 / 2)
    VH = (4.0 / 3.0) * np.pi * inp["horizon"] ** 3
    bs = G.buildbonddata(bl, nfam, None, inp["bondStiffnessConcrete"], 0.0, inp["cellVolume"], VH)[0]
    mass = G.buildmassmatrix(inp["nNodes"], 5e-3, inp["bondStiffnessConcrete"], inp["DT"], nfam)
    gpu = dict(inp, BONDLIST=bl, UNDEFORMEDLENGTH=L0, VOLUMECORRECTIONFACTORS=vcf, BONDSTIFFNESS=bs,
               nFAMILYMEMBERS=nfam, massVector=mass)
    kw = dict(law="trilinear", s0=1e-4, s1=3e-4, sc=2e-3, scheme="adr", rate=-2e-6)
    a, b = bb.Solver(inp, **kw), bb.Solver(gpu, **kw)
    a.step(60)
    b.step(60)
    for f in ("displacement", "force", "bsf", "fail"):
        assert same(a.get(f), b.get(f)), f


def test_device_pointer_forms_match_host_forms():
    """bbpd_dev_buildhorizons / bbpd_dev_buildnotch on device arrays (torch
    tensors in the reference layouts) give the host-pointer forms' results."""
    import ctypes as C
    import torch
    L = bb._native.lib()
    p, i64 = C.c_void_p, C.c_int64
    L.bbpd_dev_buildhorizons.argtypes = [p, i64, C.c_double, i64, C.POINTER(i64), p, p, p, p, p, p]
    L.bbpd_dev_buildnotch.argtypes = [p, i64, p, p, i64, C.c_double, C.c_double, C.c_double, C.POINTER(i64),
                                      p, p, p, p, p, p]
    dx = 5e-3
    inp = bb.beam.build(bb.beam.small(nx=30, ny=5, nz=8))
    X = inp["undeformedCoordinates"]
    n = inp["nNodes"]
    dev = torch.device("cuda:0")
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)          # column-major n x 3
    ptr = lambda t: C.c_void_p(t.data_ptr())
    nb = C.c_int64()
    nfam, fptr = torch.zeros(n, dtype=torch.float64, device=dev), torch.zeros(n, dtype=torch.float64, device=dev)
    bb._native.check(L.bbpd_dev_buildhorizons(ptr(Xd), n, inp["horizon"], 0, C.byref(nb), ptr(nfam), ptr(fptr),
                                              None, None, None, None))
    m = nb.value
    fam = torch.zeros(2 * m, dtype=torch.float64, device=dev)
    bl = torch.zeros(2 * m, dtype=torch.float64, device=dev)
    L0 = torch.zeros(m, dtype=torch.float64, device=dev)
    bb._native.check(L.bbpd_dev_buildhorizons(ptr(Xd), n, inp["horizon"], m, C.byref(nb), None, None, ptr(fam),
                                              ptr(bl), ptr(L0), None))
    hn, hp, hf, hbl, hL = G.buildhorizons(X, inp["horizon"])
    assert same(nfam.cpu().numpy(), hn) and same(fptr.cpu().numpy(), hp) and same(fam.cpu().numpy(), hf)
    assert same(bl.cpu().numpy(), hbl.ravel(order="F")) and same(L0.cpu().numpy(), hL)
    out_n = C.c_int64()
    blo = torch.zeros(2 * m, dtype=torch.float64, device=dev)
    Lo = torch.zeros(m, dtype=torch.float64, device=dev)
    nf2 = torch.zeros(n, dtype=torch.float64, device=dev)
    bb._native.check(L.bbpd_dev_buildnotch(ptr(Xd), n, ptr(bl), ptr(L0), m, dx, 15.5, 3.7, C.byref(out_n), ptr(blo),
                                           ptr(Lo), ptr(nf2), None, None, None))
    k = out_n.value
    hblo, hLo, hnf, _, _ = G.buildnotch(X, hbl, hL, dx, 15.5, 3.7)
    assert k == hblo.shape[0] < m
    assert same(blo.cpu().numpy()[:2 * k], hblo.ravel(order="F")) and same(Lo.cpu().numpy()[:k], hLo)
    assert same(nf2.cpu().numpy(), hnf)
