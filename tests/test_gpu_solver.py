"""GPU parity of the fused persistent time-step kernel against the oracle: the
reference loop (dynamicsolverdisplacementcontrolled.m:71-105 and its ADR form)
run on the CPU by the restatement or by the reference's compiled MEX routines.

Bar: plain FP64 form bit-identical in displacement, velocity, force, damage,
softening flags and fail flags (up to the sign of zero), every law included
when the oracle's exponential law rounds exp correctly as the device does;
against libm's exp (the compiled reference) the exponential law within 1e-9
of the largest magnitude with identical softening and broken-bond sets; the
FP32 form within the stated tolerances of the FP64 form with an identical
broken-bond set."""
import os

import numpy as np
import pytest

import bb_pd_b200 as bb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

LAWKW = {
    "linear": dict(law="linear", sc=2e-3),
    "bilinear": dict(law="bilinear", s0=1e-4, sc=2e-3),
    "trilinear": dict(law="trilinear", s0=1e-4, s1=3e-4, sc=2e-3),
    "exponential": dict(law="exponential", s0=1e-4, sc=2e-3),
}
NODAL = ("displacement", "velocity", "force", "deformed")
BOND = ("bsf", "flag", "fail")


def orun(inp, **kw):
    """The oracle with the restated routines and a correctly rounded exp in the
    exponential law (the device's exp rounds correctly; libm's misrounds about
    8 in 10^4 of the law's arguments, which the libm runs below measure)."""
    return po.Run(inp, law_exp="cr", **kw)


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def compare(s, r, law, fields=NODAL + BOND, rtol=1e-9):
    """Bit-identical, except the exponential law against an oracle whose exp
    is libm's (the compiled reference routines): libm's exp misrounds about 8
    in 10^4 arguments where the device's is correctly rounded, and undamped
    dynamics carry a last-bit difference along; there nodal fields must agree
    within 1e-9 of their largest magnitude, damage within 1e-8, and softening
    flags and the broken-bond set exactly."""
    libm = law == "exponential" and getattr(r, "law_exp", "libm") == "libm"
    for f in fields:
        a, b = s.get(f), r.get(f)
        if libm and f not in ("flag", "fail"):
            atol = 1e-8 if f == "bsf" else rtol * max(np.abs(b).max(), 1e-300)
            np.testing.assert_allclose(a, b, rtol=0, atol=atol, err_msg=f)
        else:
            assert same(a, b), f"{f}: {np.sum(a != b)} of {a.size} differ"
    assert np.array_equal(s.get("bsf") == 1, r.get("bsf") == 1)


@pytest.fixture(scope="module")
def small():
    return bb.beam.build(bb.beam.small(nx=20, ny=4, nz=6))


@pytest.mark.parametrize("law", list(LAWKW))
@pytest.mark.parametrize("scheme", ["eulercromer", "adr"])
def test_fused_vs_oracle(small, law, scheme):
    kw = dict(LAWKW[law], scheme=scheme, rate=-4e-6 if scheme == "eulercromer" else -2e-6)
    s = bb.Solver(small, **kw)
    r = orun(small, **kw)
    for n in (1, 40, 119):
        s.step(n)
        r.step(n)
        compare(s, r, law)
    if scheme == "adr":
        assert s.cn == r.cn
    # the run exercises the law: some bonds soften or break
    if law == "linear":
        assert (r.get("fail") == 0).any()
    else:
        assert (r.get("bsf") > 0).any()
    s.close()


def test_fused_vs_golden_reference_loop():
    g = dict(np.load(os.path.join(GOLD, "loop_ec_exponential.npz")))
    keys = ("undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH", "BONDSTIFFNESS",
            "VOLUMECORRECTIONFACTORS", "DENSITY", "massVector", "CONSTRAINTFLAG", "BODYFORCEFLAG")
    inp = {k: np.asfortranarray(g[k]) for k in keys}
    inp.update(nNodes=int(g["nNodes"]), nBonds=int(g["nBonds"]), DT=float(g["DT"]), cellVolume=float(g["cellVolume"]))
    s = bb.Solver(inp, law="exponential", scheme="eulercromer", rate=float(g["rate"]), s0=1e-4, sc=2e-3)
    s.step(int(g["steps"]))
    for f in ("displacement", "velocity", "force", "deformed", "acceleration", "bsf"):
        ref = g["out_" + f]
        np.testing.assert_allclose(s.get(f), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max(), err_msg=f)
    for f in ("flag", "fail"):
        assert same(s.get(f), g["out_" + f]), f
    assert np.array_equal(s.get("bsf") == 1, g["out_bsf"] == 1)


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("law", ["exponential", "linear"])
def test_fused_vs_reference_mex_loop(law):
    inp = bb.beam.build(bb.beam.small(nx=18, ny=5, nz=5))
    kw = dict(LAWKW[law], scheme="eulercromer", rate=-3e-6)
    s = bb.Solver(inp, **kw)
    r = po.Run(inp, kernels="reference", **kw)
    s.step(100)
    r.step(100)
    compare(s, r, law)


def test_per_bond_sc_notched_adr():
    """Notched beam, per-bond lognormal sc, exponential law, ADR (the mixed-mode case, small)."""
    sp = bb.beam.spec(40, 4, 12, 2.5e-3, supports=(7.5e-3, 0.0925), notch_x=0.05 + 1.25e-3 + 0.01,
                      notch_depth=0.01, sc_lognormal=(2e-3, 0.1))
    inp = bb.beam.build(sp)
    kw = dict(law="exponential", scheme="adr", s0=1e-4, rate=-1e-6)
    s = bb.Solver(inp, **kw)
    r = orun(inp, **kw)
    s.step(150)
    r.step(150)
    compare(s, r, "exponential")


@pytest.mark.parametrize("T", [1, 3, 64])
def test_chunk_counts(small, T):
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-2e-6, n_chunks=T)
    s = bb.Solver(small, **kw)
    r = orun(small, **kw)
    s.step(30)
    r.step(30)
    compare(s, r, "trilinear")


@pytest.fixture(scope="module")
def tiled_beam():
    """48 x 8 x 10 nodes: eight 512-node tiles of the tiled kernel, each with a halo."""
    return bb.beam.build(bb.beam.small(nx=48, ny=8, nz=10))


@pytest.mark.parametrize("law", list(LAWKW))
@pytest.mark.parametrize("scheme", ["eulercromer", "adr"])
def test_tiled_vs_oracle(tiled_beam, law, scheme):
    kw = dict(LAWKW[law], scheme=scheme, rate=-4e-6 if scheme == "eulercromer" else -2e-6)
    s = bb.Solver(tiled_beam, node_order="tiled", **kw)
    assert s.info()["layout"] & 16, "tiled kernel expected"
    r = orun(tiled_beam, **kw)
    for n in (1, 60):
        s.step(n)
        r.step(n)
        compare(s, r, law)
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tiled_identical_to_global_gather(tiled_beam, precision):
    """Staging neighbours in shared memory changes where data is read from,
    not the arithmetic: the tiled and the global-gather kernels agree bit for bit."""
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-4e-6, precision=precision)
    a = bb.Solver(tiled_beam, node_order="input", **kw)
    b = bb.Solver(tiled_beam, node_order="tiled", **kw)
    assert not a.info()["layout"] & 16 and b.info()["layout"] & 16
    a.step(80)
    b.step(80)
    for f in NODAL + BOND:
        assert same(a.get(f), b.get(f)), f
    assert (a.get("bsf") > 0).any()


def test_morton_order_identical(small):
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-2e-6)
    a = bb.Solver(small, node_order="input", **kw)
    b = bb.Solver(small, node_order="morton", **kw)
    a.step(80)
    b.step(80)
    for f in NODAL + BOND:
        assert same(a.get(f), b.get(f)), f


@pytest.fixture(scope="module")
def medium():
    """40 000 nodes, 2.4M bonds: the bond arrays cross the host-device boundary
    in several staged chunks per host thread, and the device-built layout (input
    and Morton orders) meets the host-built one (tiled order) at scale."""
    return bb.beam.build(bb.beam.small(nx=100, ny=20, nz=20))


@pytest.mark.parametrize("law", ["trilinear", "exponential"])
def test_layouts_identical_at_scale(medium, law):
    nB = medium["nBonds"]
    rng = np.random.default_rng(11)
    inp = dict(medium)
    inp["fail"] = (rng.random(nB) > 0.02).astype(np.float64)        # 2 % of the bonds start broken
    if law == "exponential":
        inp["BONDTYPE"] = rng.integers(0, 3, nB).astype(np.float64)
    kw = dict(LAWKW[law], scheme="adr", rate=-2e-6)
    runs = [bb.Solver(inp, node_order=o, **kw) for o in ("input", "morton", "tiled")]
    for s in runs:
        s.step(40)
    for f in NODAL + BOND:
        ref = runs[0].get(f)
        for s in runs[1:]:
            assert same(ref, s.get(f)), f
    assert np.array_equal(runs[0].get("fail"), np.where(inp["fail"] == 0, 0.0, runs[0].get("fail")))
    # per-bond fields round-trip through the staged copies
    v = rng.random(nB)
    v[rng.random(nB) < 0.5] = 0.0
    runs[1].set("bsf", v)
    assert same(runs[1].get("bsf"), v)
    flags = (rng.random(nB) < 0.3).astype(np.float64)
    runs[2].set("flag", flags)
    assert same(runs[2].get("flag"), flags)
    for s in runs:
        s.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_bad_bondlist_first_row_reported(medium, precision):
    """BONDLIST rows are checked while they are staged (FP64) or before the
    dictionary pass (FP32): either way the first bad row is the one reported."""
    nN = medium["nNodes"]
    bl = medium["BONDLIST"].copy(order="F")
    bl[2_000_000, 0] = nN + 1          # out of range
    bl[1_234_567, 1] = 2.5             # not an integer
    bad = dict(medium, BONDLIST=bl)
    with pytest.raises(bb.BBPDError) as e:
        bb.Solver(bad, **LAWKW["trilinear"], scheme="adr", precision=precision)
    assert e.value.status == bb._native.ERR_ARG
    assert "row 1234568 " in str(e.value), str(e.value)


@pytest.mark.parametrize("law", ["trilinear", "bilinear", "exponential"])
def test_damage_energy_tracking_vs_oracle(small, law):
    """The fused solver's damage energy against the oracle's loop with
    calculatedamageenergy.m applied to every step's stretch (the drivers'
    order): bit-identical for every law (the oracle's exponential law with a
    correctly rounded exp, as the device's)."""
    kw = dict(LAWKW[law], scheme="adr", rate=-4e-6)
    s = bb.Solver(small, **kw)
    s.track_damage_energy()
    r = orun(small, **kw)
    nB = small["nBonds"]
    s0 = np.full(nB, kw.get("s0", 1e-4))
    sc = np.full(nB, kw["sc"])
    E = np.zeros(nB)
    bs, L0, V = small["BONDSTIFFNESS"], small["UNDEFORMEDLENGTH"], small["cellVolume"]
    P = po.P
    for step in range(90):
        r.step(1)
        st = r.get("stretch")
        po.lib().orc_damageenergy(P(bs), P(s0), P(sc), P(L0), P(st), 25.0, 0.25, V, P(E), nB)
    s.step(40)
    s.step(50)
    got = s.get("damage_energy")
    assert (E > 0).any()
    assert same(got, E)
    s.track_damage_energy()                    # restart: nothing recorded yet
    assert not s.get("damage_energy").any()
    s.close()


def test_damage_energy_tracking_rejections(small):
    s = bb.Solver(small, **LAWKW["trilinear"], scheme="adr")
    with pytest.raises(bb.BBPDError) as e:
        s.get("damage_energy")
    assert e.value.status == bb._native.ERR_ARG
    s.close()
    s = bb.Solver(small, **LAWKW["linear"], scheme="adr")
    with pytest.raises(bb.BBPDError) as e:
        s.track_damage_energy()
    assert e.value.status == bb._native.ERR_UNSUPPORTED
    s.close()


def test_split_launches_identical(small):
    kw = dict(LAWKW["bilinear"], scheme="adr", rate=-2e-6)
    a, b = bb.Solver(small, **kw), bb.Solver(small, **kw)
    a.step(100)
    b.step(37)
    b.step(1)
    b.step(62)
    for f in NODAL + BOND:
        assert same(a.get(f), b.get(f)), f


@pytest.mark.parametrize("scheme", ["eulercromer", "adr"])
def test_checkpoint_resume_bit_identical(small, scheme):
    kw = dict(LAWKW["trilinear"], scheme=scheme, rate=-2e-6)
    a = bb.Solver(small, **kw)
    a.step(45)
    ck = a.checkpoint()
    a.step(55)
    b = bb.Solver(small, **kw)          # fresh solver, restored from the checkpoint
    b.restore(ck)
    b.step(55)
    for f in NODAL + BOND:
        assert same(a.get(f), b.get(f)), f
    c = bb.Solver(small, **kw)          # odd step count: buffers of the other parity
    c.step(3)
    c.restore(ck)
    c.step(55)
    for f in NODAL + BOND:
        assert same(a.get(f), c.get(f)), f


def test_smoothstep_amplitude(small):
    kw = dict(LAWKW["trilinear"], scheme="adr", amplitude="smoothstep", applied_final=-2e-4, n_time_steps=120)
    s, r = bb.Solver(small, **kw), orun(small, **kw)
    s.step(120)
    r.step(120)
    compare(s, r, "trilinear")
    pf = small["BODYFORCEFLAG"][:, 2] == 1
    u = s.get("displacement")
    assert np.all(u[pf, 2] == po.lib().orc_smoothstep(121.0, 1.0, 120.0, 0.0, -2e-4))   # held at U(next step)


def test_fp32_form_tolerance(small):
    """FP32 stretch/force with FP64 sums and guard band: one step from the same
    state matches the FP64 force to 1e-5 of the largest nodal force and breaks
    exactly the same bonds; over a run the displacement stays within 1e-4."""
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-2e-6)
    a = bb.Solver(small, precision="fp64", **kw)
    b = bb.Solver(small, precision="fp32", **kw)
    a.step(60)
    b.restore(a.checkpoint())
    a.step(1)
    b.step(1)
    Fa, Fb = a.get("force"), b.get("force")
    err = np.abs(Fa - Fb).max() / np.abs(Fa).max()
    assert err < 1e-5, err
    assert np.array_equal(a.get("bsf") == 1, b.get("bsf") == 1)
    a.step(100)
    b.step(100)
    ua, ub = a.get("displacement"), b.get("displacement")
    assert np.abs(ua - ub).max() / np.abs(ua).max() < 1e-4


def test_nonfinite_detected(small):
    s = bb.Solver(small, **LAWKW["trilinear"], scheme="adr", rate=-2e-6)
    s.step(2)
    u = s.get("displacement")
    u[5, 0] = np.nan
    s.set("displacement", u)
    with pytest.raises(bb.BBPDError) as e:
        s.step(1)
    assert e.value.status == bb._native.ERR_NONFINITE


def test_invalid_inputs_rejected(small):
    bad = dict(small)
    bl = small["BONDLIST"].copy(order="F")
    bl[0, 1] = bl[0, 0]                       # self-bond
    bad["BONDLIST"] = bl
    with pytest.raises(bb.BBPDError) as e:
        bb.Solver(bad, **LAWKW["trilinear"], scheme="adr")
    assert e.value.status == bb._native.ERR_ARG
    bad = dict(small, stretchPlastic=np.full(small["nBonds"], 1e-4))
    with pytest.raises(bb.BBPDError) as e:
        bb.Solver(bad, **LAWKW["trilinear"], scheme="adr")
    assert e.value.status == bb._native.ERR_UNSUPPORTED


def test_info(small):
    s = bb.Solver(small, **LAWKW["trilinear"], scheme="adr")
    i = s.info()
    assert i["n_nodes"] == small["nNodes"] and i["n_bonds"] == small["nBonds"]
    assert i["n_entries"] >= 2 * small["nBonds"] and i["n_entries"] % 32 == 0
    assert i["grid_blocks"] >= 1 and i["device_bytes"] > 0


def _contact_setup(small, inc):
    """Midspan loading cylinder and two support cylinders, no prescribed DOFs
    (the cylinder loads the beam, as in the reference's drivers)."""
    inp = dict(small)
    inp["BODYFORCEFLAG"] = np.zeros_like(small["BODYFORCEFLAG"], order="F")
    X = small["undeformedCoordinates"]
    x0, x1 = X[:, 0].min(), X[:, 0].max()
    pens = [bb.beam.penetrator(inp, 0.5 * (x0 + x1), 0.01, 0.03, inc),
            bb.beam.penetrator(inp, x0 + 0.015, 0.005, 0.015, 0.0, top=False, reaction=False),
            bb.beam.penetrator(inp, x1 - 0.015, 0.005, 0.015, 0.0, top=False, reaction=False)]
    return inp, pens


@pytest.mark.parametrize("scheme", ["eulercromer", "adr"])
def test_contact_vs_oracle(small, scheme):
    """calculatecontactforce.m fused into the integration: state bit-identical
    to the oracle's literal restatement, reaction equal."""
    inp, pens = _contact_setup(small, -2e-6 if scheme == "adr" else -4e-6)
    kw = dict(LAWKW["trilinear"], scheme=scheme)
    s = bb.Solver(inp, **kw)
    s.set_contact(pens)
    r = orun(inp, penetrators=pens, **kw)
    for n in (1, 60, 79):
        s.step(n)
        r.step(n)
        compare(s, r, "trilinear")
        assert s.reaction(n)[-1] == r.reaction
    assert r.reaction != 0.0 and (np.abs(s.get("displacement")[:, 2]) > 0).any()


def test_contact_in_batch_identical(small):
    inp, pens = _contact_setup(small, -2e-6)
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=0.0)
    a = bb.Solver(inp, **kw)
    a.set_contact(pens)
    a.step(70)
    b = bb.Solver(inp, **kw)
    b.set_contact(pens)
    other = bb.Solver(small, **kw, )
    batch = bb.Batch("fp64")
    batch.add(b)
    batch.add(other)
    batch.step(70)
    for f in NODAL + BOND:
        assert same(a.get(f), b.get(f)), f
    assert same(a.reaction(70), b.reaction(70))
    batch.close()


def test_contact_rejects_overlap_and_missing_density(small):
    inp, pens = _contact_setup(small, -2e-6)
    s = bb.Solver(inp, **LAWKW["linear"], scheme="adr")
    with pytest.raises(bb.BBPDError) as e:
        s.set_contact([pens[0], dict(pens[0], increment=0.0)])
    assert e.value.status == bb._native.ERR_UNSUPPORTED
    nod = dict(inp)
    del nod["DENSITY"]
    t = bb.Solver(nod, **LAWKW["linear"], scheme="adr")
    with pytest.raises(bb.BBPDError):
        t.set_contact(pens[:1])


@pytest.mark.parametrize("scheme", ["eulercromer", "adr"])
def test_probes_record_every_step(small, scheme):
    """Probes hold each step's displacement of their DOFs: the history of one
    40-step launch equals 40 single-step launches read back one by one."""
    kw = dict(LAWKW["trilinear"], scheme=scheme, rate=-3e-6)
    nodes = [3, 17, small["nNodes"]]
    dofs = [0, 0, 2]
    a = bb.Solver(small, **kw)
    a.set_probes(nodes, dofs)
    a.step(40)
    hist = a.probes(40)
    b = bb.Solver(small, **kw)
    for it in range(40):
        b.step(1)
        u = b.get("displacement")
        assert all(hist[it, k] == u[n - 1, c] for k, (n, c) in enumerate(zip(nodes, dofs))), it
    cmod = hist[:, 1] - hist[:, 0]
    assert cmod.shape == (40,)


def test_savedata_mat(small, tmp_path):
    import scipy.io
    s = bb.Solver(small, **LAWKW["trilinear"], scheme="adr", rate=-3e-6)
    s.step(12)
    path = s.savedata(str(tmp_path), "beam")
    assert path.endswith("beam_12.mat")
    m = scipy.io.loadmat(path)
    assert same(m["deformedCoordinates"], s.get("deformed"))
    assert m["fail"].shape == (small["nBonds"], 1) and m["flagBondSoftening"].shape == (small["nBonds"], 1)


# ---------------------------------------------------------------- lattice form

def _lattice(inp, **kw):
    s = bb.Solver(inp, node_order="lattice", **kw)
    assert s.info()["layout"] & 32, "lattice form expected"
    return s


@pytest.mark.parametrize("law", list(LAWKW))
@pytest.mark.parametrize("scheme", ["eulercromer", "adr"])
def test_lattice_vs_oracle(small, law, scheme):
    """Stencil-addressed neighbours and one state slot per bond: the same
    arithmetic in the same order as the reference loop, bit for bit."""
    kw = dict(LAWKW[law], scheme=scheme, rate=-4e-6 if scheme == "eulercromer" else -2e-6)
    s = _lattice(small, **kw)
    r = orun(small, **kw)
    for n in (1, 40, 119):
        s.step(n)
        r.step(n)
        compare(s, r, law)
    if scheme == "adr":
        assert s.cn == r.cn
    if law == "linear":
        assert (r.get("fail") == 0).any()
    else:
        assert (r.get("bsf") > 0).any()
    s.close()


@pytest.fixture(scope="module")
def ragged():
    """70 x 9 x 11 nodes: partial tiles along every axis (x rows of 32, rows of
    the tile's y and z extents), supports and load away from tile edges."""
    return bb.beam.build(bb.beam.small(nx=70, ny=9, nz=11))


@pytest.mark.parametrize("law", ["trilinear", "linear"])
def test_lattice_ragged_tiles_vs_input_order(ragged, law):
    nB = ragged["nBonds"]
    rng = np.random.default_rng(5)
    inp = dict(ragged)
    inp["fail"] = (rng.random(nB) > 0.03).astype(np.float64)
    inp["BONDTYPE"] = rng.integers(0, 3, nB).astype(np.float64)
    kw = dict(LAWKW[law], scheme="adr", rate=-4e-6)
    a = bb.Solver(inp, node_order="input", **kw)
    b = _lattice(inp, **kw)
    for n in (1, 30, 90):
        a.step(n)
        b.step(n)
        for f in NODAL + BOND:
            assert same(a.get(f), b.get(f)), (n, f)
    assert a.cn == b.cn
    a.close()
    b.close()


def test_lattice_notched_per_bond_sc_vs_oracle():
    """Bonds across the notch are missing from the list (absent slots) and the
    critical stretch is per bond (lognormal): exponential law, ADR."""
    sp = bb.beam.spec(40, 4, 12, 2.5e-3, supports=(7.5e-3, 0.0925), notch_x=0.05 + 1.25e-3 + 0.01,
                      notch_depth=0.01, sc_lognormal=(2e-3, 0.1))
    inp = bb.beam.build(sp)
    kw = dict(law="exponential", scheme="adr", s0=1e-4, rate=-1e-6)
    s = _lattice(inp, **kw)
    r = orun(inp, **kw)
    s.step(150)
    r.step(150)
    compare(s, r, "exponential")


@pytest.mark.parametrize("T", [1, 3])
def test_lattice_chunk_counts(small, T):
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-2e-6, n_chunks=T)
    s = _lattice(small, **kw)
    r = orun(small, **kw)
    s.step(30)
    r.step(30)
    compare(s, r, "trilinear")


def test_lattice_falls_back_when_not_a_lattice(small):
    """Inputs the lattice form does not cover run the input-order kernel:
    jittered coordinates, a bond list not ordered by first node, and more
    OpenMP chunk starts in a list than the form records."""
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-2e-6)
    X = small["undeformedCoordinates"].copy(order="F")
    X[7, 1] += 1e-9
    nB = small["nBonds"]
    shuffled = dict(small)
    perm = np.random.default_rng(3).permutation(nB)
    for k, v in small.items():
        if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == nB:
            shuffled[k] = np.asfortranarray(v[perm])
    for inp, extra in ((dict(small, undeformedCoordinates=X), {}), (shuffled, {}), (small, {"n_chunks": 64})):
        s = bb.Solver(inp, node_order="lattice", **kw, **extra)
        assert not s.info()["layout"] & 32
        r = orun(inp, **kw, **extra)
        s.step(20)
        r.step(20)
        compare(s, r, "trilinear")
        s.close()


def test_lattice_state_roundtrip_and_restore(ragged):
    """Per-bond fields cross the C ABI through the bond -> slot map; a
    checkpoint restored into a fresh lattice solver continues bit for bit."""
    nB = ragged["nBonds"]
    rng = np.random.default_rng(9)
    kw = dict(LAWKW["bilinear"], scheme="adr", rate=-4e-6)
    a = _lattice(ragged, **kw)
    v = rng.random(nB)
    v[rng.random(nB) < 0.7] = 0.0
    a.set("bsf", v)
    assert same(a.get("bsf"), v)
    fl = (rng.random(nB) < 0.2).astype(np.float64)
    a.set("flag", fl)
    assert same(a.get("flag"), fl)
    fa = (rng.random(nB) > 0.1).astype(np.float64)
    a.set("fail", fa)
    assert same(a.get("fail"), fa)
    a.step(25)
    ck = a.checkpoint()
    b = _lattice(ragged, **kw)
    b.restore(ck)
    a.step(40)
    b.step(40)
    for f in NODAL + BOND:
        assert same(a.get(f), b.get(f)), f
    a.close()
    b.close()


def test_lattice_damage_energy_tracking(small):
    kw = dict(LAWKW["trilinear"], scheme="adr", rate=-4e-6)
    a = bb.Solver(small, **kw)
    b = _lattice(small, **kw)
    a.track_damage_energy()
    b.track_damage_energy()
    a.step(90)
    b.step(90)
    ea, eb = a.get("damage_energy"), b.get("damage_energy")
    assert (ea > 0).any() and same(ea, eb)
