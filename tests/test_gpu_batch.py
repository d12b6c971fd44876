"""GPU tests of the batching and serving form.

A batch shares the SMs among its members but leaves each member's arithmetic
untouched, so the stated tolerance is exact equality: every member's state is
bit-identical to the same solve run alone, whatever joins or leaves the batch
around it, whichever schedule the autotuner picks, with or without CUDA-graph
replay. The reaction (force on the prescribed DOFs) is checked against the
oracle's fixed-order tree sum of the same per-node terms."""
import numpy as np
import pytest

import bb_pd_b200 as bb
from bb_pd_b200 import serving
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

FIELDS = ("displacement", "velocity", "force", "deformed", "bsf", "flag", "fail")
LAWKW = serving.LAWKW


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


@pytest.fixture(scope="module")
def beams():
    return [bb.beam.build(bb.beam.small(nx=20, ny=4, nz=6)),
            bb.beam.build(bb.beam.small(nx=36, ny=5, nz=8)),
            bb.beam.build(bb.beam.small(nx=28, ny=4, nz=6, sc_lognormal=(2e-3, 0.1)))]


def _solver(inp, law, precision="fp64", rate=-3e-6):
    return bb.Solver(inp, scheme="adr", rate=rate, precision=precision, **LAWKW[law])


@pytest.mark.parametrize("mixed", [True, False], ids=["one_launch", "launch_per_law"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_alone_and_in_mix_identical(beams, precision, mixed):
    """Members of uneven size and law join and leave a batch at different
    steps; each ends bit-identical to its solo run of the same length. With
    mixing (the default) the three laws, one member with a per-bond critical
    stretch, run in a single persistent launch per kernel variant."""
    laws = ["trilinear", "linear", "exponential"]
    solo = []
    for inp, law, n in zip(beams, laws, (90, 70, 50)):
        s = _solver(inp, law, precision)
        s.step(n)
        solo.append(s)
    batch = bb.Batch(precision)
    batch.set_mixing(mixed)
    m = [_solver(inp, law, precision) for inp, law in zip(beams, laws)]
    batch.add(m[0])
    batch.step(20)                      # member 0 alone in the batch
    batch.add(m[1])
    batch.step(30)                      # 0 at 50, 1 at 30
    batch.add(m[2])
    batch.step(40)                      # 0 at 90, 1 at 70, 2 at 40
    variants = len({mm.info()["layout"] & 15 for mm in m})
    assert batch.info()["n_classes"] == (variants if mixed else 3)
    batch.remove(m[0])
    batch.remove(m[1])
    batch.step(10)                      # 2 at 50
    for k in range(3):
        assert m[k].next_step == solo[k].next_step
        for f in FIELDS:
            assert same(m[k].get(f), solo[k].get(f)), (k, f)
        assert m[k].cn == solo[k].cn
    assert (solo[0].get("bsf") > 0).any()
    batch.close()


def test_schedules_and_graph_identical(beams):
    ref = [_solver(inp, "trilinear") for inp in beams[:2]]
    for s in ref:
        s.step(60)
    for bps, grab, graph in ((1, 1, False), (2, 4, True), (1, 2, True)):
        batch = bb.Batch("fp64")
        m = [_solver(inp, "trilinear") for inp in beams[:2]]
        for s in m:
            batch.add(s)
        batch.set_schedule(bps, grab, graph)
        for _ in range(3):              # graph replays after the first capture
            batch.step(20)
        info = batch.info()
        assert info["n_members"] == 2 and info["grab"] == grab
        for a, b in zip(m, ref):
            for f in FIELDS:
                assert same(a.get(f), b.get(f)), (bps, grab, graph, f)
        batch.close()


def test_autotuner_runs_real_steps(beams):
    batch = bb.Batch("fp64")
    m = [_solver(inp, "trilinear") for inp in beams[:2]]
    for s in m:
        batch.add(s)
    bps, grab = batch.tune(3)
    assert bps >= 1 and grab in (1, 2, 4)
    n = m[0].next_step - 1
    assert n > 0 and n % 3 == 0
    ref = _solver(beams[0], "trilinear")
    ref.step(n)
    for f in FIELDS:
        assert same(m[0].get(f), ref.get(f)), f
    batch.close()


def _tree_reaction(inp, F):
    pf = np.asarray(inp["BODYFORCEFLAG"]) == 1
    t = np.zeros(inp["nNodes"])
    for d in range(3):
        t = np.where(pf[:, d], t + F[:, d], t)
    return po.tree_sum(t)


def test_reaction_is_the_tree_sum_of_prescribed_forces(beams):
    inp = beams[1]
    kw = dict(scheme="adr", rate=-3e-6, **LAWKW["trilinear"])
    s = bb.Solver(inp, **kw)
    r = po.Run(inp, **kw)
    for n in (1, 25, 40):
        s.step(n)
        r.step(n)
        rea = s.reaction(n)
        assert rea[-1] == _tree_reaction(inp, s.get("force"))
        assert rea[-1] == _tree_reaction(inp, r.get("force"))
    assert rea[-1] != 0.0


def test_batch_rejections(beams):
    batch = bb.Batch("fp64")
    ec = bb.Solver(beams[0], scheme="eulercromer", rate=-1e-6, **LAWKW["linear"])
    with pytest.raises(bb.BBPDError) as e:
        batch.add(ec)
    assert e.value.status == bb._native.ERR_UNSUPPORTED
    f32 = _solver(beams[0], "linear", "fp32")
    with pytest.raises(bb.BBPDError):
        batch.add(f32)
    s = _solver(beams[0], "linear")
    batch.add(s)
    with pytest.raises(bb.BBPDError) as e:
        s.step(1)                       # members are stepped by the batch
    assert e.value.status == bb._native.ERR_ARG
    batch.close()
    s.step(1)                           # free again once the batch is gone


def test_serving_results_same_alone_and_in_mix(beams):
    """Requests arriving while others run are admitted into the running
    batch; each result (every per-step reaction) equals its solo run."""
    reqs = [serving.Request(k, arr, inp, law, rate=-3e-6, max_steps=steps)
            for k, (inp, law, steps, arr) in enumerate(zip(beams, ["trilinear", "bilinear", "exponential"],
                                                             (1200, 600, 800), (0.0, 0.0, 0.005)))]
    res, stats = serving.run_batched(reqs, chunk=20, tune=False)
    assert len(res) == 3
    seq, _ = serving.run_sequential(reqs, chunk=20)
    by_id = {r.id: r for r in seq}
    for r in res:
        assert r.steps == by_id[r.id].steps
        assert same(r.reactions, by_id[r.id].reactions), r.id
    assert stats["peak_members"] >= 2
