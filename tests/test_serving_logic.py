"""Host-side logic of the serving form (no GPU): the peak / post-peak stop
rule on reaction histories, the admission estimate, and the synthetic request
generators."""
import numpy as np

import bb_pd_b200 as bb
from bb_pd_b200 import serving


def _req(max_steps=10_000, post=0.8):
    return serving.Request(0, 0.0, {"nBonds": 10, "nNodes": 5}, "linear", -1e-6, max_steps, post)


def test_stop_after_post_peak_drop():
    tr = serving._Track(_req())
    load = np.concatenate([np.linspace(0, 10, 50), np.linspace(10, 7.5, 30)])   # peak, then 25 % drop
    fins = [tr.update(-c) for c in np.split(load, 8)]
    assert fins[-1] and not any(fins[:5])
    assert tr.peak == 10.0 and tr.peak_step == 50


def test_no_stop_before_the_drop_and_step_cap():
    tr = serving._Track(_req(max_steps=60))
    assert not tr.update(np.linspace(0, 5, 30))
    assert tr.update(np.linspace(5, 6, 30))          # cap reached
    tr2 = serving._Track(_req())
    assert not tr2.update(np.array([1.0, 2.0, 3.0, 2.9]))


def test_skip_keeps_step_count():
    tr = serving._Track(_req())
    tr.skip(12)
    tr.update(np.ones(8))
    assert tr.steps == 20 and tr.peak_step == 13


def test_admission_estimate_grows_with_bonds():
    a = serving.device_bytes_estimate({"nBonds": 1000, "nNodes": 100}, False)
    b = serving.device_bytes_estimate({"nBonds": 2000, "nNodes": 100}, True)
    assert b > 2 * a - (1 << 21)


def test_generators():
    series = bb.beam.size_effect_series(64)
    assert len(series) == 64 and {law for _, law in series} <= {"linear", "trilinear"}
    depths = [s.nz * s.dx for s, _ in series]
    assert 0.045 < min(depths) and max(depths) < 0.41
    st = bb.beam.serving_stream(200)
    t = [r["arrival"] for r in st]
    assert all(np.diff(t) > 0) and len({r["law"] for r in st}) == 4
    nodes = [r["nodes"] for r in st]
    assert 5e3 < min(nodes) and max(nodes) < 2e6
