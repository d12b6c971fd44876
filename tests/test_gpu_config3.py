"""GPU parity on the third configuration's beam at its full size: the notched
mixed-mode beam (400 x 100 x 50 mm, dx 2.5 mm, 128 000 nodes; bonds crossing
the 40 mm notch at 0.625 half-span off midspan removed as buildnotch.m does),
exponential softening (calculatebsfexponentialMex.c:26-66, k = 25,
alpha = 0.25), a seeded lognormal critical stretch per bond (mean 2e-3, CoV
0.1), ADR, both device forms (input order and lattice).

  * Against the oracle's restated loop with a correctly rounded exp, as the
    device's: every field bit-identical after steps 1, 2, 10 and 40.
  * Against the loop of the reference's compiled MEX routines (libm's exp,
    which misrounds about 8 in 10^4 of the law's arguments): displacement,
    velocity and nodal force within the bar below of their largest
    magnitudes, with identical softening and broken-bond sets.

Two loading rates: the benchmark's 1e-7 mm per step, and 5e-3 mm per step, at
which bonds round the loaded nodes soften and break within the 40 steps
(measured: 6 250 softening, 683 broken; largest difference from the libm
reference 1.0e-20 of the largest magnitude)."""
import numpy as np
import pytest

import bb_pd_b200 as bb
from oracle import pyoracle as po

from test_gpu_solver import same

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref (reference MEX routines) not built")]

FIELDS = ("displacement", "velocity", "force", "deformed", "bsf", "flag", "fail")
LIBM_BAR = 1e-12     # of the largest magnitude, against the libm-exp reference loop


@pytest.fixture(scope="module")
def beam3():
    inp = bb.beam.build(bb.beam.config3())
    assert inp["nNodes"] == 128000 and "sc" in inp
    return inp


@pytest.mark.parametrize("rate", [-1e-10, -5e-6], ids=["1e-7mm_per_step", "5e-3mm_per_step"])
def test_config3_vs_oracle_and_reference_mex(beam3, rate):
    kw = dict(law="exponential", s0=1e-4, scheme="adr", rate=rate)
    forms = {"input": bb.Solver(beam3, **kw), "lattice": bb.Solver(beam3, node_order="lattice", **kw)}
    assert forms["lattice"].info()["layout"] & 32
    cr = po.Run(beam3, law_exp="cr", cn_order="tree", **kw)
    libm = po.Run(beam3, kernels="reference", cn_order="tree", **kw)
    done = 0
    worst = 0.0
    for m in (1, 2, 10, 40):
        for s in forms.values():
            s.step(m - done)
        cr.step(m - done)
        libm.step(m - done)
        done = m
        for name, s in forms.items():
            for f in FIELDS:
                a, b = s.get(f), cr.get(f)
                assert same(a, b), f"{name} form, step {m}: {f}: {int(np.sum(a != b))} of {a.size} differ"
            assert s.cn == cr.cn
            for f in ("displacement", "velocity", "force"):
                a, b = s.get(f), libm.get(f)
                scale = max(np.abs(b).max(), 1e-300)
                worst = max(worst, np.abs(a - b).max() / scale)
                np.testing.assert_allclose(a, b, rtol=0, atol=LIBM_BAR * scale,
                                           err_msg=f"{name} form, step {m}, libm reference: {f}")
            assert np.array_equal(s.get("flag"), libm.get("flag")), f"{name}, step {m}: softening set"
            assert np.array_equal(s.get("bsf") == 1, libm.get("bsf") == 1), f"{name}, step {m}: broken set"
    soft, broken = int((cr.get("flag") > 0).sum()), int((cr.get("bsf") == 1).sum())
    print(f"rate {rate}: {soft} softening, {broken} broken after {done} steps; "
          f"largest difference from the libm reference {worst:.3g} of the largest magnitude")
    if rate == -5e-6:
        assert soft > 0 and broken > 0
    for s in forms.values():
        s.close()
