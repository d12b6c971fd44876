"""The mexFunction gateways against the reference's own gateways: the same
mxArray arguments go to both (stub mex.h layout), outputs compared in place."""
import numpy as np
import pytest

import bb_pd_b200 as bb
from oracle import pyoracle as po
from tests.mexstub import call_gateway, call_ref_gateway

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built")]


def same(a, b):
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


@pytest.fixture(scope="module")
def state():
    """A mid-run state of a small beam (positions, stretches, forces)."""
    inp = bb.beam.build(bb.beam.small(nx=16, ny=4, nz=5))
    r = po.Run(inp, law="exponential", scheme="eulercromer", rate=-4e-6)
    r.step(80)
    return inp, r


def pair(name, ref_symbol, make_args, outputs):
    a, b = make_args(), make_args()
    n_err, msg = call_gateway(name, a)
    assert n_err == 0, msg
    call_ref_gateway(po.ref(), ref_symbol, b)
    for i in outputs:
        assert same(np.asarray(a[i]), np.asarray(b[i])), (name, i)


def test_deformedlength(state):
    inp, r = state
    nB = inp["nBonds"]
    x = np.asfortranarray(r.get("deformed"))
    pair("calculatedeformedlengthMex", "ref_mex_calculatedeformedlength",
         lambda: [x, inp["BONDLIST"], inp["UNDEFORMEDLENGTH"]] + [np.zeros(nB) for _ in range(5)], range(3, 8))


def test_bsfexponential(state):
    inp, r = state
    nB = inp["nBonds"]
    s = r.get("stretch")
    s0, sc = np.full(nB, 1e-4), np.full(nB, 2e-3)
    BT = np.zeros(nB)
    BSF0, f0 = r.get("bsf"), r.get("flag")
    mk = lambda: [s, s0, sc, 25.0, 0.25, np.zeros(nB), BSF0.copy(), BT, f0.copy()]
    a, b = mk(), mk()
    assert call_gateway("calculatebsfexponentialMex", a)[0] == 0
    call_ref_gateway(po.ref(), "ref_mex_calculatebsfexponential", b)
    assert same(a[8], b[8])
    np.testing.assert_allclose(a[6], b[6], rtol=1e-12, atol=0)


def test_bondforces(state):
    inp, r = state
    nB = inp["nBonds"]
    a = r.arr
    mk = lambda: [np.zeros(nB), np.zeros(nB), np.zeros(nB), a["fail"], a["dX"], a["dY"], a["dZ"], a["L"], a["s"],
                  np.zeros(nB), inp["BONDSTIFFNESS"], inp["cellVolume"], inp["VOLUMECORRECTIONFACTORS"], a["BSF"]]
    pair("calculatebondforcesMex", "ref_mex_calculatebondforces", mk, (0, 1, 2))


@pytest.mark.parametrize("name,sym,nargs", [
    ("calculatenodalforcesopenmpMex", "ref_mex_calculatenodalforcesopenmp", 8),
    ("calculatenodalforcesMex", "ref_mex_calculatenodalforces", 5)])
def test_nodalforces(state, name, sym, nargs):
    inp, r = state
    nN = inp["nNodes"]
    a = r.arr

    def mk():
        args = [inp["BONDLIST"], np.zeros((nN, 3), order="F"), a["fX"], a["fY"], a["fZ"]]
        if nargs == 8:
            args += [np.zeros((nN, 8), order="F") for _ in range(3)]
        return args
    pair(name, sym, mk, (1,))


def test_eulercromer(state):
    inp, r = state
    nN = inp["nNodes"]
    F, v, u, x = (np.asfortranarray(r.get(f)) for f in ("force", "velocity", "displacement", "deformed"))
    mk = lambda: [np.zeros((nN, 3), order="F"), F, 0.0, v.copy(order="F"), inp["DENSITY"], inp["CONSTRAINTFLAG"],
                  inp["DT"], u.copy(order="F"), x.copy(order="F"), inp["undeformedCoordinates"]]
    pair("timeintegrationeulercromerMex", "ref_mex_timeintegrationeulercromer", mk, (0, 3, 7, 8))


def test_bondfailure(state):
    inp, r = state
    nB = inp["nBonds"]
    s = r.get("stretch")
    BT = np.zeros(nB)
    BT[::7] = 1
    BT[::11] = 2
    mk = lambda: [np.ones(nB), 0.0, BT, s, 1e-3, 2e-3]
    pair("calculatebondfailureMex", "ref_mex_calculatebondfailure", mk, (0,))
