"""CPU tests of the C ABI: the library and the gateways load and export what
include/bbpd.h declares; without a GPU every compute entry fails loudly; the
host-side beam builder reproduces the reference input conventions."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import bb_pd_b200 as bb
from bb_pd_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "bbpd.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bbpd_\w+)\s*\(", txt)))


def test_header_symbols_exported():
    names = declared_functions()
    assert len(names) > 30
    lib = N.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_gateways_export_mexfunction():
    from bb_pd_b200.build import GATEWAYS
    for g in GATEWAYS:
        path = os.path.join(N.MEX_DIR, g + ".mexa64")
        assert os.path.exists(path), path
        so = C.CDLL(path)
        assert hasattr(so, "mexFunction")
        assert hasattr(so, "mexstub_error_count")


no_gpu = pytest.mark.skipif(N.device_count() > 0, reason="checks the no-GPU behaviour")


@no_gpu
def test_no_device_fails_loudly():
    inp = bb.beam.build(bb.beam.small(nx=8, ny=3, nz=3))
    with pytest.raises(bb.BBPDError) as e:
        bb.Solver(inp, law="trilinear", scheme="adr")
    assert e.value.status == N.ERR_NO_DEVICE
    nB = inp["nBonds"]
    z = lambda: np.zeros(nB)
    with pytest.raises(bb.BBPDError) as e:
        bb.routines.calculatedeformedlengthMex(inp["undeformedCoordinates"], inp["BONDLIST"],
                                               inp["UNDEFORMEDLENGTH"], z(), z(), z(), z(), z())
    assert e.value.status == N.ERR_NO_DEVICE


@no_gpu
def test_gateway_reports_error_through_mexerrmsgtxt():
    """A gateway with the right argument count reaches the library, which has no
    device here: the error comes back through mexErrMsgTxt, as in MATLAB."""
    from tests.mexstub import MxArray, call_gateway
    inp = bb.beam.build(bb.beam.small(nx=8, ny=3, nz=3))
    nB = inp["nBonds"]
    args = [inp["undeformedCoordinates"], inp["BONDLIST"], inp["UNDEFORMEDLENGTH"]] + [np.zeros(nB) for _ in range(5)]
    n_err, msg = call_gateway("calculatedeformedlengthMex", args)
    assert n_err == 1 and "no CUDA device" in msg
    n_err, msg = call_gateway("calculatedeformedlengthMex", args[:7])
    assert n_err == 1 and "Eight input arguments required" in msg


def test_beam_counts_match_reference_lattice():
    c1 = bb.beam.count(bb.beam.config1())
    assert (c1.n_nodes, c1.n_bonds) == (20000, 1005544)
    c2 = bb.beam.count(bb.beam.config2())
    assert (c2.n_nodes, c2.n_bonds) == (1280000, 74534404)
    c3 = bb.beam.count(bb.beam.config3())
    assert c3.n_nodes == 128000 and c3.n_bonds < 7096204      # notch removes bonds


def test_beam_arrays():
    inp = bb.beam.build(bb.beam.config1())
    X, bl = inp["undeformedCoordinates"], inp["BONDLIST"]
    nN, nB = inp["nNodes"], inp["nBonds"]
    i, j = bl[:, 0].astype(int) - 1, bl[:, 1].astype(int) - 1
    assert np.all(i < j) and np.all(np.diff(i) >= 0)            # i < j, rows sorted by i
    assert np.all(np.diff(j)[np.diff(i) == 0] > 0)             # then by j
    d = np.sqrt(((X[i] - X[j]) ** 2).sum(1))
    np.testing.assert_array_equal(d, inp["UNDEFORMEDLENGTH"])
    assert d.max() <= inp["horizon"]
    fam = np.bincount(i, minlength=nN) + np.bincount(j, minlength=nN)
    np.testing.assert_array_equal(fam, inp["nFAMILYMEMBERS"])
    assert fam.max() == 122
    vcf = inp["VOLUMECORRECTIONFACTORS"]
    assert np.all((vcf > 0) & (vcf <= 1))
    c = inp["bondStiffnessConcrete"]
    assert np.isclose(c, 18 * 37e9 / (np.pi * inp["horizon"] ** 4))
    interior = (fam[i] == 122) & (fam[j] == 122)
    np.testing.assert_allclose(inp["BONDSTIFFNESS"][interior], c * 2 * (4 / 3) * np.pi * inp["horizon"] ** 3
                               / (244 * inp["cellVolume"]), rtol=1e-14)
    # supports: bottom layer at x = 50 and 450 mm, all DOFs; load: midspan top, z only
    CF, PF = inp["CONSTRAINTFLAG"], inp["BODYFORCEFLAG"]
    sup = CF[:, 0] == 1
    assert sup.sum() == 20 and np.all(CF[sup] == 1)
    assert set(np.round(X[sup, 0] * 1000, 6)) == {50.0, 450.0} and np.all(X[sup, 2] == X[:, 2].min())
    pre = PF[:, 2] == 1
    assert pre.sum() == 20 and PF[:, :2].sum() == 0 and np.all(X[pre, 2] == X[:, 2].max())


def test_notch_removes_crossing_bonds():
    inp = bb.beam.build(bb.beam.config3())
    X, bl = inp["undeformedCoordinates"], inp["BONDLIST"]
    i, j = bl[:, 0].astype(int) - 1, bl[:, 1].astype(int) - 1
    xn = 0.2 + 0.625 * 0.15
    cross = (X[i, 0] - xn) * (X[j, 0] - xn) < 0
    t = (xn - X[i, 0]) / (X[j, 0] - X[i, 0] + 1e-300)
    zc = X[i, 2] + t * (X[j, 2] - X[i, 2])
    assert not np.any(cross & (zc <= X[:, 2].min() - 1.25e-3 + 0.04))   # none cut by the notch
    assert np.any(cross)                                                # bonds above it remain
    sc = inp["sc"]
    assert abs(sc.mean() / 2e-3 - 1) < 0.01 and abs(sc.std() / sc.mean() - 0.1) < 0.01


def test_python_api_validates_layout():
    with pytest.raises(TypeError):
        bb.routines.calculatedeformedlengthMex(np.zeros((4, 3), dtype=np.float32), None, None, None, None, None, None, None)
