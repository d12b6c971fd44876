"""The reference's input module on the GPU, under its own function names.

Each function takes the arguments of the MATLAB function it replaces
(input/functions/buildhorizons.m, buildnotch.m, calculatevolumecorrectionfactors.m,
buildbonddata.m, solvers/functions/buildmassmatrix.m) and returns its outputs
in the same order, as float64 numpy arrays in MATLAB layout (column-major,
node ids 1-based). The work runs in libbbpd (builder.cu): a cell-list horizon
search instead of rangesearch, so families are listed by ascending node id
where rangesearch lists them by distance.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

_L = None


def _lib():
    global _L
    if _L is None:
        L = N.lib()
        p, d, i64 = C.c_void_p, C.c_double, C.c_int64
        L.bbpd_buildhorizons.argtypes = [p, i64, d, i64, C.POINTER(i64), p, p, p, p, p]
        L.bbpd_buildnotch.argtypes = [p, i64, p, p, i64, d, d, d, C.POINTER(i64), p, p, p, p, p]
        L.bbpd_calculatevolumecorrectionfactors.argtypes = [p, i64, d, d, p]
        L.bbpd_buildbonddata.argtypes = [p, i64, i64, p, p, d, d, d, d, p, p, p, p]
        L.bbpd_buildmassmatrix.argtypes = [i64, d, d, d, p, p]
        _L = L
    return _L


def _in(a, name, ndim=None):
    a = np.asfortranarray(np.asarray(a, dtype=np.float64))
    if ndim is not None and a.ndim != ndim:
        raise ValueError(f"{name} must have {ndim} dimension(s)")
    return a


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def buildhorizons(undeformedCoordinates, horizonRadius):
    """buildhorizons.m:1 -> (nFAMILYMEMBERS, NODEFAMILYPOINTERS, NODEFAMILY,
    BONDLIST, UNDEFORMEDLENGTH)."""
    X = _in(undeformedCoordinates, "undeformedCoordinates", 2)
    if X.shape[1] != 3:
        raise ValueError("undeformedCoordinates must be nNodes x 3")
    n = X.shape[0]
    nb = C.c_int64()
    nfam, fptr = np.zeros(n), np.zeros(n)
    N.check(_lib().bbpd_buildhorizons(_p(X), n, float(horizonRadius), 0, C.byref(nb), _p(nfam), _p(fptr),
                                      None, None, None))
    m = nb.value
    family = np.zeros(2 * m)
    bl = np.zeros((m, 2), order="F")
    L0 = np.zeros(m)
    N.check(_lib().bbpd_buildhorizons(_p(X), n, float(horizonRadius), m, C.byref(nb), None, None, _p(family),
                                      _p(bl), _p(L0)))
    return nfam, fptr, family, bl, L0


def buildnotch(undeformedCoordinates, BONDLIST, UNDEFORMEDLENGTH, DX, xlocation, depth):
    """buildnotch.m:1 -> (BONDLIST, UNDEFORMEDLENGTH, nFAMILYMEMBERS,
    NODEFAMILYPOINTERS, NODEFAMILY)."""
    X = _in(undeformedCoordinates, "undeformedCoordinates", 2)
    bl = _in(BONDLIST, "BONDLIST", 2)
    L0 = _in(UNDEFORMEDLENGTH, "UNDEFORMEDLENGTH").reshape(-1)
    n, nB = X.shape[0], bl.shape[0]
    if X.shape[1] != 3 or bl.shape[1] != 2 or L0.size != nB:
        raise ValueError("need nNodes x 3 coordinates, nBonds x 2 BONDLIST and nBonds lengths")
    m = C.c_int64()
    blo, L0o = np.zeros(2 * nB), np.zeros(nB)
    nfam, fptr, family = np.zeros(n), np.zeros(n), np.zeros(2 * nB)
    N.check(_lib().bbpd_buildnotch(_p(X), n, _p(bl), _p(L0), nB, float(DX), float(xlocation), float(depth),
                                   C.byref(m), _p(blo), _p(L0o), _p(nfam), _p(fptr), _p(family)))
    k = m.value
    return (np.asfortranarray(blo[:2 * k].reshape((k, 2), order="F")), L0o[:k].copy(), nfam, fptr,
            family[:2 * k].copy())


def calculatevolumecorrectionfactors(UNDEFORMEDLENGTH, horizon, RADIJ):
    """calculatevolumecorrectionfactors.m:1 -> VOLUMECORRECTIONFACTORS."""
    L0 = _in(UNDEFORMEDLENGTH, "UNDEFORMEDLENGTH").reshape(-1)
    out = np.zeros(L0.size)
    N.check(_lib().bbpd_calculatevolumecorrectionfactors(_p(L0), L0.size, float(horizon), float(RADIJ), _p(out)))
    return out


def buildbonddata(BONDLIST, nFAMILYMEMBERS, MATERIALFLAG, bondStiffnessConcrete, bondStiffnessSteel,
                  cellVolume, neighbourhoodVolume, VOLUMECORRECTIONFACTORS=None):
    """buildbonddata.m:1 -> (BONDSTIFFNESS, BONDTYPE, BFMULTIPLIER,
    stiffeningFactor). MATERIALFLAG None: every node concrete."""
    bl = _in(BONDLIST, "BONDLIST", 2)
    nfam = _in(nFAMILYMEMBERS, "nFAMILYMEMBERS").reshape(-1)
    mat = None if MATERIALFLAG is None else _in(MATERIALFLAG, "MATERIALFLAG").reshape(-1)
    if mat is not None and mat.size != nfam.size:
        raise ValueError("MATERIALFLAG and nFAMILYMEMBERS must have one entry per node")
    if bl.shape[1] != 2:
        raise ValueError("BONDLIST must be nBonds x 2")
    nB = bl.shape[0]
    bs, bt, bfm, sf = (np.zeros(nB) for _ in range(4))
    N.check(_lib().bbpd_buildbonddata(_p(bl), nB, nfam.size, _p(nfam), _p(mat), float(bondStiffnessConcrete),
                                      float(bondStiffnessSteel), float(cellVolume), float(neighbourhoodVolume),
                                      _p(bs), _p(bt), _p(bfm), _p(sf)))
    return bs, bt, bfm, sf


def buildmassmatrix(nNodes, DX, bondStiffnessConcrete, DT, nFAMILYMEMBERS):
    """buildmassmatrix.m:1 -> massVector."""
    nfam = _in(nFAMILYMEMBERS, "nFAMILYMEMBERS").reshape(-1)
    if nfam.size < int(nNodes):
        raise ValueError("nFAMILYMEMBERS needs nNodes entries")
    out = np.zeros(int(nNodes))
    N.check(_lib().bbpd_buildmassmatrix(int(nNodes), float(DX), float(bondStiffnessConcrete), float(DT), _p(nfam),
                                        _p(out)))
    return out
