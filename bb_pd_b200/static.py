"""Static (implicit) solver: displacement-controlled Newton-Raphson on the GPU.

The reference's static driver (solvers/scripts/static/newtonraphsondisplacementcontrolled.m)
moves the loaded DOFs by a fixed increment per load step and iterates to
equilibrium, assembling the tangent with buildstiffnessmatrixCSCformat.m and
solving it with MATLAB's iterative solvers. `StaticSolver` does the same on
resident device data with a matrix-free preconditioned conjugate gradient
(static.cu); `step()` returns the step's iteration counts and residuals.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .solver import _f64, make_params


class StaticStats(C.Structure):
    _fields_ = [("newton_iterations", C.c_int32), ("cg_iterations", C.c_int32), ("residual", C.c_double),
                ("reaction", C.c_double), ("converged", C.c_int32), ("reserved", C.c_int32)]


_L = None


def _lib():
    global _L
    if _L is None:
        L = N.lib()
        p = C.c_void_p
        L.bbpd_static_create.argtypes = [C.POINTER(N.Problem), C.POINTER(N.Params), C.c_int, C.POINTER(p)]
        L.bbpd_static_step.argtypes = [p, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                       C.POINTER(StaticStats)]
        L.bbpd_static_get.argtypes = [p, C.c_int, p]
        L.bbpd_static_destroy.argtypes = [p]
        _L = L
    return _L


class StaticSolver:
    """Quasi-static loading of a bond list: supports (CONSTRAINTFLAG) held,
    loaded DOFs (BODYFORCEFLAG) moved by `increment` at each step."""

    def __init__(self, inp: dict, device: int = 0, **kw):
        self.params = make_params(inp, **kw)
        self.nN, self.nB = int(inp["nNodes"]), int(inp["nBonds"])
        keep = {k: _f64(inp.get(k)) for k in (
            "undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH", "BONDSTIFFNESS", "VOLUMECORRECTIONFACTORS",
            "BONDTYPE", "fail", "CONSTRAINTFLAG", "BODYFORCEFLAG")}
        pb = N.Problem()
        pb.n_nodes, pb.n_bonds = self.nN, self.nB
        P = N.ptr
        pb.undeformed_coordinates = P(keep["undeformedCoordinates"])
        pb.bondlist = P(keep["BONDLIST"])
        pb.undeformed_length = P(keep["UNDEFORMEDLENGTH"])
        pb.bond_stiffness = P(keep["BONDSTIFFNESS"])
        pb.volume_correction = P(keep["VOLUMECORRECTIONFACTORS"])
        pb.bond_type = P(keep["BONDTYPE"])
        pb.fail = P(keep["fail"])
        pb.constraint_flag = P(keep["CONSTRAINTFLAG"])
        pb.prescribed_flag = P(keep["BODYFORCEFLAG"])
        h = C.c_void_p()
        N.check(_lib().bbpd_static_create(C.byref(pb), C.byref(self.params), device, C.byref(h)))
        self._h = h

    def step(self, increment: float, tol: float = 5e-3, max_newton: int = 50, cg_tol: float = 1e-10,
             max_cg: int = 20000) -> StaticStats:
        st = StaticStats()
        N.check(_lib().bbpd_static_step(self._h, float(increment), float(tol), int(max_newton), float(cg_tol),
                                        int(max_cg), C.byref(st)))
        return st

    def get(self, field: str) -> np.ndarray:
        fid = N.FIELD[field]
        out = np.zeros((self.nN, 3) if fid < 16 else (self.nB,), dtype=np.float64, order="F")
        N.check(_lib().bbpd_static_get(self._h, fid, N.ptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib().bbpd_static_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def buildstiffnessmatrixCSCformat(nodalCoordinates, BONDLIST, VOLUMECORRECTIONFACTORS, VOLUME, BONDSTIFFNESS,
                                  BFMULTIPLIER, fail, bondSofteningFactor, UNDEFORMEDLENGTH=None):
    """buildstiffnessmatrixCSCformat.m:1 on the GPU -> (globalRowIndex,
    globalColumnIndex, globalNonZeroValues, massVector)."""
    X = np.asfortranarray(nodalCoordinates, dtype=np.float64)
    n, nod = X.shape
    bl = np.asfortranarray(BONDLIST, dtype=np.float64)
    arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
            for a in (VOLUMECORRECTIONFACTORS, BONDSTIFFNESS, BFMULTIPLIER, fail, bondSofteningFactor)]
    nB = bl.shape[0]
    if bl.ndim != 2 or bl.shape[1] != 2 or any(a.size != nB for a in arrs):
        raise ValueError("need an nBonds x 2 BONDLIST and nBonds entries in every per-bond array")
    L = N.lib()
    p, i64 = C.c_void_p, C.c_int64
    L.bbpd_buildstiffnessmatrix.argtypes = [p, i64, C.c_int, p, p, C.c_double, p, p, p, p, i64, i64,
                                            C.POINTER(i64), p, p, p, p]
    P = lambda a: None if a is None else a.ctypes.data_as(p)
    nnz = C.c_int64()
    mass = np.zeros(n)
    vcf, bs, bfm, fl, bsf = arrs
    N.check(L.bbpd_buildstiffnessmatrix(P(X), n, nod, P(bl), P(vcf), float(VOLUME), P(bs), P(bfm), P(fl), P(bsf), nB,
                                        0, C.byref(nnz), None, None, None, P(mass)))
    m = nnz.value
    rows, cols, vals = np.zeros(m), np.zeros(m), np.zeros(m)
    N.check(L.bbpd_buildstiffnessmatrix(P(X), n, nod, P(bl), P(vcf), float(VOLUME), P(bs), P(bfm), P(fl), P(bsf), nB,
                                        m, C.byref(nnz), P(rows), P(cols), P(vals), None))
    return rows, cols, vals, mass
