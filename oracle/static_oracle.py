"""Test infrastructure, not product code: a CPU restatement of the static
(implicit) solver for checking the GPU one.

It follows solvers/scripts/static/newtonraphsondisplacementcontrolled.m:56-160:
the prescribed DOFs move by the increment. Each Newton iteration then updates
the bonds: calculatedeformedlength.m, the law (the bilinear law of
calculatebondsofteningfactor.m:42-48 restated here; the trilinear and
exponential laws through the oracle's C routines orc_bsf_trilinear and
orc_bsf_exponential; no softening for the linear law), and calculatebondfailure
with the law's sc. It forms the bond forces of
calculatebondforces.m:9-17 (BFMULTIPLIER included) and sums them over nodes in
bond order (calculatenodalforces.m:25-35), times cellVolume (driver :111).
The free nodes move by the solution of K delta = F, with K assembled as in
buildstiffnessmatrixCSCformat.m (NOD = 3). Each linear system is solved
directly (scipy's sparse LU), where the GPU uses a conjugate gradient; the two
agree to that solver's tolerance. Bond and nodal arithmetic keep the GPU
kernels' operation order, so the forces of the same positions agree bit for bit.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class StaticOracle:
    def __init__(self, inp: dict, law: str = "bilinear", s0: float = 1e-4, sc: float = 2e-3,
                 sc_steel: float = 1.0, failure_functionality: float = 0.0, cell_volume: float | None = None,
                 s1: float = 3e-4, beta_tri: float = 0.25, k_exp: float = 25.0, alpha_exp: float = 0.25):
        if law not in ("bilinear", "linear", "trilinear", "exponential"):
            raise ValueError("unknown law")
        self.law, self.s0, self.sc, self.sc_steel, self.ff = law, s0, sc, sc_steel, failure_functionality
        self.s1, self.beta, self.k, self.alpha = s1, beta_tri, k_exp, alpha_exp
        self.n, self.nB = int(inp["nNodes"]), int(inp["nBonds"])
        self.V = float(cell_volume if cell_volume is not None else inp["cellVolume"])
        self.X = np.asfortranarray(inp["undeformedCoordinates"], dtype=np.float64)
        self.x = self.X.copy(order="F")
        bl = np.asarray(inp["BONDLIST"], dtype=np.float64)
        self.a = bl[:, 0].astype(np.int64) - 1
        self.b = bl[:, 1].astype(np.int64) - 1
        self.L0 = np.asarray(inp["UNDEFORMEDLENGTH"], dtype=np.float64)
        self.BS = np.asarray(inp["BONDSTIFFNESS"], dtype=np.float64)
        self.VCF = np.asarray(inp["VOLUMECORRECTIONFACTORS"], dtype=np.float64)
        bt = inp.get("BONDTYPE")
        self.BT = np.zeros(self.nB, dtype=np.int64) if bt is None else np.asarray(bt).astype(np.int64)
        self.BFM = np.where(self.BT == 1, 3.0, 1.0)
        f0 = inp.get("fail")
        self.fail = np.ones(self.nB) if f0 is None else np.asarray(f0, dtype=np.float64).copy()
        self.bsf = np.zeros(self.nB)
        self.flag = np.zeros(self.nB)
        cf = np.asarray(inp["CONSTRAINTFLAG"]) == 1
        pf = np.asarray(inp["BODYFORCEFLAG"]) == 1
        self.held = np.where(cf, 1, np.where(pf, 2, 0)).astype(np.int8)   # (n, 3)
        self.F = np.zeros((self.n, 3), order="F")

    def _bonds(self):
        x = self.x
        d = x[self.b] - x[self.a]                                  # (nB, 3): x_b - x_a
        L = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        s = (L - self.L0) / self.L0
        B = self.bsf
        if self.law == "bilinear":
            f = self.flag.copy()
            f[(self.BT == 0) & (s > self.s0)] = 1
            with np.errstate(divide="ignore", invalid="ignore"):
                bs = ((s - self.s0) / s) * (self.sc / (self.sc - self.s0))
                cand = bs * f
            B = np.where(np.isnan(cand), B, np.where(np.isnan(B), cand, np.where(cand > B, cand, B)))
            B = np.where(B > 1, 1.0, B)
            B = np.where(np.isnan(B), 0.0, B)
            self.flag = f
        elif self.law in ("trilinear", "exponential"):
            from oracle import pyoracle as po
            lib, P = po.lib(), po.P
            s_c = np.ascontiguousarray(s)
            B = np.ascontiguousarray(B.copy())
            bt = np.ascontiguousarray(self.BT.astype(np.float64))
            flag = np.ascontiguousarray(self.flag.copy())
            s0a, s1a, sca = (np.array([v]) for v in (self.s0, self.s1, self.sc))
            if self.law == "trilinear":
                lib.orc_bsf_trilinear(P(s_c), P(s0a), 0, P(s1a), 0, P(sca), 0, self.beta, P(B), P(bt), P(flag), self.nB)
            else:
                scratch = np.zeros(self.nB)
                lib.orc_bsf_exponential(P(s_c), P(s0a), 0, P(sca), 0, self.k, self.alpha, P(scratch), P(B), P(bt),
                                      P(flag), self.nB)
            self.flag = flag
        self.bsf = B
        fl = self.fail
        fl = np.where((fl == 1) & (self.BT == 0) & (s > self.sc), self.ff, fl)
        fl = np.where((fl == 1) & (self.BT == 1) & (s > 3 * self.sc), self.ff, fl)
        fl = np.where((fl == 1) & (self.BT == 2) & (s > self.sc_steel), self.ff, fl)
        self.fail = fl
        t = self.BFM * fl * self.BS * (1 - B) * s * self.V * self.VCF
        with np.errstate(divide="ignore", invalid="ignore"):
            fb = t[:, None] * (d / L[:, None])
        fb[np.isnan(fb)] = 0.0
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            rig = np.where(fl == 1, self.BFM * ((self.BS / (L * L * L)) * self.VCF * (self.V * self.V)) * (1 - B), 0.0)
        rig[~np.isfinite(rig)] = 0.0
        return d, fb, rig

    def _nodal(self, fb):
        # node i gets +f of the bonds it starts and -f of those it ends, in bond order
        idx = np.empty(2 * self.nB, dtype=np.int64)
        idx[0::2], idx[1::2] = self.a, self.b
        F = np.zeros((self.n, 3))
        for c in range(3):
            v = np.empty(2 * self.nB)
            v[0::2], v[1::2] = fb[:, c], -fb[:, c]
            col = np.zeros(self.n)
            np.add.at(col, idx, v)
            F[:, c] = col * self.V
        return F

    def _stiffness(self, d, rig):
        n = self.n
        rows, cols, vals = [], [], []
        for u in range(3):
            for v in range(3):
                k = rig * d[:, u] * d[:, v]
                for (p, q, sgn) in ((self.a, self.a, 1), (self.b, self.b, 1), (self.a, self.b, -1), (self.b, self.a, -1)):
                    rows.append(3 * p + u)
                    cols.append(3 * q + v)
                    vals.append(sgn * k)
        K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(3 * n, 3 * n))
        return K.tocsr()

    def step(self, increment: float, tol: float = 5e-3, max_newton: int = 50):
        if increment != 0:
            self.x = np.where(self.held == 2, self.x + increment, self.x)
        free_dof = (self.held == 0).reshape(-1)           # node-major DOF index 3 i + c
        it = 0
        while True:
            d, fb, rig = self._bonds()
            self.F = self._nodal(fb)
            Fv = self.F.reshape(-1)
            rf = float(np.sqrt(np.sum(Fv[free_dof] ** 2)))
            rh = float(np.sqrt(np.sum(Fv[~free_dof] ** 2)))
            if rf <= tol * rh or rf == 0:
                return dict(newton_iterations=it, residual=rf, reaction=rh, converged=1)
            if it == max_newton:
                return dict(newton_iterations=it, residual=rf, reaction=rh, converged=0)
            K = self._stiffness(d, rig)
            solve = free_dof & (K.diagonal() > 0)
            idx = np.nonzero(solve)[0]
            delta = np.zeros(3 * self.n)
            delta[idx] = spla.spsolve(K[idx][:, idx].tocsc(), Fv[idx])
            self.x = self.x + delta.reshape(self.n, 3)
            it += 1

    def get(self, field: str) -> np.ndarray:
        return {"displacement": lambda: self.x - self.X, "deformed": lambda: self.x.copy(),
                "force": lambda: self.F.copy(), "bsf": lambda: self.bsf.copy(), "flag": lambda: self.flag.copy(),
                "fail": lambda: self.fail.copy()}[field]()
