"""Fused solver (bbpd_create / bbpd_step / bbpd_get): the reference time loop
of solvers/scripts/dynamic/dynamicsolverdisplacementcontrolled.m:71-143
(Euler-Cromer) or its ADR form, run on the GPU with state resident between calls.

    import bb_pd_b200 as bb
    inp = bb.beam.build(bb.beam.config1())
    s = bb.Solver(inp, law="trilinear", scheme="adr", rate=-1e-10)
    s.step(5000)
    u = s.get("displacement")          # nNodes x 3, column-major
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def default_params() -> N.Params:
    p = N.Params()
    N.lib().bbpd_params_default(C.byref(p))
    return p


def make_params(inp: dict | None = None, *, law: str | int = "exponential",
                scheme: str | int = "eulercromer", precision: str | int = "fp64",
                n_chunks: int = 8, amplitude: str | int = "linear", rate: float = 0.0,
                applied_final: float = 0.0, n_time_steps: int = 0, node_order: str = "input",
                s0: float = 1e-4, s1: float = 3e-4, sc: float = 2e-3, sc_steel: float = 1.0,
                k_exp: float = 25.0, alpha_exp: float = 0.25, beta_tri: float = 0.25,
                failure_functionality: float = 0.0, damping: float = 0.0,
                dt: float | None = None, cell_volume: float | None = None,
                guard_band: float = 1e-5, barrier_timeout_s: float = 2.0) -> N.Params:
    p = default_params()
    p.law = N.LAWS[law] if isinstance(law, str) else int(law)
    p.scheme = {"eulercromer": N.SCHEME_EULERCROMER, "adr": N.SCHEME_ADR}[scheme] if isinstance(scheme, str) else int(scheme)
    p.precision = {"fp64": N.PREC_FP64, "fp32": N.PREC_FP32}[precision] if isinstance(precision, str) else int(precision)
    p.n_chunks = n_chunks
    p.amplitude = {"linear": N.AMP_LINEAR, "smoothstep": N.AMP_SMOOTHSTEP}[amplitude] if isinstance(amplitude, str) else int(amplitude)
    p.node_order = {"input": N.ORDER_INPUT, "morton": N.ORDER_MORTON, "tiled": N.ORDER_TILED,
                    "lattice": N.ORDER_LATTICE}[node_order]
    p.rate, p.applied_final, p.n_time_steps = rate, applied_final, n_time_steps
    p.s0, p.s1, p.sc, p.sc_steel = s0, s1, sc, sc_steel
    p.k_exp, p.alpha_exp, p.beta_tri = k_exp, alpha_exp, beta_tri
    p.failure_functionality, p.damping = failure_functionality, damping
    p.guard_band, p.barrier_timeout_s = guard_band, barrier_timeout_s
    p.dt = dt if dt is not None else (inp["DT"] if inp and "DT" in inp else 1.0)
    p.cell_volume = cell_volume if cell_volume is not None else (inp["cellVolume"] if inp and "cellVolume" in inp else 1.0)
    return p


def _f64(a):
    if a is None:
        return None
    return np.asfortranarray(a, dtype=np.float64)


class Solver:
    """A problem resident on one GPU, advanced by a persistent kernel."""

    def __init__(self, inp: dict, params: N.Params | None = None, device: int = 0,
                 per_bond_sc: bool | None = None, **kw):
        self.params = params if params is not None else make_params(inp, **kw)
        self.nN, self.nB = int(inp["nNodes"]), int(inp["nBonds"])
        # keep the host arrays alive for the duration of bbpd_create
        keep = {k: _f64(inp.get(k)) for k in (
            "undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH", "BONDSTIFFNESS",
            "VOLUMECORRECTIONFACTORS", "BONDTYPE", "fail", "stretchPlastic", "DENSITY",
            "massVector", "CONSTRAINTFLAG", "BODYFORCEFLAG")}
        if per_bond_sc is None:
            per_bond_sc = "sc" in inp
        keep["s0"] = _f64(inp.get("s0")) if isinstance(inp.get("s0"), np.ndarray) else None
        keep["s1"] = _f64(inp.get("s1")) if isinstance(inp.get("s1"), np.ndarray) else None
        keep["sc"] = _f64(inp.get("sc")) if per_bond_sc else None
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
        pb.stretch_plastic = P(keep["stretchPlastic"])
        pb.s0, pb.s1, pb.sc = P(keep["s0"]), P(keep["s1"]), P(keep["sc"])
        pb.density = P(keep["DENSITY"])
        pb.mass = P(keep["massVector"])
        pb.constraint_flag = P(keep["CONSTRAINTFLAG"])
        pb.prescribed_flag = P(keep["BODYFORCEFLAG"])
        h = C.c_void_p()
        N.check(N.lib().bbpd_create(C.byref(pb), C.byref(self.params), device, C.byref(h)))
        self._h = h

    # -- time stepping --
    def step(self, nsteps: int = 1) -> None:
        N.check(N.lib().bbpd_step(self._h, nsteps))

    def step_async(self, nsteps: int = 1) -> None:
        N.check(N.lib().bbpd_step_async(self._h, nsteps))

    def sync(self) -> None:
        N.check(N.lib().bbpd_sync(self._h))

    def last_kernel_ms(self) -> float:
        ms = C.c_float()
        N.check(N.lib().bbpd_last_kernel_ms(self._h, C.byref(ms)))
        return float(ms.value)

    # -- state --
    def get(self, field: str) -> np.ndarray:
        fid = N.FIELD[field]
        out = np.zeros((self.nN, 3) if fid < 16 else (self.nB,), dtype=np.float64, order="F")
        N.check(N.lib().bbpd_get(self._h, fid, N.ptr(out)))
        return out

    def set(self, field: str, values: np.ndarray) -> None:
        fid = N.FIELD[field]
        a = np.asfortranarray(values, dtype=np.float64)
        N.check(N.lib().bbpd_set(self._h, fid, N.ptr(a)))

    @property
    def next_step(self) -> int:
        st, cn = C.c_int64(), C.c_double()
        N.check(N.lib().bbpd_get_step(self._h, C.byref(st), C.byref(cn)))
        return int(st.value)

    @property
    def cn(self) -> float:
        st, cn = C.c_int64(), C.c_double()
        N.check(N.lib().bbpd_get_step(self._h, C.byref(st), C.byref(cn)))
        return float(cn.value)

    def track_damage_energy(self) -> None:
        """Record, from now on, what calculatedamageenergy.m needs at every step;
        get("damage_energy") then returns the energy dissipated per bond."""
        N.check(N.lib().bbpd_track_damage_energy(self._h))

    def set_step(self, step: int, cn: float = 0.0) -> None:
        N.check(N.lib().bbpd_set_step(self._h, step, cn))

    def set_contact(self, penetrators: list[dict]) -> None:
        """Rigid cylinders applied after every integration (calculatecontactforce.m):
        dicts with centre_x, centre_z, radius, increment (per step), family
        (1-based node ids) and reaction (bool)."""
        self._fam = [np.ascontiguousarray(np.asarray(q["family"], dtype=np.float64)) for q in penetrators]
        arr = (N.Penetrator * max(1, len(penetrators)))()
        for j, q in enumerate(penetrators):
            a = arr[j]
            a.centre_x, a.centre_z, a.radius, a.increment = q["centre_x"], q["centre_z"], q["radius"], q["increment"]
            a.family, a.n_family, a.reaction = N.ptr(self._fam[j]), len(self._fam[j]), int(bool(q.get("reaction", 0)))
        N.check(N.lib().bbpd_set_contact(self._h, len(penetrators), arr))

    def set_probes(self, nodes, dofs) -> None:
        """Record the displacement of these DOFs (1-based node ids; dof 0 x,
        1 y, 2 z) at every step; CMOD is the difference of two x probes."""
        self._pn = np.ascontiguousarray(np.asarray(nodes, dtype=np.float64))
        self._pd = np.ascontiguousarray(np.asarray(dofs, dtype=np.int32))
        N.check(N.lib().bbpd_set_probes(self._h, len(self._pn), N.ptr(self._pn),
                                        self._pd.ctypes.data_as(C.POINTER(C.c_int32))))

    def probes(self, n: int) -> np.ndarray:
        """Probe values of the first n steps of the last launch, shape (n, n_probes)."""
        out = np.zeros((n, len(self._pn)), dtype=np.float64)
        N.check(N.lib().bbpd_get_probes(self._h, n, N.ptr(out)))
        return out

    def savedata(self, folder: str, name: str) -> str:
        """Write the state as savedata.m does (output/savedata.m:33-53): a .mat
        file `<name>_<step>.mat` with deformedCoordinates, fail and
        flagBondSoftening, step = the last completed time step."""
        import os
        import scipy.io
        step = self.next_step - 1
        os.makedirs(folder, exist_ok=True)
        path = os.path.join(folder, f"{name}_{step}.mat")
        scipy.io.savemat(path, {"deformedCoordinates": self.get("deformed"),
                                "fail": self.get("fail")[:, None],
                                "flagBondSoftening": self.get("flag")[:, None]})
        return path

    def reaction(self, n: int) -> np.ndarray:
        """Reaction of the first n steps of the last launch (ADR): the internal
        force summed over the prescribed DOFs; the applied load is its negative."""
        out = np.zeros(n, dtype=np.float64)
        N.check(N.lib().bbpd_get_reaction(self._h, n, N.ptr(out)))
        return out

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def info(self) -> dict:
        i = N.Info()
        N.check(N.lib().bbpd_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in N.Info._fields_}

    # -- checkpoint / resume (savedata / checkpoint of the solver script, :133-141) --
    FIELDS_NODAL = ("displacement", "velocity", "force", "force_prev", "deformed")
    FIELDS_BOND = ("bsf", "flag", "fail")

    def checkpoint(self) -> dict:
        ck = {f: self.get(f) for f in self.FIELDS_NODAL + self.FIELDS_BOND
              if not (f == "force_prev" and self.params.scheme != N.SCHEME_ADR)}
        ck["step"], ck["cn"] = self.next_step, self.cn
        return ck

    def restore(self, ck: dict) -> None:
        self.set_step(int(ck["step"]), float(ck["cn"]))
        for f in self.FIELDS_NODAL + self.FIELDS_BOND:
            if f in ck:
                self.set(f, ck[f])

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().bbpd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
