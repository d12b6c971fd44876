"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU checkers.

    liboracle.so     C restatement of the BB_PD hot path (bbpd_oracle.c)
    libbbpd_ref.so   the reference's own MEX routines compiled from their sources

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker. The product (bb_pd_b200/) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbbpd_ref.so")

LAW = {"linear": 0, "bilinear": 1, "trilinear": 2, "exponential": 3}
SCHEME = {"eulercromer": 0, "adr": 1}
AMP = {"linear": 0, "smoothstep": 1}

_P = C.POINTER(C.c_double)


class OrcPenetrator(C.Structure):
    _fields_ = [("cx", C.c_double), ("cz", C.c_double), ("radius", C.c_double), ("increment", C.c_double),
                ("family", _P), ("nFamily", C.c_int64), ("reaction", C.c_int)]


class OrcProblem(C.Structure):
    _fields_ = [
        ("nNodes", C.c_int64), ("nBonds", C.c_int64), ("X", _P), ("bl", _P), ("L0", _P),
        ("BS", _P), ("VCF", _P), ("BT", _P), ("sp", _P), ("s0", _P), ("s1", _P), ("sc", _P),
        ("s0v", C.c_double), ("s1v", C.c_double), ("scv", C.c_double), ("scSteel", C.c_double),
        ("kexp", C.c_double), ("alphaexp", C.c_double), ("beta", C.c_double),
        ("failureFunctionality", C.c_double), ("V", C.c_double), ("dt", C.c_double),
        ("damping", C.c_double), ("rho", _P), ("mass", _P), ("CF", _P), ("PF", _P),
        ("law", C.c_int), ("scheme", C.c_int), ("amplitude", C.c_int), ("nChunks", C.c_int),
        ("rate", C.c_double), ("appliedFinal", C.c_double), ("nTimeSteps", C.c_int64),
        ("cnOrder", C.c_int), ("nPen", C.c_int), ("pen", OrcPenetrator * 4),
    ]


class OrcState(C.Structure):
    _fields_ = [("step", C.c_int64), ("cn", C.c_double)] + [
        (n, _P) for n in ("x", "u", "v", "a", "F", "Fp", "fail", "BSF", "flag", "L", "dX", "dY",
                          "dZ", "s", "fX", "fY", "fZ", "bsf", "nfX", "nfY", "nfZ")] + [
        ("penCz", C.c_double * 4), ("reaction", C.c_double)]


def build(ref_dir: str | None = None) -> None:
    """Compile the restatement (and the reference MEX routines when the
    reference tree is present)."""
    cmd = ["make", "-C", HERE, "-s"]
    if ref_dir:
        cmd.append(f"REF={ref_dir}")
    subprocess.run(cmd, check=True)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_tree_sum.restype = C.c_double
        L.orc_tree_sum.argtypes = [_P, C.c_int64]
        L.orc_damping_coefficient_seq.restype = C.c_double
        L.orc_damping_coefficient_tree.restype = C.c_double
        for n in ("orc_damping_coefficient_seq", "orc_damping_coefficient_tree"):
            getattr(L, n).argtypes = [_P, _P, _P, C.c_double, _P, _P, C.c_int64]
        L.orc_cn_from_sums.restype = C.c_double
        L.orc_cn_from_sums.argtypes = [C.c_double, C.c_double]
        L.orc_smoothstep.restype = C.c_double
        L.orc_smoothstep.argtypes = [C.c_double] * 5
        L.orc_restated_kernels.restype = C.c_void_p
        L.orc_use_cr_exp.argtypes = [C.c_int]
        L.orc_load_reference.restype = C.c_void_p
        L.orc_load_reference.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.orc_run.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState), C.c_void_p, C.c_int64]
        L.orc_init_state.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcState)]
        L.orc_chunk_range.argtypes = [C.c_int64, C.c_int, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_deformedlength.argtypes = [_P, _P, _P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P]
        L.orc_bsf_exponential.argtypes = [_P, _P, C.c_int, _P, C.c_int, C.c_double, C.c_double, _P, _P, _P, _P, C.c_int64]
        L.orc_bsf_trilinear.argtypes = [_P, _P, C.c_int, _P, C.c_int, _P, C.c_int, C.c_double, _P, _P, _P, C.c_int64]
        L.orc_bsf_bilinear.argtypes = [_P, _P, C.c_int, _P, C.c_int, _P, _P, _P, C.c_int64]
        L.orc_bondfailure.argtypes = [_P, C.c_double, _P, _P, _P, C.c_int, C.c_double, C.c_int64]
        L.orc_damage.argtypes = [_P, _P, _P, C.c_int64, C.c_int64, _P]
        L.orc_buildhorizons.argtypes = [_P, C.c_int64, C.c_double, C.c_int64, _P, _P, _P, _P, _P]
        L.orc_buildhorizons.restype = C.c_int64
        L.orc_volumecorrection.argtypes = [_P, C.c_int64, C.c_double, C.c_double, _P]
        L.orc_bonddata.argtypes = [_P, C.c_int64, _P, _P, C.c_double, C.c_double, C.c_double, C.c_double,
                                   _P, _P, _P, _P]
        L.orc_massmatrix.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_double, _P, _P]
        L.orc_buildnotch.argtypes = [_P, C.c_int64, _P, _P, C.c_int64, C.c_double, C.c_double, C.c_double,
                                     _P, _P, _P, _P, _P]
        L.orc_buildnotch.restype = C.c_int64
        L.orc_stiffness_coo.argtypes = [_P, C.c_int64, C.c_int, _P, _P, C.c_double, _P, _P, _P, _P, C.c_int64,
                                        C.c_int64, _P, _P, _P, _P]
        L.orc_stiffness_coo.restype = C.c_int64
        L.orc_damageenergy.argtypes = [_P, _P, _P, _P, _P, C.c_double, C.c_double, C.c_double, _P, C.c_int64]
        L.orc_bondforces.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_double, _P, _P, C.c_int64]
        L.orc_nodalforces_chunked.argtypes = [C.c_int64, C.c_int64, _P, _P, _P, _P, _P, C.c_int]
        L.orc_eulercromer.argtypes = [_P, _P, C.c_double, _P, _P, _P, C.c_double, _P, _P, _P, C.c_int64, C.c_int]
        L.orc_adr_integrate.argtypes = [C.c_int64, C.c_double, _P, _P, _P, C.c_double, _P, _P, _P, C.c_int64]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    """The reference's compiled MEX routines (computational functions prefixed ref_,
    gateways prefixed ref_mex_)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        R = C.CDLL(REF_SO)
        i, d = C.c_int, C.c_double
        R.ref_calculatedeformedlength.argtypes = [_P, _P, _P, i, i, _P, _P, _P, _P, _P]
        R.ref_calculatebsfexponential.argtypes = [_P, _P, _P, d, d, _P, _P, _P, _P, i]
        R.ref_calculatebondforces.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, d, _P, _P, i]
        R.ref_calculatenodalforces_omp.argtypes = [i, i, _P, _P, _P, _P, _P, _P, _P, _P]
        R.ref_calculatenodalforces_serial.argtypes = [i, i, _P, _P, _P, _P, _P]
        R.ref_timeintegrationeulercromer.argtypes = [_P, _P, d, _P, _P, _P, d, _P, _P, _P, i, i]
        R.ref_calculatebondfailure.argtypes = [_P, d, _P, _P, d, d, i]
        _ref = R
    return _ref


def P(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags["F_CONTIGUOUS"] or a.flags["C_CONTIGUOUS"])
    return a.ctypes.data_as(_P)


def f64(a):
    return None if a is None else np.asfortranarray(a, dtype=np.float64)


class Run:
    """The time loop of the reference on the CPU (restated, or with the
    reference's compiled MEX routines for every step they cover)."""

    def __init__(self, inp: dict, *, law="exponential", scheme="eulercromer", n_chunks=8,
                 amplitude="linear", rate=0.0, applied_final=0.0, n_time_steps=0,
                 s0=1e-4, s1=3e-4, sc=2e-3, sc_steel=1.0, k_exp=25.0, alpha_exp=0.25,
                 beta_tri=0.25, failure_functionality=0.0, damping=0.0, dt=None,
                 cell_volume=None, per_bond_sc=None, cn_order="tree", kernels="restated",
                 penetrators=(), law_exp="libm"):
        L = lib()
        nN, nB = int(inp["nNodes"]), int(inp["nBonds"])
        self.nN, self.nB = nN, nB
        if law_exp not in ("libm", "cr") or (law_exp == "cr" and kernels != "restated"):
            raise ValueError("law_exp is 'libm', or 'cr' with the restated kernels")
        self.law_exp = law_exp
        self.keep = {k: f64(inp.get(k)) for k in (
            "undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH", "BONDSTIFFNESS",
            "VOLUMECORRECTIONFACTORS", "BONDTYPE", "stretchPlastic", "DENSITY", "massVector",
            "CONSTRAINTFLAG", "BODYFORCEFLAG")}
        if per_bond_sc is None:
            per_bond_sc = "sc" in inp
        sc_arr = f64(inp["sc"]) if per_bond_sc else None
        self.keep["sc"] = sc_arr
        p = OrcProblem()
        p.nNodes, p.nBonds = nN, nB
        k = self.keep
        p.X, p.bl, p.L0 = P(k["undeformedCoordinates"]), P(k["BONDLIST"]), P(k["UNDEFORMEDLENGTH"])
        p.BS, p.VCF, p.BT = P(k["BONDSTIFFNESS"]), P(k["VOLUMECORRECTIONFACTORS"]), P(k["BONDTYPE"])
        p.sp = P(k["stretchPlastic"])
        p.s0 = p.s1 = None
        p.sc = P(sc_arr)
        p.s0v, p.s1v, p.scv, p.scSteel = s0, s1, sc, sc_steel
        p.kexp, p.alphaexp, p.beta, p.failureFunctionality = k_exp, alpha_exp, beta_tri, failure_functionality
        p.V = cell_volume if cell_volume is not None else inp.get("cellVolume", 1.0)
        p.dt = dt if dt is not None else inp.get("DT", 1.0)
        p.damping = damping
        p.rho, p.mass = P(k["DENSITY"]), P(k["massVector"])
        p.CF, p.PF = P(k["CONSTRAINTFLAG"]), P(k["BODYFORCEFLAG"])
        p.law, p.scheme, p.amplitude, p.nChunks = LAW[law], SCHEME[scheme], AMP[amplitude], n_chunks
        p.rate, p.appliedFinal, p.nTimeSteps = rate, applied_final, n_time_steps
        p.cnOrder = 0 if cn_order == "tree" else 1
        # contact bodies: dicts with centre_x, centre_z, radius, increment, family (1-based ids), reaction
        self.fam = [f64(np.asarray(q["family"], dtype=np.float64)) for q in penetrators]
        p.nPen = len(penetrators)
        for j, q in enumerate(penetrators):
            pp = p.pen[j]
            pp.cx, pp.cz, pp.radius, pp.increment = q["centre_x"], q["centre_z"], q["radius"], q["increment"]
            pp.family, pp.nFamily, pp.reaction = P(self.fam[j]), len(self.fam[j]), int(q.get("reaction", 0))
        self.p = p
        z3 = lambda: np.zeros((nN, 3), order="F")
        zb = lambda: np.zeros(nB)
        self.arr = dict(x=z3(), u=z3(), v=z3(), a=z3(), F=z3(), Fp=z3(), fail=zb(), BSF=zb(),
                        flag=zb(), L=zb(), dX=zb(), dY=zb(), dZ=zb(), s=zb(), fX=zb(), fY=zb(),
                        fZ=zb(), bsf=zb(), nfX=np.zeros(nN * n_chunks), nfY=np.zeros(nN * n_chunks),
                        nfZ=np.zeros(nN * n_chunks))
        st = OrcState()
        for n, a in self.arr.items():
            setattr(st, n, P(a))
        self.st = st
        L.orc_init_state(C.byref(p), C.byref(st))
        if kernels == "reference":
            err = C.create_string_buffer(512)
            t = L.orc_load_reference(REF_SO.encode(), err, 512)
            if not t:
                raise RuntimeError(err.value.decode())
            self.kern = t
        else:
            self.kern = L.orc_restated_kernels()

    def step(self, n: int = 1) -> None:
        # the restated exponential law's exp: libm's (the reference's call) or
        # a correctly rounded one ("cr"); the compiled reference always uses libm
        lib().orc_use_cr_exp(1 if self.law_exp == "cr" else 0)
        lib().orc_run(C.byref(self.p), C.byref(self.st), self.kern, n)

    @property
    def next_step(self) -> int:
        return int(self.st.step)

    @property
    def cn(self) -> float:
        return float(self.st.cn)

    @property
    def reaction(self) -> float:
        """reactionForce of the last step (contact runs)."""
        return float(self.st.reaction)

    def get(self, field: str) -> np.ndarray:
        m = {"displacement": "u", "velocity": "v", "force": "F", "deformed": "x",
             "force_prev": "Fp", "acceleration": "a", "bsf": "BSF", "flag": "flag",
             "fail": "fail", "stretch": "s"}
        return self.arr[m[field]].copy()


def tree_sum(t: np.ndarray) -> float:
    t = np.ascontiguousarray(t, dtype=np.float64)
    return lib().orc_tree_sum(P(t), t.size)


def chunk_range(n: int, T: int, c: int) -> tuple[int, int]:
    lo, hi = C.c_int64(), C.c_int64()
    lib().orc_chunk_range(n, T, c, C.byref(lo), C.byref(hi))
    return lo.value, hi.value
