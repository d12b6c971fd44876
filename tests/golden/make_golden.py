"""Generate the golden vectors under tests/golden/ from the reference's own MEX
routines (compiled from the reference sources by oracle/Makefile into
oracle/_ref/libbbpd_ref.so) on small seeded inputs.

    make -C oracle REF=<reference tree>      # builds oracle/_ref/libbbpd_ref.so
    python tests/golden/make_golden.py

Each .npz holds the inputs and the reference's outputs. The reference ships no
tests or fixtures of its own; these vectors pin both the C restatement in
oracle/ and the CUDA routines to the reference's compiled code.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402

P = po.P


def lattice(nx, ny, nz, dx, hf=3.015, jitter=0.0, rng=None):
    """Small lattice and its bond list (i < j, sorted), 1-based, as doubles."""
    idx = np.arange(nx * ny * nz)
    a, b, c = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    X = np.stack([(a + 1) * dx, (b + 1) * dx, (c + 1) * dx], axis=1)
    if jitter:
        X = X + rng.uniform(-jitter, jitter, X.shape) * dx
    bonds = []
    r2 = (hf * dx) ** 2
    for i in range(len(X)):
        d = ((X[i + 1:] - X[i]) ** 2).sum(1)
        for j in np.nonzero(d <= r2)[0]:     # j indexes X[i + 1:]
            bonds.append((i + 1, i + 2 + j))
    bl = np.asfortranarray(np.array(bonds, dtype=np.float64))
    return np.asfortranarray(X), bl


def gen_deformedlength(rng):
    X, bl = lattice(7, 4, 3, 5e-3, jitter=0.05, rng=rng)
    nN, nB = len(X), len(bl)
    i, j = bl[:, 0].astype(int) - 1, bl[:, 1].astype(int) - 1
    L0 = np.sqrt(((X[i] - X[j]) ** 2).sum(1))
    x = np.asfortranarray(X + rng.normal(0, 1e-5, X.shape))
    out = {k: np.zeros(nB) for k in ("L", "dX", "dY", "dZ", "s")}
    po.ref().ref_calculatedeformedlength(P(x), P(bl), P(L0), nB, nN, P(out["L"]), P(out["dX"]),
                                         P(out["dY"]), P(out["dZ"]), P(out["s"]))
    return dict(x=x, bl=bl, L0=L0, **out)


def stretch_sample(rng, n, s0, sc):
    """Stretches in every branch of the laws, including exact breakpoints."""
    s = np.concatenate([
        rng.uniform(-2e-4, s0, n // 4),
        rng.uniform(s0, sc, n // 4),
        rng.uniform(sc, 3 * sc, n // 4),
        np.array([0.0, s0, sc, np.nextafter(s0, 1), np.nextafter(sc, 1), -1e-3, 3 * sc,
                  np.nextafter(3 * sc, 1), 1.0]),
        rng.uniform(-1e-3, 5e-3, n - 3 * (n // 4) - 9),
    ])
    return s


def gen_bsfexponential(rng):
    n = 4000
    s0v, scv = 1e-4, 2e-3
    s = stretch_sample(rng, n, s0v, scv)
    s0 = np.full(n, s0v)
    sc = scv * np.exp(rng.normal(0, 0.1, n))
    sc[: n // 8] = scv
    BT = rng.choice([0.0, 1.0, 2.0], n, p=[0.8, 0.1, 0.1])
    BSF0 = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
    BSF0[:5] = [0.0, 1.0, 0.5, 0.99, 0.0]
    flag0 = (rng.random(n) < 0.2).astype(np.float64)
    bsf = np.zeros(n)
    BSF, flag = BSF0.copy(), flag0.copy()
    po.ref().ref_calculatebsfexponential(P(s), P(s0), P(sc), 25.0, 0.25, P(bsf), P(BSF), P(BT), P(flag), n)
    return dict(s=s, s0=s0, sc=sc, BT=BT, BSF0=BSF0, flag0=flag0, k=25.0, alpha=0.25,
                bsf=bsf, BSF=BSF, flag=flag)


def gen_bondforces(rng):
    n = 3000
    fail = (rng.random(n) < 0.9).astype(np.float64)
    dX, dY, dZ = (rng.normal(0, 5e-3, n) for _ in range(3))
    L = np.sqrt(dX * dX + dY * dY + dZ * dZ)
    dX[:3] = dY[:3] = dZ[:3] = L[:3] = 0.0          # 0/0 -> NaN -> 0 guard
    s = rng.uniform(-1e-3, 3e-3, n)
    sp = np.zeros(n)
    BS = rng.uniform(1e18, 5e18, n)
    VCF = rng.choice([1.0, 0.5, 0.2], n)
    BSF = np.where(rng.random(n) < 0.3, rng.random(n), 0.0)
    BSF[3:6] = 1.0
    V = 1.25e-7
    out = {k: np.zeros(n) for k in ("fX", "fY", "fZ")}
    po.ref().ref_calculatebondforces(P(out["fX"]), P(out["fY"]), P(out["fZ"]), P(fail), P(dX), P(dY),
                                     P(dZ), P(L), P(s), P(sp), P(BS), V, P(VCF), P(BSF), n)
    return dict(fail=fail, dX=dX, dY=dY, dZ=dZ, L=L, s=s, sp=sp, BS=BS, V=V, VCF=VCF, BSF=BSF, **out)


def gen_nodalforces(rng):
    X, bl = lattice(6, 5, 4, 5e-3)
    nN, nB = len(X), len(bl)          # nB is not a multiple of 8: uneven chunks
    fX, fY, fZ = (rng.normal(0, 1e6, nB) for _ in range(3))
    F_omp = np.zeros((nN, 3), order="F")
    scr = [np.zeros(nN * 8) for _ in range(3)]
    po.ref().ref_calculatenodalforces_omp(nB, nN, P(bl), P(F_omp), P(fX), P(fY), P(fZ), *(P(a) for a in scr))
    F_ser = np.zeros((nN, 3), order="F")
    po.ref().ref_calculatenodalforces_serial(nB, nN, P(bl), P(F_ser), P(fX), P(fY), P(fZ))
    return dict(bl=bl, nN=nN, fX=fX, fY=fY, fZ=fZ, F_omp=F_omp, F_serial=F_ser)


def gen_eulercromer(rng):
    nN = 500
    a = np.zeros((nN, 3), order="F")
    F = np.asfortranarray(rng.normal(0, 1e9, (nN, 3)))
    v0 = np.asfortranarray(rng.normal(0, 1e-2, (nN, 3)))
    rho = rng.uniform(2000, 8000, nN)
    CF = np.asfortranarray((rng.random((nN, 3)) < 0.1).astype(np.float64))
    u0 = np.asfortranarray(rng.normal(0, 1e-5, (nN, 3)))
    X = np.asfortranarray(rng.uniform(0, 0.5, (nN, 3)))
    x = np.zeros((nN, 3), order="F")
    D, dt = 0.3, 1.0122532852569628e-06
    v, u = v0.copy(order="F"), u0.copy(order="F")
    po.ref().ref_timeintegrationeulercromer(P(a), P(F), D, P(v), P(rho), P(CF), dt, P(u), P(x), P(X), nN, 3)
    return dict(F=F, v0=v0, rho=rho, CF=CF, u0=u0, X=X, D=D, dt=dt, a=a, v=v, u=u, x=x)


def gen_bondfailure(rng):
    n = 3000
    scv, scs = 2e-3, 1e-2
    s = np.concatenate([rng.uniform(0, 4 * scv, n - 1000), rng.uniform(0, 2 * scs, 991),
                        [scv, 3 * scv, scs, np.nextafter(scv, 1), np.nextafter(3 * scv, 1),
                         np.nextafter(scs, 1), 0.0, -1.0, 1.0]])
    BT = rng.choice([0.0, 1.0, 2.0], n)
    fail0 = (rng.random(n) < 0.95).astype(np.float64)
    out = {}
    for ff in (0.0, 1.0):
        f = fail0.copy()
        po.ref().ref_calculatebondfailure(P(f), ff, P(BT), P(s), scv, scs, n)
        out[f"fail_ff{int(ff)}"] = f
    return dict(s=s, BT=BT, fail0=fail0, sc=scv, scSteel=scs, **out)


def gen_loop(rng):
    """The reference's MEX chain (dynamicsolverdisplacementcontrolled.m:79-105)
    for 150 steps of a small notched-free beam, exponential law, Euler-Cromer."""
    from bb_pd_b200 import beam
    inp = beam.build(beam.small(nx=14, ny=4, nz=5))
    keys = ("undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH", "BONDSTIFFNESS",
            "VOLUMECORRECTIONFACTORS", "DENSITY", "massVector", "CONSTRAINTFLAG", "BODYFORCEFLAG")
    fix = {k: inp[k] for k in keys}
    fix.update(nNodes=inp["nNodes"], nBonds=inp["nBonds"], DT=inp["DT"], cellVolume=inp["cellVolume"])
    kw = dict(law="exponential", scheme="eulercromer", rate=-4e-6, sc=2e-3, s0=1e-4)
    r = po.Run(fix, kernels="reference", **kw)
    r.step(150)
    out = {f: r.get(f) for f in ("displacement", "velocity", "force", "deformed", "acceleration", "bsf", "flag", "fail")}
    fix["steps"] = 150
    fix["rate"] = kw["rate"]
    return dict(**fix, **{"out_" + k: v for k, v in out.items()})


def main():
    if not po.ref_available():
        sys.exit("oracle/_ref/libbbpd_ref.so missing: run `make -C oracle REF=<reference tree>`")
    rng = np.random.default_rng(20261203)
    gens = [("deformedlength", gen_deformedlength), ("bsfexponential", gen_bsfexponential),
            ("bondforces", gen_bondforces), ("nodalforces", gen_nodalforces),
            ("eulercromer", gen_eulercromer), ("bondfailure", gen_bondfailure),
            ("loop_ec_exponential", gen_loop)]
    for name, g in gens:
        d = g(rng)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **d)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
