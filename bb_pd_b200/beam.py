"""Synthetic concrete beams: the inputs the reference's MATLAB input module
builds (input/scripts/Gregoire_beam_tests.m), made by libbbpd's host builder.

`beam(...)` returns a dict of reference-named arrays, column-major like
MATLAB: undeformedCoordinates (nNodes x 3), BONDLIST (nBonds x 2, 1-based),
UNDEFORMEDLENGTH, BONDSTIFFNESS, VOLUMECORRECTIONFACTORS, nFAMILYMEMBERS,
DENSITY, massVector, CONSTRAINTFLAG, BODYFORCEFLAG (the prescribed DOFs),
and, with per-bond critical stretch, sc.
"""
from __future__ import annotations

import numpy as np

from . import _native as N


def spec(nx: int, ny: int, nz: int, dx: float, *, horizon_factor: float = 3.015,
         E: float = 37e9, stiffness_factor: float = 18.0, density: float = 2346.0,
         supports: tuple[float, ...] = (), load_midspan_top: bool = True,
         notch_x: float | None = None, notch_depth: float = 0.0,
         sc_lognormal: tuple[float, float] | None = None, seed: int = 20261203) -> N.BeamSpec:
    s = N.BeamSpec()
    s.nx, s.ny, s.nz, s.dx = nx, ny, nz, dx
    s.horizon_factor, s.E, s.stiffness_factor, s.density = horizon_factor, E, stiffness_factor, density
    for i, x in enumerate(supports[:2]):
        s.support_x[i] = x
    s.n_supports = min(len(supports), 2)
    s.load_midspan_top = int(load_midspan_top)
    s.notch = int(notch_x is not None)
    s.notch_x = notch_x if notch_x is not None else 0.0
    s.notch_depth = notch_depth
    s.sc_lognormal = int(sc_lognormal is not None)
    if sc_lognormal is not None:
        s.sc_mean, s.sc_cov = sc_lognormal
    s.seed = seed
    return s


def count(s: N.BeamSpec) -> N.BeamScalars:
    out = N.BeamScalars()
    N.check(N.lib().bbpd_beam_count(s, out))
    return out


def build(s: N.BeamSpec) -> dict:
    sc_ = count(s)
    nN, nB = sc_.n_nodes, sc_.n_bonds
    f = lambda *shape: np.zeros(shape, dtype=np.float64, order="F")
    a = dict(undeformedCoordinates=f(nN, 3), BONDLIST=f(nB, 2), UNDEFORMEDLENGTH=f(nB),
             BONDSTIFFNESS=f(nB), VOLUMECORRECTIONFACTORS=f(nB), nFAMILYMEMBERS=f(nN),
             DENSITY=f(nN), massVector=f(nN), CONSTRAINTFLAG=f(nN, 3), BODYFORCEFLAG=f(nN, 3))
    sc = f(nB) if s.sc_lognormal else None
    N.check(N.lib().bbpd_beam_build(
        s, N.ptr(a["undeformedCoordinates"]), N.ptr(a["BONDLIST"]), N.ptr(a["UNDEFORMEDLENGTH"]),
        N.ptr(a["BONDSTIFFNESS"]), N.ptr(a["VOLUMECORRECTIONFACTORS"]), N.ptr(a["nFAMILYMEMBERS"]),
        N.ptr(a["DENSITY"]), N.ptr(a["massVector"]), N.ptr(a["CONSTRAINTFLAG"]),
        N.ptr(a["BODYFORCEFLAG"]), N.ptr(sc)))
    if sc is not None:
        a["sc"] = sc
    a.update(nNodes=nN, nBonds=nB, horizon=sc_.horizon, cellVolume=sc_.cell_volume,
             bondStiffnessConcrete=sc_.bond_stiffness_concrete, DT=sc_.dt,
             nSupported=sc_.n_supported, nPrescribed=sc_.n_prescribed)
    return a


# The beams of the benchmark configurations. Dimensions: nx along the length,
# ny across the width, nz through the depth (loading direction z).
def config1() -> N.BeamSpec:
    """500 x 100 (depth) x 50 (width) mm, dx 5 mm: 100 x 10 x 20 = 20 000 nodes."""
    return spec(100, 10, 20, 5e-3, supports=(0.05, 0.45))


def config2() -> N.BeamSpec:
    """Same beam at dx 1.25 mm: 400 x 40 x 80 = 1 280 000 nodes."""
    return spec(400, 40, 80, 1.25e-3, supports=(0.05, 0.45))


def config3() -> N.BeamSpec:
    """400 x 100 x 50 mm at dx 2.5 mm (160 x 20 x 40 = 128 000 nodes), supports at
    50 and 350 mm, a 40 mm notch at 0.625 half-span right of midspan, lognormal sc."""
    L = 0.4
    half_span = 0.15
    notch = 0.2 + 0.625 * half_span  # 293.75 mm: between two node planes
    return spec(160, 20, 40, 2.5e-3, supports=(0.05, 0.35), notch_x=notch, notch_depth=0.04,
                sc_lognormal=(2e-3, 0.1))


def small(nx: int = 24, ny: int = 5, nz: int = 6, dx: float = 5e-3, **kw) -> N.BeamSpec:
    """A small beam for parity tests (supports at 2 dx from each end)."""
    kw.setdefault("supports", (3 * dx, (nx - 2) * dx))
    return spec(nx, ny, nz, dx, **kw)


def geometric_beam(depth: float, dx: float, *, span_to_depth: float = 5.0, width: float = 0.05,
                   **kw) -> N.BeamSpec:
    """A 3-point-bending beam of the given depth: span = span_to_depth x depth,
    half a depth of overhang at each end, supports on the bottom layer at the
    span ends, midspan top nodes under prescribed displacement."""
    span = span_to_depth * depth
    length = span + depth
    nx = max(4, int(round(length / dx)))
    nz = max(3, int(round(depth / dx)))
    ny = max(2, int(round(width / dx)))
    # support lines on node planes (nodes sit at dx * (k + 1))
    x0 = dx * (int(round(0.5 * depth / dx)) + 1)
    x1 = dx * (int(round((0.5 * depth + span) / dx)) + 1)
    return spec(nx, ny, nz, dx, supports=(x0 - 0.25 * dx, x1 - 0.25 * dx), **kw)


def size_effect_series(n: int = 64, seed: int = 20261203, depth_range=(0.05, 0.4), dx: float = 2.5e-3,
                       sc_mean: float = 2e-3, sc_cov: float = 0.1) -> list[tuple[N.BeamSpec, str]]:
    """Geometrically similar beams with log-uniform depths, span/depth 5, width
    50 mm, seeded lognormal critical stretch; laws alternate linear/trilinear.
    Returns (spec, law) pairs."""
    rng = np.random.default_rng(seed)
    depths = np.exp(rng.uniform(np.log(depth_range[0]), np.log(depth_range[1]), n))
    laws = rng.choice(["linear", "trilinear"], n)
    return [(geometric_beam(float(d), dx, sc_lognormal=(sc_mean, sc_cov), seed=seed + k), str(l))
            for k, (d, l) in enumerate(zip(depths, laws))]


def serving_stream(n: int = 200, seed: int = 20261203, nodes_range=(1e4, 1e6), rate_hz: float = 2.0,
                   dx_choices=(1.25e-3, 2.5e-3, 5e-3)) -> list[dict]:
    """Poisson arrivals of beam solves: node counts log-uniform in nodes_range,
    dx drawn from dx_choices, law uniform over the four laws. A beam of depth d
    is 6d long and d/2 wide, so nodes ~ 3 (d/dx)^3. Returns dicts with
    arrival (s), spec, law and nodes (estimate)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    laws = rng.choice(["linear", "bilinear", "trilinear", "exponential"], n)
    out = []
    for k in range(n):
        target = float(np.exp(rng.uniform(np.log(nodes_range[0]), np.log(nodes_range[1]))))
        dx = float(rng.choice(dx_choices))
        cells = (target / 3.0) ** (1.0 / 3.0)
        depth = cells * dx
        s = geometric_beam(depth, dx, width=0.5 * depth)
        out.append(dict(arrival=float(t[k]), spec=s, law=str(laws[k]), nodes=int(s.nx) * int(s.ny) * int(s.nz)))
    return out


def penetrator(inp: dict, centre_x: float, radius: float, search_radius: float, increment: float,
               *, top: bool = True, reaction: bool = True) -> dict:
    """A rigid cylinder (axis along y) resting on the top (or, for a support,
    under the bottom) surface at x = centre_x, as the reference's
    buildpenetrator.m and its centre correction build it: the family is every
    node within search_radius (x-z distance) of the centre, and the centre is
    moved until the nearest family node touches the cylinder."""
    X = np.asarray(inp["undeformedCoordinates"])
    z = X[:, 2].max() + radius if top else X[:, 2].min() - radius
    d = np.sqrt((X[:, 0] - centre_x) ** 2 + (X[:, 2] - z) ** 2)
    fam = np.nonzero(d < search_radius)[0]
    gap = d[fam].min() - radius
    z = z - gap if top else z + gap
    return dict(centre_x=float(centre_x), centre_z=float(z), radius=float(radius), increment=float(increment),
                family=(fam + 1).astype(np.float64), reaction=bool(reaction))
