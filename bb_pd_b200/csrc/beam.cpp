// Synthetic beam builder: the inputs that the reference's MATLAB input module
// produces for a regular-lattice concrete beam (input/scripts/Gregoire_beam_tests.m
// and the functions it calls), written as multi-threaded host code.
//
//   coordinates   buildmaterialpointcoordinates.m:39-59 (x fastest, X = dx * k, k from 1)
//   families      buildhorizons.m:13-97 (every node within the horizon; BONDLIST
//                 holds each pair once with i < j, rows sorted by i then j)
//   notch         buildnotch.m:13-119 + determineintersection.m:59-150 (bonds whose
//                 segment crosses a vertical rectangle are removed; family
//                 counts rebuilt from the reduced list)
//   VCF           calculatevolumecorrectionfactors.m:16-34 (RADIJ = dx / 2)
//   stiffness     buildbonddata.m:16-57 (surface correction 2 V_H / (n_i V + n_j V))
//   time step     Gregoire_beam_tests.m:244 (0.8 sqrt(2 rho dx / (pi d^2 dx c)))
//   ADR mass      buildmassmatrix.m:32-40 (0.25 dt^2 n_i dx^2 c / dx)
//
// The neighbour search replaces MATLAB's KD-tree rangesearch with the lattice
// stencil (integer offsets within the horizon); rangesearch orders each family
// by distance, this builder by node index. Both are valid bond lists.
#include "bbpd.h"
#include "bbpd_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Offset { int da, db, dc; };

struct Lattice {
    int nx, ny, nz;
    int64_t n;
    double dx, horizon;
    std::vector<Offset> offs;  // all offsets within the horizon, sorted by (dc, db, da)
};

bool make_lattice(const bbpd_beam_spec *s, Lattice &L)
{
    if (s->nx < 1 || s->ny < 1 || s->nz < 1 || !(s->dx > 0) || !(s->horizon_factor > 0))
        return false;
    L.nx = s->nx; L.ny = s->ny; L.nz = s->nz;
    L.n = (int64_t)s->nx * s->ny * s->nz;
    L.dx = s->dx;
    L.horizon = s->horizon_factor * s->dx;
    int r = (int)std::ceil(s->horizon_factor) + 1;
    double lim = s->horizon_factor * s->horizon_factor * (1.0 + 1e-12);
    for (int dc = -r; dc <= r; dc++)
        for (int db = -r; db <= r; db++)
            for (int da = -r; da <= r; da++) {
                if (!da && !db && !dc) continue;
                if ((double)(da * da + db * db + dc * dc) <= lim) L.offs.push_back({da, db, dc});
            }
    return true;
}

inline bool forward(const Offset &o)  // j > i in x-fastest order
{
    return o.dc > 0 || (o.dc == 0 && (o.db > 0 || (o.db == 0 && o.da > 0)));
}

template <class F>
void parallel_for(int64_t n, F fn)
{
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 4096) nt = 1;
    std::vector<std::thread> th;
    int64_t per = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        int64_t lo = (int64_t)t * per, hi = std::min(n, lo + per);
        if (lo >= hi) break;
        th.emplace_back([=]() { for (int64_t i = lo; i < hi; i++) fn(i); });
    }
    for (auto &x : th) x.join();
}

struct Beam {
    const bbpd_beam_spec *s;
    Lattice L;
    double zt = 0, ymin = 0, ymax = 0, zmin = 0;

    void coord(int64_t i, double *p) const
    {
        int64_t a = i % L.nx, b = (i / L.nx) % L.ny, c = i / ((int64_t)L.nx * L.ny);
        p[0] = L.dx * (double)(a + 1);
        p[1] = L.dx * (double)(b + 1);
        p[2] = L.dx * (double)(c + 1);
    }
    // neighbour of i at offset o, or -1 if outside the lattice
    int64_t nbr(int64_t i, const Offset &o) const
    {
        int64_t a = i % L.nx, b = (i / L.nx) % L.ny, c = i / ((int64_t)L.nx * L.ny);
        int64_t a2 = a + o.da, b2 = b + o.db, c2 = c + o.dc;
        if (a2 < 0 || a2 >= L.nx || b2 < 0 || b2 >= L.ny || c2 < 0 || c2 >= L.nz) return -1;
        return a2 + (int64_t)L.nx * (b2 + (int64_t)L.ny * c2);
    }
    // determineintersection.m:59-86 / plane_line_intersect :126-150 for the
    // notch rectangle x = notch_x, y in [ymin, ymax], z in [zmin, zt].
    bool crosses(int64_t i, int64_t j) const
    {
        if (!s->notch) return false;
        double P0[3], P1[3];
        coord(i, P0); coord(j, P1);
        double u = P1[0] - P0[0];
        double N = -(P0[0] - s->notch_x);
        if (std::fabs(u) < 1e-7) return false;     // parallel to the plane
        double sI = N / u;
        if (sI < 0 || sI > 1) return false;
        double Iy = P0[1] + sI * (P1[1] - P0[1]);
        double Iz = P0[2] + sI * (P1[2] - P0[2]);
        return ymin <= Iy && Iy <= ymax && zmin <= Iz && Iz <= zt;
    }
};

bool setup(const bbpd_beam_spec *s, Beam &B)
{
    B.s = s;
    if (!make_lattice(s, B.L)) return false;
    B.ymin = s->dx;
    B.ymax = s->dx * s->ny;
    B.zmin = s->dx;
    B.zt = (s->dx * 0.5) + s->notch_depth;   // notch height measured from the bottom face
    return true;
}

// forward-bond count of node i and its family size (after notch removal)
void node_counts(const Beam &B, int64_t i, int32_t *fwd, int32_t *fam)
{
    int f = 0, n = 0;
    for (const Offset &o : B.L.offs) {
        int64_t j = B.nbr(i, o);
        if (j < 0 || B.crosses(i, j)) continue;
        n++;
        if (forward(o)) f++;
    }
    *fwd = f;
    *fam = n;
}

uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

}  // namespace

static void beam_scalars(const bbpd_beam_spec *s, const Beam &B, bbpd_beam_scalars *o)
{
    double d = B.L.horizon;
    o->horizon = d;
    o->cell_volume = s->dx * s->dx * s->dx;                      // cellVolume = DX^3
    o->bond_stiffness_concrete = (s->stiffness_factor * s->E) / (M_PI * (d * d * d * d));
    double c = o->bond_stiffness_concrete;
    o->dt = (0.8 * std::sqrt(2 * s->density * s->dx / (M_PI * (d * d) * s->dx * c))) / 1.0;
}

extern "C" int bbpd_beam_count(const bbpd_beam_spec *spec, bbpd_beam_scalars *out)
{
    if (!spec || !out) return bbpd::fail(BBPD_ERR_ARG, "null argument");
    Beam B;
    if (!setup(spec, B)) return bbpd::fail(BBPD_ERR_ARG, "invalid beam spec");
    std::vector<int32_t> fwd(B.L.n), fam(B.L.n);
    parallel_for(B.L.n, [&](int64_t i) { node_counts(B, i, &fwd[i], &fam[i]); });
    int64_t nb = 0;
    for (int64_t i = 0; i < B.L.n; i++) nb += fwd[i];
    std::memset(out, 0, sizeof(*out));
    out->n_nodes = B.L.n;
    out->n_bonds = nb;
    beam_scalars(spec, B, out);
    int64_t ns = 0, np = 0;
    double xmid = 0.5 * (spec->dx + spec->dx * spec->nx), tol = 0.5 * spec->dx * (1 + 1e-9);
    for (int64_t i = 0; i < B.L.n; i++) {
        double p[3];
        B.coord(i, p);
        int64_t c = i / ((int64_t)B.L.nx * B.L.ny);
        for (int k = 0; k < spec->n_supports && k < 2; k++)
            if (c == 0 && std::fabs(p[0] - spec->support_x[k]) <= tol) { ns++; break; }
        if (spec->load_midspan_top && c == B.L.nz - 1 && std::fabs(p[0] - xmid) <= tol) np++;
    }
    out->n_supported = ns;
    out->n_prescribed = np;
    return BBPD_OK;
}

extern "C" int bbpd_beam_build(const bbpd_beam_spec *spec, double *X, double *bondlist,
                               double *L0, double *BS, double *VCF, double *nfam,
                               double *density, double *mass, double *CF, double *PF,
                               double *sc)
{
    if (!spec || !X || !bondlist || !L0 || !BS || !VCF || !nfam || !density || !mass ||
        !CF || !PF)
        return bbpd::fail(BBPD_ERR_ARG, "null array");
    if (spec->sc_lognormal && !sc) return bbpd::fail(BBPD_ERR_ARG, "sc array required");
    Beam B;
    if (!setup(spec, B)) return bbpd::fail(BBPD_ERR_ARG, "invalid beam spec");
    const int64_t n = B.L.n;
    std::vector<int32_t> fwd(n), fam(n);
    parallel_for(n, [&](int64_t i) { node_counts(B, i, &fwd[i], &fam[i]); });
    std::vector<int64_t> base(n + 1, 0);
    for (int64_t i = 0; i < n; i++) base[i + 1] = base[i] + fwd[i];
    const int64_t nb = base[n];
    bbpd_beam_scalars sca;
    beam_scalars(spec, B, &sca);
    const double d = B.L.horizon, V = sca.cell_volume, c = sca.bond_stiffness_concrete;
    const double VH = (4.0 / 3.0) * M_PI * (d * d * d);          // neighbourhoodVolume
    const double R = spec->dx / 2;                                // RADIJ
    const double dt = sca.dt;

    parallel_for(n, [&](int64_t i) {
        double p[3];
        B.coord(i, p);
        X[i] = p[0]; X[i + n] = p[1]; X[i + 2 * n] = p[2];
        nfam[i] = (double)fam[i];
        density[i] = spec->density;
        // buildmassmatrix.m:36-40
        double Kij = ((double)fam[i] * (spec->dx * spec->dx)) * (c / spec->dx);
        mass[i] = 0.25 * (dt * dt) * Kij;
        int64_t k = base[i];
        for (const Offset &o : B.L.offs) {
            if (!forward(o)) continue;
            int64_t j = B.nbr(i, o);
            if (j < 0 || B.crosses(i, j)) continue;
            double q[3];
            B.coord(j, q);
            bondlist[k] = (double)(i + 1);
            bondlist[k + nb] = (double)(j + 1);
            double e0 = p[0] - q[0], e1 = p[1] - q[1], e2 = p[2] - q[2];
            double ul = std::sqrt(e0 * e0 + e1 * e1 + e2 * e2);   // buildhorizons.m:93,97
            L0[k] = ul;
            double vcf;                                          // calculatevolumecorrectionfactors.m:23-33
            if (ul <= (d - R)) vcf = 1;
            else if ((ul > (d - R)) && (ul <= d)) vcf = (d + R - ul) / (2 * R);
            else vcf = 0;
            VCF[k] = vcf;
            double sf = (2 * VH) / (((double)fam[i] * V + (double)fam[j] * V));  // buildbonddata.m:193
            BS[k] = sf * c;                                                     // :194
            k++;
        }
    });

    // supports and prescribed DOFs
    std::memset(CF, 0, sizeof(double) * 3 * n);
    std::memset(PF, 0, sizeof(double) * 3 * n);
    double xmid = 0.5 * (spec->dx + spec->dx * spec->nx), tol = 0.5 * spec->dx * (1 + 1e-9);
    for (int64_t i = 0; i < n; i++) {
        double p[3];
        B.coord(i, p);
        int64_t cz = i / ((int64_t)B.L.nx * B.L.ny);
        for (int k = 0; k < spec->n_supports && k < 2; k++)
            if (cz == 0 && std::fabs(p[0] - spec->support_x[k]) <= tol) {
                CF[i] = CF[i + n] = CF[i + 2 * n] = 1;
                break;
            }
        if (spec->load_midspan_top && cz == B.L.nz - 1 && std::fabs(p[0] - xmid) <= tol)
            PF[i + 2 * n] = 1;
    }

    if (spec->sc_lognormal) {
        double cov = spec->sc_cov, s2 = std::log(1 + cov * cov);
        double mu = std::log(spec->sc_mean) - 0.5 * s2, sg = std::sqrt(s2);
        parallel_for(nb, [&](int64_t k) {
            uint64_t h1 = splitmix64(spec->seed ^ (0xA0761D6478BD642Full * (uint64_t)(2 * k + 1)));
            uint64_t h2 = splitmix64(h1 ^ 0xE7037ED1A0B428DBull);
            double u1 = ((double)(h1 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            double u2 = ((double)(h2 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            double z = std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2);
            sc[k] = std::exp(mu + sg * z);
        });
    }
    return BBPD_OK;
}
