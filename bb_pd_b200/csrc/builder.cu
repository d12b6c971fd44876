// Input builder on the GPU: the reference's input module for any point cloud.
//
//   buildhorizons.m:13-97        families and bond list (cell-list search)
//   buildnotch.m:13-119          bonds crossing the notch rectangle removed,
//   + determineintersection.m    families rebuilt from the reduced list
//   calculatevolumecorrectionfactors.m:16-34
//   buildbonddata.m:16-66        bond type, stiffness with surface correction
//   buildmassmatrix.m:32-40      ADR mass
//
// Horizons. The nodes are binned into a uniform grid whose cell edge is the
// horizon widened by 1e-6 (so rounding in the binning never puts two nodes
// within the horizon more than one cell apart) and sorted by cell with a radix
// sort. Every node scans the 27 cells around its own and keeps each j != i with
// sqrt(((xi-xj)^2 + (yi-yj)^2) + (zi-zj)^2) <= horizon: the expression of the
// reference's UNDEFORMEDLENGTH, so the test and the stored length agree bit for
// bit (the squared differences are the same both ways, so the relation is
// symmetric). A count pass sizes the families, a fill pass writes (i, j) keys,
// and a radix sort of the keys lists every family by ascending node id (the
// reference's rangesearch lists them by distance; both are valid families).
// Bonds are the pairs with j > i, by i then j.
//
// Notch. The rectangle's corners and unit normal are formed on the host
// exactly as determineintersection.m forms them; one thread per bond runs the
// segment test, a stable compaction keeps the other bonds in order, and the
// families are rebuilt in bond order by a stable sort of the directed entries
// by node (buildnotch.m:90-119 appends in bond order).
#include "bbpd_internal.h"
#include "staging.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

using namespace bbpd;

namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n)
{
    int64_t b = (n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 64));
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

inline int bits_for(int64_t n)   // smallest b with 2^b >= n, at least 1
{
    int b = 1;
    while (b < 62 && ((int64_t)1 << b) < n) b++;
    return b;
}

// Device buffers released in stream order when the builder call returns.
struct Scratch {
    cudaStream_t st;
    std::vector<void *> p;
    explicit Scratch(cudaStream_t s) : st(s) {}
    template <class T>
    int get(T **out, size_t count)
    {
        BBPD_CUDA_TRY(cudaMallocAsync((void **)out, sizeof(T) * std::max<size_t>(count, 1), st));
        p.push_back((void *)*out);
        return BBPD_OK;
    }
    ~Scratch()
    {
        for (void *q : p) cudaFreeAsync(q, st);
    }
};

#define TRY(x) do { int r_ = (x); if (r_) return r_; } while (0)

int launch_check()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return BBPD_OK;
}

__device__ __forceinline__ double pair_length(const double *__restrict__ X, int64_t n, int64_t i, int64_t j)
{
    const double e0 = X[i] - X[j], e1 = X[i + n] - X[j + n], e2 = X[i + 2 * n] - X[j + 2 * n];
    return sqrt(e0 * e0 + e1 * e1 + e2 * e2);
}

struct Grid {
    double lo[3];
    double h;
    int64_t nc[3];
};

__global__ void k_cell_of(const double *__restrict__ X, int64_t n, Grid g, uint32_t *cell, uint32_t *node)
{
    GRID_STRIDE(i, n)
    {
        int64_t c[3];
        for (int a = 0; a < 3; a++) {
            const double q = floor((X[i + a * n] - g.lo[a]) / g.h);
            c[a] = q >= 0 ? (q < (double)g.nc[a] ? (int64_t)q : g.nc[a] - 1) : 0;   // NaN -> cell 0
        }
        cell[i] = (uint32_t)(c[0] + g.nc[0] * (c[1] + g.nc[1] * c[2]));
        node[i] = (uint32_t)i;
    }
}

__global__ void k_cell_bounds(const uint32_t *__restrict__ scell, int64_t n, uint32_t *first, uint32_t *last)
{
    GRID_STRIDE(q, n)
    {
        const uint32_t c = scell[q];
        if (q == 0 || scell[q - 1] != c) first[c] = (uint32_t)q;
        if (q == n - 1 || scell[q + 1] != c) last[c] = (uint32_t)(q + 1);
    }
}

// FILL = false: family size and forward (j > i) count of every node.
// FILL = true: the (i, j) keys of every family, unordered within it.
template <bool FILL>
__global__ void k_horizon_scan(const double *__restrict__ X, int64_t n, double horizon, Grid g,
                               const uint32_t *__restrict__ scell, const uint32_t *__restrict__ snode,
                               const uint32_t *__restrict__ first, const uint32_t *__restrict__ last,
                               int32_t *fam, int32_t *fwd, const int64_t *__restrict__ famoff, int bits,
                               uint64_t *keys)
{
    GRID_STRIDE(q, n)
    {
        const int64_t i = snode[q];
        const int64_t c = scell[q];
        const int64_t cx = c % g.nc[0], cy = (c / g.nc[0]) % g.nc[1], cz = c / (g.nc[0] * g.nc[1]);
        int32_t nf = 0, nfw = 0;
        int64_t out = FILL ? famoff[i] : 0;
        const int64_t end = FILL ? famoff[i + 1] : 0;   // the count pass sized this family
        for (int64_t z = cz - 1; z <= cz + 1; z++) {
            if (z < 0 || z >= g.nc[2]) continue;
            for (int64_t y = cy - 1; y <= cy + 1; y++) {
                if (y < 0 || y >= g.nc[1]) continue;
                for (int64_t x = cx - 1; x <= cx + 1; x++) {
                    if (x < 0 || x >= g.nc[0]) continue;
                    const int64_t cc = x + g.nc[0] * (y + g.nc[1] * z);
                    const uint32_t a = first[cc], b = last[cc];
                    for (uint32_t r = a; r < b; r++) {
                        const int64_t j = snode[r];
                        if (j == i || !(pair_length(X, n, i, j) <= horizon)) continue;
                        if (FILL) {
                            if (out < end) keys[out++] = ((uint64_t)i << bits) | (uint64_t)j;
                        } else {
                            nf++;
                            nfw += j > i;
                        }
                    }
                }
            }
        }
        if (!FILL) {
            fam[i] = nf;
            fwd[i] = nfw;
        }
    }
}

// int32 counts to an (n + 1)-entry int64 array for an exclusive scan
__global__ void k_widen(const int32_t *__restrict__ c, int64_t n, int64_t *w)
{
    GRID_STRIDE(i, n + 1) w[i] = i < n ? (int64_t)c[i] : 0;
}

struct HorizonOut {
    double *nfam, *famptr, *family, *bl, *L0;   // any may be null
    int64_t nb;                                 // leading dimension of bl
};

// Sorted family keys to the reference's arrays.
__global__ void k_horizon_emit(const uint64_t *__restrict__ skeys, int64_t nf, int bits, const double *__restrict__ X,
                               int64_t n, const int64_t *__restrict__ famoff, const int64_t *__restrict__ boff,
                               const int32_t *__restrict__ fwd, HorizonOut o)
{
    const uint64_t mask = ((uint64_t)1 << bits) - 1;
    GRID_STRIDE(e, nf)
    {
        const uint64_t key = skeys[e];
        const int64_t i = (int64_t)(key >> bits), j = (int64_t)(key & mask);
        if (i >= n || j >= n) continue;
        if (o.family) o.family[e] = (double)(j + 1);
        if (j > i && o.bl) {
            const int64_t b = boff[i] + (e - (famoff[i + 1] - fwd[i]));
            if (b < boff[i] || b >= boff[i + 1]) continue;
            o.bl[b] = (double)(i + 1);
            o.bl[b + o.nb] = (double)(j + 1);
            o.L0[b] = pair_length(X, n, i, j);
        }
    }
}

__global__ void k_family_sizes(const int32_t *__restrict__ fam, const int64_t *__restrict__ famoff, int64_t n,
                               double *nfam, double *famptr)
{
    GRID_STRIDE(i, n)
    {
        if (nfam) nfam[i] = (double)fam[i];
        if (famptr) famptr[i] = (double)(famoff[i] + 1);
    }
}

// ---- notch ----

struct Notch {
    double A[3], B[3], D[3], nrm[3];
};

__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// determineintersection.m:59-86 with plane_line_intersect :126-150
__device__ bool notch_hit(const Notch &q, const double *P0, const double *P1)
{
    double AB[3], AD[3], u[3], w[3], I[3];
    for (int c = 0; c < 3; c++) {
        AB[c] = q.B[c] - q.A[c];
        AD[c] = q.D[c] - q.A[c];
        u[c] = P1[c] - P0[c];
        w[c] = P0[c] - q.A[c];
    }
    const double Dn = dot3(q.nrm, u), N = -dot3(q.nrm, w);
    if (fabs(Dn) < 1e-7) return false;   // parallel to the plane: no crossing counted
    const double sI = N / Dn;
    for (int c = 0; c < 3; c++) I[c] = P0[c] + (sI * u[c]);
    if (sI < 0 || sI > 1) return false;
    return (dot3(q.A, AB) <= dot3(I, AB)) && (dot3(I, AB) <= dot3(q.B, AB)) && (dot3(q.A, AD) <= dot3(I, AD)) &&
           (dot3(I, AD) <= dot3(q.D, AD));
}

__global__ void k_notch_keep(const double *__restrict__ X, int64_t n, const double *__restrict__ bl, int64_t nB,
                             Notch q, uint8_t *keep, int *bad)
{
    GRID_STRIDE(k, nB)
    {
        const double di = bl[k], dj = bl[nB + k];
        if (!(di >= 1 && dj >= 1 && di <= (double)n && dj <= (double)n)) {
            *bad = 1;
            keep[k] = 0;
            continue;
        }
        const int64_t i = (int64_t)di - 1, j = (int64_t)dj - 1;
        const double P0[3] = {X[i], X[i + n], X[i + 2 * n]}, P1[3] = {X[j], X[j + n], X[j + 2 * n]};
        keep[k] = notch_hit(q, P0, P1) ? 0 : 1;
    }
}

__global__ void k_iota32(uint32_t *v, int64_t n)
{
    GRID_STRIDE(i, n) v[i] = (uint32_t)i;
}

// kept rows to the output (leading dimension m), directed-entry keys for the
// family rebuild and the family counts
__global__ void k_notch_gather(const uint32_t *__restrict__ idx, int64_t m, const double *__restrict__ bl, int64_t nB,
                               const double *__restrict__ L0, double *blo, double *L0o, uint32_t *ekey,
                               int32_t *fam)
{
    GRID_STRIDE(r, m)
    {
        const int64_t k = idx[r];
        const double a = bl[k], b = bl[nB + k];
        blo[r] = a;
        blo[r + m] = b;
        L0o[r] = L0[k];
        ekey[2 * r] = (uint32_t)((int64_t)a - 1);
        ekey[2 * r + 1] = (uint32_t)((int64_t)b - 1);
        atomicAdd(&fam[(int64_t)a - 1], 1);
        atomicAdd(&fam[(int64_t)b - 1], 1);
    }
}

// NODEFAMILY in bond order: entry q = 2r + side sorted stably by its node;
// the family member is the other end of bond r
__global__ void k_notch_family(const uint32_t *__restrict__ ekey, const uint32_t *__restrict__ sval, int64_t ne,
                               double *family)
{
    GRID_STRIDE(e, ne) family[e] = (double)ekey[sval[e] ^ 1u] + 1.0;
}

// ---- per-bond and per-node tables ----

// calculatevolumecorrectionfactors.m:23-33
__global__ void k_volumecorrection(const double *__restrict__ L0, int64_t nB, double horizon, double radij, double *VCF)
{
    GRID_STRIDE(k, nB)
    {
        const double UL = L0[k];
        double v;
        if (UL <= (horizon - radij)) v = 1;
        else if ((UL > (horizon - radij)) && (UL <= horizon)) v = (horizon + radij - UL) / (2 * radij);
        else v = 0;
        VCF[k] = v;
    }
}

// buildbonddata.m:27-71
__global__ void k_bonddata(const double *__restrict__ bl, int64_t nB, int64_t n, const double *__restrict__ nfam,
                           const double *__restrict__ mat, double bsc, double bss, double V, double VH, double *BS,
                           double *BT, double *BFM, double *SF, int *bad)
{
    GRID_STRIDE(k, nB)
    {
        const double di = bl[k], dj = bl[nB + k];
        if (!(di >= 1 && dj >= 1 && di <= (double)n && dj <= (double)n)) {
            *bad = 1;
            continue;
        }
        const int64_t i = (int64_t)di - 1, j = (int64_t)dj - 1;
        const double mi = mat ? mat[i] : 0.0, mj = mat ? mat[j] : 0.0;
        double bst, bt;
        if (mi == 0 && mj == 0) { bst = bsc; bt = 0; }
        else if (mi == 0 && mj == 1) { bst = bsc; bt = 1; }
        else if (mi == 1 && mj == 0) { bst = bsc; bt = 1; }
        else if (mi == 1 && mj == 1) { bst = bss; bt = 2; }
        else {
            *bad = 2;
            continue;
        }
        const double sf = (2 * VH) / ((nfam[i] * V + nfam[j] * V));
        if (SF) SF[k] = sf;
        BS[k] = sf * bst;
        if (BT) BT[k] = bt;
        if (BFM) BFM[k] = bt == 1 ? 3 : 1;
    }
}

// buildmassmatrix.m:36-38
__global__ void k_massmatrix(const double *__restrict__ nfam, int64_t n, double dx, double bsc, double dt, double *mass)
{
    GRID_STRIDE(i, n)
    {
        const double Kij = (nfam[i] * (dx * dx)) * (bsc / dx);
        mass[i] = 0.25 * (dt * dt) * Kij;
    }
}

__global__ void k_nonfinite(const double *__restrict__ X, int64_t n, int *bad)
{
    GRID_STRIDE(i, n)
    if (!isfinite(X[i])) *bad = 1;
}

// min and max of every coordinate column: six values to the host; fails on a
// coordinate that is not finite
int coord_bounds(const double *X, int64_t n, cudaStream_t st, double lo[3], double hi[3])
{
    Scratch s(st);
    double *out = nullptr;
    int *bad = nullptr;
    TRY(s.get(&out, 6));
    TRY(s.get(&bad, 1));
    BBPD_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    k_nonfinite<<<blocks_for(3 * n), kThreads, 0, st>>>(X, 3 * n, bad);
    TRY(launch_check());
    size_t tb = 0, tmax = 0;
    for (int a = 0; a < 3; a++) {
        BBPD_CUDA_TRY(cub::DeviceReduce::Min(nullptr, tb, X + a * n, out + a, n, st));
        tmax = std::max(tmax, tb);
        BBPD_CUDA_TRY(cub::DeviceReduce::Max(nullptr, tb, X + a * n, out + 3 + a, n, st));
        tmax = std::max(tmax, tb);
    }
    uint8_t *tmp = nullptr;
    TRY(s.get(&tmp, tmax));
    for (int a = 0; a < 3; a++) {
        tb = tmax;
        BBPD_CUDA_TRY(cub::DeviceReduce::Min(tmp, tb, X + a * n, out + a, n, st));
        tb = tmax;
        BBPD_CUDA_TRY(cub::DeviceReduce::Max(tmp, tb, X + a * n, out + 3 + a, n, st));
    }
    double h[6];
    int hb = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    if (hb) return fail(BBPD_ERR_ARG, "coordinates must be finite");
    for (int a = 0; a < 3; a++) {
        lo[a] = h[a];
        hi[a] = h[3 + a];
    }
    return BBPD_OK;
}

}  // namespace

namespace {

// The horizon search in two phases: count() bins, sorts and counts;
// emit() lists the families and bonds once the caller has room for them.
struct Horizons {
    cudaStream_t st;
    Scratch s;
    const double *X = nullptr;
    int64_t n = 0, nb = 0, nf = 0;
    double horizon = 0;
    int bits = 1;
    Grid g{};
    uint32_t *scell = nullptr, *snode = nullptr, *first = nullptr, *last = nullptr;
    int32_t *fam = nullptr, *fwd = nullptr;
    int64_t *famoff = nullptr, *boff = nullptr;
    explicit Horizons(cudaStream_t s_) : st(s_), s(s_) {}

    int count(const double *X_, int64_t n_, double r)
    {
        X = X_;
        n = n_;
        horizon = r;
        bits = bits_for(n);
        double lo[3], hi[3];
        TRY(coord_bounds(X, n, st, lo, hi));
        for (int a = 0; a < 3; a++)
            if (!std::isfinite(hi[a] - lo[a])) return fail(BBPD_ERR_ARG, "coordinate range too large");
        // cells of edge >= horizon (1e-6 wider), at most 2^26 of them
        g.h = r * (1 + 1e-6);
        for (;;) {
            double cells = 1;
            for (int a = 0; a < 3; a++) {
                g.lo[a] = lo[a];
                g.nc[a] = (int64_t)std::floor((hi[a] - lo[a]) / g.h) + 1;
                cells *= (double)g.nc[a];
            }
            if (cells <= (double)(1 << 26)) break;
            g.h *= 1.25;
        }
        const int64_t ncell = g.nc[0] * g.nc[1] * g.nc[2];
        uint32_t *cell = nullptr, *node = nullptr;
        TRY(s.get(&cell, n));
        TRY(s.get(&node, n));
        TRY(s.get(&scell, n));
        TRY(s.get(&snode, n));
        k_cell_of<<<blocks_for(n), kThreads, 0, st>>>(X, n, g, cell, node);
        TRY(launch_check());
        size_t tb = 0;
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, cell, scell, node, snode, n, 0, bits_for(ncell), st));
        uint8_t *tmp = nullptr;
        TRY(s.get(&tmp, tb));
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, cell, scell, node, snode, n, 0, bits_for(ncell), st));
        TRY(s.get(&first, ncell));
        TRY(s.get(&last, ncell));
        BBPD_CUDA_TRY(cudaMemsetAsync(first, 0, sizeof(uint32_t) * ncell, st));
        BBPD_CUDA_TRY(cudaMemsetAsync(last, 0, sizeof(uint32_t) * ncell, st));
        k_cell_bounds<<<blocks_for(n), kThreads, 0, st>>>(scell, n, first, last);
        TRY(launch_check());
        TRY(s.get(&fam, n));
        TRY(s.get(&fwd, n));
        k_horizon_scan<false><<<blocks_for(n), kThreads, 0, st>>>(X, n, r, g, scell, snode, first, last, fam, fwd,
                                                                  nullptr, bits, nullptr);
        TRY(launch_check());
        int64_t *w = nullptr;
        TRY(s.get(&w, n + 1));
        TRY(s.get(&famoff, n + 1));
        TRY(s.get(&boff, n + 1));
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, w, famoff, n + 1, st));
        uint8_t *stmp = nullptr;
        TRY(s.get(&stmp, tb));
        k_widen<<<blocks_for(n + 1), kThreads, 0, st>>>(fam, n, w);
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(stmp, tb, w, famoff, n + 1, st));
        k_widen<<<blocks_for(n + 1), kThreads, 0, st>>>(fwd, n, w);
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(stmp, tb, w, boff, n + 1, st));
        TRY(launch_check());
        BBPD_CUDA_TRY(cudaMemcpyAsync(&nf, famoff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        BBPD_CUDA_TRY(cudaMemcpyAsync(&nb, boff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        BBPD_CUDA_TRY(cudaStreamSynchronize(st));
        if (nf != 2 * nb) return fail(BBPD_ERR_CUDA, "horizon search: %lld family entries for %lld bonds",
                                      (long long)nf, (long long)nb);
        return BBPD_OK;
    }

    int sizes(double *nfam, double *famptr)
    {
        if (!nfam && !famptr) return BBPD_OK;
        k_family_sizes<<<blocks_for(n), kThreads, 0, st>>>(fam, famoff, n, nfam, famptr);
        return launch_check();
    }

    int emit(HorizonOut o)
    {
        if (nf == 0 || (!o.family && !o.bl)) return BBPD_OK;
        uint64_t *keys = nullptr, *skeys = nullptr;
        TRY(s.get(&keys, nf));
        TRY(s.get(&skeys, nf));
        k_horizon_scan<true><<<blocks_for(n), kThreads, 0, st>>>(X, n, horizon, g, scell, snode, first, last, fam,
                                                                 fwd, famoff, bits, keys);
        TRY(launch_check());
        size_t tb = 0;
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, skeys, nf, 0, 2 * bits, st));
        uint8_t *tmp = nullptr;
        TRY(s.get(&tmp, tb));
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, skeys, nf, 0, 2 * bits, st));
        o.nb = nb;
        k_horizon_emit<<<blocks_for(nf), kThreads, 0, st>>>(skeys, nf, bits, X, n, famoff, boff, fwd, o);
        return launch_check();
    }
};

// A stream of its own for each host-pointer call, destroyed on return.
struct CallStream {
    cudaStream_t st = nullptr;
    ~CallStream()
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
};

int check_horizon_args(const double *X, int64_t n, double r)
{
    if (!X && n > 0) return fail(BBPD_ERR_ARG, "null coordinates");
    if (n < 0 || n >= ((int64_t)1 << 31)) return fail(BBPD_ERR_ARG, "nNodes must be in [0, 2^31)");
    if (!(r > 0) || !std::isfinite(r)) return fail(BBPD_ERR_ARG, "horizon must be positive and finite");
    return BBPD_OK;
}

}  // namespace

extern "C" int bbpd_dev_buildhorizons(const double *X, int64_t nNodes, double horizon, int64_t capacity,
        int64_t *nBonds, double *nFAMILYMEMBERS, double *NODEFAMILYPOINTERS, double *NODEFAMILY,
        double *BONDLIST, double *UNDEFORMEDLENGTH, void *stream)
{
    if (!nBonds) return fail(BBPD_ERR_ARG, "null nBonds");
    TRY(check_horizon_args(X, nNodes, horizon));
    *nBonds = 0;
    if (nNodes == 0) return BBPD_OK;
    TRY(require_device());
    Horizons h(as_stream(stream));
    TRY(h.count(X, nNodes, horizon));
    *nBonds = h.nb;
    TRY(h.sizes(nFAMILYMEMBERS, NODEFAMILYPOINTERS));
    if (capacity >= h.nb) {
        if (BONDLIST && !UNDEFORMEDLENGTH) return fail(BBPD_ERR_ARG, "BONDLIST needs UNDEFORMEDLENGTH");
        TRY(h.emit(HorizonOut{nullptr, nullptr, NODEFAMILY, BONDLIST, UNDEFORMEDLENGTH, 0}));
    }
    BBPD_CUDA_TRY(cudaStreamSynchronize(h.st));
    return BBPD_OK;
}

extern "C" int bbpd_buildhorizons(const double *X, int64_t nNodes, double horizon, int64_t capacity,
        int64_t *nBonds, double *nFAMILYMEMBERS, double *NODEFAMILYPOINTERS, double *NODEFAMILY,
        double *BONDLIST, double *UNDEFORMEDLENGTH)
{
    if (!nBonds) return fail(BBPD_ERR_ARG, "null nBonds");
    TRY(check_horizon_args(X, nNodes, horizon));
    *nBonds = 0;
    if (nNodes == 0) return BBPD_OK;
    TRY(require_device());
    CallStream cs;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
    Horizons h(cs.st);
    double *dX = nullptr;
    TRY(h.s.get(&dX, 3 * nNodes));
    TRY(staging::upload_copy(dX, X, 3 * nNodes, cs.st));
    TRY(h.count(dX, nNodes, horizon));
    const int64_t nb = h.nb;
    *nBonds = nb;
    double *dnf = nullptr, *dfp = nullptr;
    if (nFAMILYMEMBERS) TRY(h.s.get(&dnf, nNodes));
    if (NODEFAMILYPOINTERS) TRY(h.s.get(&dfp, nNodes));
    TRY(h.sizes(dnf, dfp));
    HorizonOut o{nullptr, nullptr, nullptr, nullptr, nullptr, 0};
    const bool lists = capacity >= nb && nb > 0;
    if (lists && NODEFAMILY) TRY(h.s.get(&o.family, 2 * nb));
    if (lists && (BONDLIST || UNDEFORMEDLENGTH)) {
        TRY(h.s.get(&o.bl, 2 * nb));
        TRY(h.s.get(&o.L0, nb));
    }
    TRY(h.emit(o));
    if (dnf) TRY(staging::download_copy(nFAMILYMEMBERS, dnf, nNodes, cs.st));
    if (dfp) TRY(staging::download_copy(NODEFAMILYPOINTERS, dfp, nNodes, cs.st));
    if (o.family) TRY(staging::download_copy(NODEFAMILY, o.family, 2 * nb, cs.st));
    if (o.bl && BONDLIST) TRY(staging::download_copy(BONDLIST, o.bl, 2 * nb, cs.st));
    if (o.L0 && UNDEFORMEDLENGTH) TRY(staging::download_copy(UNDEFORMEDLENGTH, o.L0, nb, cs.st));
    return BBPD_OK;
}

namespace {

// buildnotch.m on device arrays; outputs may be null except nOut.
int notch_dev(const double *X, int64_t n, const double *bl, const double *L0, int64_t nB, double DX,
              double xlocation, double depth, int64_t *nOut, double *blo, double *L0o, double *nfam,
              double *famptr, double *family, cudaStream_t st, Scratch &s)
{
    double lo[3], hi[3];
    TRY(coord_bounds(X, n, st, lo, hi));
    // buildnotch.m:52-55 corners, determineintersection.m:59-68 normal
    Notch q;
    const double xl = xlocation * DX;
    const double A[3] = {xl, lo[1], lo[2]}, B[3] = {xl, hi[1], lo[2]}, D[3] = {xl, lo[1], depth * DX};
    double AB[3], AD[3];
    for (int c = 0; c < 3; c++) {
        q.A[c] = A[c];
        q.B[c] = B[c];
        q.D[c] = D[c];
        AB[c] = B[c] - A[c];
        AD[c] = D[c] - A[c];
    }
    const double cr[3] = {AB[1] * AD[2] - AB[2] * AD[1], AB[2] * AD[0] - AB[0] * AD[2], AB[0] * AD[1] - AB[1] * AD[0]};
    const double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int c = 0; c < 3; c++) q.nrm[c] = cr[c] / len;

    uint8_t *keep = nullptr;
    uint32_t *iota = nullptr, *idx = nullptr;
    int *bad = nullptr;
    int64_t *dm = nullptr;
    TRY(s.get(&keep, nB));
    TRY(s.get(&iota, nB));
    TRY(s.get(&idx, nB));
    TRY(s.get(&bad, 1));
    TRY(s.get(&dm, 1));
    BBPD_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    BBPD_CUDA_TRY(cudaMemsetAsync(dm, 0, sizeof(int64_t), st));
    size_t tb = 0;
    uint8_t *tmp = nullptr;
    if (nB > 0) {
        k_notch_keep<<<blocks_for(nB), kThreads, 0, st>>>(X, n, bl, nB, q, keep, bad);
        k_iota32<<<blocks_for(nB), kThreads, 0, st>>>(iota, nB);
        TRY(launch_check());
        BBPD_CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, tb, iota, keep, idx, dm, (int)nB, st));
        TRY(s.get(&tmp, tb));
        BBPD_CUDA_TRY(cub::DeviceSelect::Flagged(tmp, tb, iota, keep, idx, dm, (int)nB, st));
    }
    int64_t m = 0;
    int hbad = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(&m, dm, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    if (hbad) return fail(BBPD_ERR_ARG, "BONDLIST holds node ids outside [1, nNodes]");
    *nOut = m;

    double *bo = blo, *lo2 = L0o;
    if (!bo) TRY(s.get(&bo, 2 * m));
    if (!lo2) TRY(s.get(&lo2, m));
    uint32_t *ekey = nullptr;
    int32_t *fam = nullptr;
    TRY(s.get(&ekey, 2 * m));
    TRY(s.get(&fam, n));
    BBPD_CUDA_TRY(cudaMemsetAsync(fam, 0, sizeof(int32_t) * n, st));
    if (m > 0) {
        k_notch_gather<<<blocks_for(m), kThreads, 0, st>>>(idx, m, bl, nB, L0, bo, lo2, ekey, fam);
        TRY(launch_check());
    }
    int64_t *w = nullptr, *famoff = nullptr;
    TRY(s.get(&w, n + 1));
    TRY(s.get(&famoff, n + 1));
    k_widen<<<blocks_for(n + 1), kThreads, 0, st>>>(fam, n, w);
    BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, w, famoff, n + 1, st));
    TRY(s.get(&tmp, tb));
    BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tb, w, famoff, n + 1, st));
    if (nfam || famptr) {
        k_family_sizes<<<blocks_for(n), kThreads, 0, st>>>(fam, famoff, n, nfam, famptr);
        TRY(launch_check());
    }
    if (family && m > 0) {
        uint32_t *val = nullptr, *skey = nullptr, *sval = nullptr;
        TRY(s.get(&val, 2 * m));
        TRY(s.get(&skey, 2 * m));
        TRY(s.get(&sval, 2 * m));
        k_iota32<<<blocks_for(2 * m), kThreads, 0, st>>>(val, 2 * m);
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, ekey, skey, val, sval, 2 * m, 0, bits_for(n), st));
        TRY(s.get(&tmp, tb));
        BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, ekey, skey, val, sval, 2 * m, 0, bits_for(n), st));
        k_notch_family<<<blocks_for(2 * m), kThreads, 0, st>>>(ekey, sval, 2 * m, family);
        TRY(launch_check());
    }
    return BBPD_OK;
}

int check_notch_args(const double *X, int64_t n, const double *bl, const double *L0, int64_t nB, int64_t *nOut)
{
    if (!nOut) return fail(BBPD_ERR_ARG, "null nBondsOut");
    if ((!X && n > 0) || (nB > 0 && (!bl || !L0))) return fail(BBPD_ERR_ARG, "null input array");
    if (n < 1 || n >= ((int64_t)1 << 31) || nB < 0 || nB >= ((int64_t)1 << 31))
        return fail(BBPD_ERR_ARG, "need 1 <= nNodes < 2^31 and 0 <= nBonds < 2^31");
    return BBPD_OK;
}

}  // namespace

extern "C" int bbpd_dev_buildnotch(const double *X, int64_t nNodes, const double *BONDLIST,
        const double *UNDEFORMEDLENGTH, int64_t nBonds, double DX, double xlocation, double depth,
        int64_t *nBondsOut, double *BONDLISTout, double *UNDEFORMEDLENGTHout, double *nFAMILYMEMBERS,
        double *NODEFAMILYPOINTERS, double *NODEFAMILY, void *stream)
{
    TRY(check_notch_args(X, nNodes, BONDLIST, UNDEFORMEDLENGTH, nBonds, nBondsOut));
    TRY(require_device());
    cudaStream_t st = as_stream(stream);
    Scratch s(st);
    TRY(notch_dev(X, nNodes, BONDLIST, UNDEFORMEDLENGTH, nBonds, DX, xlocation, depth, nBondsOut, BONDLISTout,
                  UNDEFORMEDLENGTHout, nFAMILYMEMBERS, NODEFAMILYPOINTERS, NODEFAMILY, st, s));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    return BBPD_OK;
}

extern "C" int bbpd_buildnotch(const double *X, int64_t nNodes, const double *BONDLIST,
        const double *UNDEFORMEDLENGTH, int64_t nBonds, double DX, double xlocation, double depth,
        int64_t *nBondsOut, double *BONDLISTout, double *UNDEFORMEDLENGTHout, double *nFAMILYMEMBERS,
        double *NODEFAMILYPOINTERS, double *NODEFAMILY)
{
    TRY(check_notch_args(X, nNodes, BONDLIST, UNDEFORMEDLENGTH, nBonds, nBondsOut));
    TRY(require_device());
    CallStream cs;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
    Scratch s(cs.st);
    double *dX = nullptr, *dbl = nullptr, *dL = nullptr, *dbo = nullptr, *dLo = nullptr;
    double *dnf = nullptr, *dfp = nullptr, *dfam = nullptr;
    TRY(s.get(&dX, 3 * nNodes));
    TRY(s.get(&dbl, 2 * nBonds));
    TRY(s.get(&dL, nBonds));
    TRY(staging::upload_copy(dX, X, 3 * nNodes, cs.st));
    TRY(staging::upload_copy(dbl, BONDLIST, 2 * nBonds, cs.st));
    TRY(staging::upload_copy(dL, UNDEFORMEDLENGTH, nBonds, cs.st));
    TRY(s.get(&dbo, 2 * nBonds));
    TRY(s.get(&dLo, nBonds));
    if (nFAMILYMEMBERS) TRY(s.get(&dnf, nNodes));
    if (NODEFAMILYPOINTERS) TRY(s.get(&dfp, nNodes));
    if (NODEFAMILY) TRY(s.get(&dfam, 2 * nBonds));
    TRY(notch_dev(dX, nNodes, dbl, dL, nBonds, DX, xlocation, depth, nBondsOut, dbo, dLo, dnf, dfp, dfam, cs.st, s));
    const int64_t m = *nBondsOut;
    if (BONDLISTout) TRY(staging::download_copy(BONDLISTout, dbo, 2 * m, cs.st));
    if (UNDEFORMEDLENGTHout) TRY(staging::download_copy(UNDEFORMEDLENGTHout, dLo, m, cs.st));
    if (dnf) TRY(staging::download_copy(nFAMILYMEMBERS, dnf, nNodes, cs.st));
    if (dfp) TRY(staging::download_copy(NODEFAMILYPOINTERS, dfp, nNodes, cs.st));
    if (dfam) TRY(staging::download_copy(NODEFAMILY, dfam, 2 * m, cs.st));
    return BBPD_OK;
}

// ---- per-bond and per-node tables ----

extern "C" int bbpd_dev_calculatevolumecorrectionfactors(const double *UNDEFORMEDLENGTH, int64_t nBonds,
        double horizon, double RADIJ, double *VOLUMECORRECTIONFACTORS, void *stream)
{
    if (nBonds < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nBonds == 0) return BBPD_OK;
    TRY(require_device());
    k_volumecorrection<<<blocks_for(nBonds), kThreads, 0, as_stream(stream)>>>(UNDEFORMEDLENGTH, nBonds, horizon,
                                                                                 RADIJ, VOLUMECORRECTIONFACTORS);
    return launch_check();
}

extern "C" int bbpd_dev_buildbonddata(const double *BONDLIST, int64_t nBonds, int64_t nNodes,
        const double *nFAMILYMEMBERS, const double *MATERIALFLAG, double bondStiffnessConcrete,
        double bondStiffnessSteel, double cellVolume, double neighbourhoodVolume, double *BONDSTIFFNESS,
        double *BONDTYPE, double *BFMULTIPLIER, double *stiffeningFactor, void *stream)
{
    if (nBonds < 0 || nNodes < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nBonds == 0) return BBPD_OK;
    TRY(require_device());
    cudaStream_t st = as_stream(stream);
    Scratch s(st);
    int *bad = nullptr;
    TRY(s.get(&bad, 1));
    BBPD_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    k_bonddata<<<blocks_for(nBonds), kThreads, 0, st>>>(BONDLIST, nBonds, nNodes, nFAMILYMEMBERS, MATERIALFLAG,
                                                          bondStiffnessConcrete, bondStiffnessSteel, cellVolume,
                                                          neighbourhoodVolume, BONDSTIFFNESS, BONDTYPE, BFMULTIPLIER,
                                                          stiffeningFactor, bad);
    TRY(launch_check());
    int h = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    if (h == 1) return fail(BBPD_ERR_ARG, "BONDLIST holds node ids outside [1, nNodes]");
    if (h == 2) return fail(BBPD_ERR_ARG, "MATERIALFLAG values must be 0 or 1");
    return BBPD_OK;
}

extern "C" int bbpd_dev_buildmassmatrix(int64_t nNodes, double DX, double bondStiffnessConcrete, double DT,
        const double *nFAMILYMEMBERS, double *massVector, void *stream)
{
    if (nNodes < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nNodes == 0) return BBPD_OK;
    TRY(require_device());
    k_massmatrix<<<blocks_for(nNodes), kThreads, 0, as_stream(stream)>>>(nFAMILYMEMBERS, nNodes, DX,
                                                                           bondStiffnessConcrete, DT, massVector);
    return launch_check();
}

extern "C" int bbpd_calculatevolumecorrectionfactors(const double *UNDEFORMEDLENGTH, int64_t nBonds,
        double horizon, double RADIJ, double *VOLUMECORRECTIONFACTORS)
{
    if (nBonds < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nBonds == 0) return BBPD_OK;
    if (!UNDEFORMEDLENGTH || !VOLUMECORRECTIONFACTORS) return fail(BBPD_ERR_ARG, "null array");
    TRY(require_device());
    CallStream cs;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
    Scratch s(cs.st);
    double *dL = nullptr, *dV = nullptr;
    TRY(s.get(&dL, nBonds));
    TRY(s.get(&dV, nBonds));
    TRY(staging::upload_copy(dL, UNDEFORMEDLENGTH, nBonds, cs.st));
    TRY(bbpd_dev_calculatevolumecorrectionfactors(dL, nBonds, horizon, RADIJ, dV, cs.st));
    return staging::download_copy(VOLUMECORRECTIONFACTORS, dV, nBonds, cs.st);
}

extern "C" int bbpd_buildbonddata(const double *BONDLIST, int64_t nBonds, int64_t nNodes,
        const double *nFAMILYMEMBERS, const double *MATERIALFLAG, double bondStiffnessConcrete,
        double bondStiffnessSteel, double cellVolume, double neighbourhoodVolume, double *BONDSTIFFNESS,
        double *BONDTYPE, double *BFMULTIPLIER, double *stiffeningFactor)
{
    if (nBonds < 0 || nNodes < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nBonds == 0) return BBPD_OK;
    if (!BONDLIST || !nFAMILYMEMBERS || !BONDSTIFFNESS) return fail(BBPD_ERR_ARG, "null array");
    TRY(require_device());
    CallStream cs;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
    Scratch s(cs.st);
    double *dbl = nullptr, *dnf = nullptr, *dmat = nullptr, *dBS = nullptr, *dBT = nullptr, *dBF = nullptr,
           *dSF = nullptr;
    TRY(s.get(&dbl, 2 * nBonds));
    TRY(s.get(&dnf, nNodes));
    TRY(staging::upload_copy(dbl, BONDLIST, 2 * nBonds, cs.st));
    TRY(staging::upload_copy(dnf, nFAMILYMEMBERS, nNodes, cs.st));
    if (MATERIALFLAG) {
        TRY(s.get(&dmat, nNodes));
        TRY(staging::upload_copy(dmat, MATERIALFLAG, nNodes, cs.st));
    }
    TRY(s.get(&dBS, nBonds));
    if (BONDTYPE) TRY(s.get(&dBT, nBonds));
    if (BFMULTIPLIER) TRY(s.get(&dBF, nBonds));
    if (stiffeningFactor) TRY(s.get(&dSF, nBonds));
    TRY(bbpd_dev_buildbonddata(dbl, nBonds, nNodes, dnf, dmat, bondStiffnessConcrete, bondStiffnessSteel, cellVolume,
                               neighbourhoodVolume, dBS, dBT, dBF, dSF, cs.st));
    TRY(staging::download_copy(BONDSTIFFNESS, dBS, nBonds, cs.st));
    if (dBT) TRY(staging::download_copy(BONDTYPE, dBT, nBonds, cs.st));
    if (dBF) TRY(staging::download_copy(BFMULTIPLIER, dBF, nBonds, cs.st));
    if (dSF) TRY(staging::download_copy(stiffeningFactor, dSF, nBonds, cs.st));
    return BBPD_OK;
}

extern "C" int bbpd_buildmassmatrix(int64_t nNodes, double DX, double bondStiffnessConcrete, double DT,
        const double *nFAMILYMEMBERS, double *massVector)
{
    if (nNodes < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nNodes == 0) return BBPD_OK;
    if (!nFAMILYMEMBERS || !massVector) return fail(BBPD_ERR_ARG, "null array");
    TRY(require_device());
    CallStream cs;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
    Scratch s(cs.st);
    double *dnf = nullptr, *dm = nullptr;
    TRY(s.get(&dnf, nNodes));
    TRY(s.get(&dm, nNodes));
    TRY(staging::upload_copy(dnf, nFAMILYMEMBERS, nNodes, cs.st));
    TRY(bbpd_dev_buildmassmatrix(nNodes, DX, bondStiffnessConcrete, DT, dnf, dm, cs.st));
    return staging::download_copy(massVector, dm, nNodes, cs.st);
}
