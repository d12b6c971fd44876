// Static (implicit) solver on the GPU: displacement-controlled Newton-Raphson
// after solvers/scripts/static/newtonraphsondisplacementcontrolled.m, with the
// tangent of buildstiffnessmatrixCSCformat.m solved matrix-free by a
// block-Jacobi preconditioned conjugate gradient over the free DOFs.
//
// One load step: the prescribed DOFs move by the increment, then each Newton
// iteration
//   1. updates every bond from the current positions (calculatedeformedlength,
//      the softening law, calculatebondfailure with the law's sc) and forms the
//      bond forces of calculatebondforces.m (BFMULTIPLIER included, unlike the
//      MEX) and their serial nodal sum in bond order (calculatenodalforces.m),
//      times cellVolume as the driver does (:111);
//   2. stops when the out-of-balance force on the free DOFs is at most `tol`
//      times the force on the held DOFs (the reference compares with 0.5 % of
//      the net internal force, checkconvergencecriteria.m:21-29);
//   3. solves K delta = F on the free DOFs, K the sum over intact bonds of
//      rig [c c^T, -c c^T; -c c^T, c c^T] with rig = BFM (BS / L^3) VCF V^2
//      (1 - BSF) at the current bond vector c (buildstiffnessmatrixCSCformat.m
//      NOD = 3 branch), and moves the free nodes by delta.
// The reference solves with MATLAB's bicgstabl and lsqr and applies its own
// corrector conventions; here every linear solve is a PCG to a relative
// residual of cg_tol, so results agree with a direct solve of the same
// equations to that tolerance.
//
// Layout: per bond its end nodes, constants and state; per node the list of
// its bond ends in bond order (a stable radix sort of the directed entries by
// node), which gives the nodal sums their serial order and the matrix-free
// products their neighbours. Reductions are two-level and fixed-order, so a
// step is deterministic.
#include "bbpd_internal.h"
#include "physics.cuh"
#include "staging.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

using namespace bbpd;

namespace {

constexpr int kThreads = 256;
constexpr int kRedBlocks = 592;   // partial-sum blocks of the dot products (4 per SM)

inline int blocks_for(int64_t n)
{
    int64_t b = (n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 64));
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

#define TRY(x) do { int r_ = (x); if (r_) return r_; } while (0)

int launch_check()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return BBPD_OK;
}

struct SBonds {
    const uint32_t *a, *b;      // end nodes (0-based)
    const double *L0, *BS, *VCF, *BFM;
    const uint8_t *BT;
    double *fail, *bsf;
    uint8_t *flag;
    double *rig;                // tangent scale, 0 for failed bonds
    double *c;                  // current bond vector x_b - x_a, [3 nB]
    double *f;                  // bond force, [3 nB]
    int64_t nB;
    int law;
    LawScalars P;
    double V;
};

// calculatedeformedlength + law + calculatebondfailure + calculatebondforces.m
// and the stiffness scale of buildstiffnessmatrixCSCformat.m for every bond
__global__ void k_static_bonds(SBonds s, const double *__restrict__ x, int64_t n)
{
    GRID_STRIDE(k, s.nB)
    {
        const int64_t i = s.a[k], j = s.b[k];
        double dX, dY, dZ, L, st;
        bond_kinematics(x[i], x[i + n], x[i + 2 * n], x[j], x[j + n], x[j + 2 * n], s.L0[k], dX, dY, dZ, L, st);
        double B = s.bsf[k], fl = s.fail[k];
        bool soft = s.flag[k] != 0;
        const int bt = s.BT[k];
        if (s.law == BBPD_LAW_BILINEAR) {
            double f = soft ? 1.0 : 0.0;
            if (bt == 0 && st > s.P.s0) f = 1;
            const double bs = ((st - s.P.s0) / st) * (s.P.sc / (s.P.sc - s.P.s0));
            B = matlab_max(B, bs * f);
            if (B > 1) B = 1;
            if (isnan(B)) B = 0;
            soft = f != 0;
        } else if (s.law == BBPD_LAW_TRILINEAR) {
            law_trilinear(st, s.P.s0, s.P.s1, s.P.sc, s.P, false, bt == 0, B, soft);
        } else if (s.law == BBPD_LAW_EXPONENTIAL) {
            law_exponential(st, s.P.s0, s.P.sc, s.P, bt == 0, B, soft);
        }
        law_linear(st, s.P.sc, s.P, bt, fl);
        s.bsf[k] = B;
        s.fail[k] = fl;
        s.flag[k] = soft ? 1 : 0;
        const double t = s.BFM[k] * fl * s.BS[k] * (1 - B) * st * s.V * s.VCF[k];
        const double d[3] = {dX, dY, dZ};
        for (int c = 0; c < 3; c++) {
            double f = t * (d[c] / L);
            if (f != f) f = 0.0;
            s.f[k + c * s.nB] = f;
            s.c[k + c * s.nB] = d[c];
        }
        // rig = BFM * ((BS / L^3) * VCF * V^2) * (1 - BSF) for intact bonds
        const double r = fl == 1 ? s.BFM[k] * ((s.BS[k] / (L * L * L)) * s.VCF[k] * (s.V * s.V)) * (1 - B) : 0.0;
        s.rig[k] = isfinite(r) ? r : 0.0;
    }
}

struct SNodes {
    const int64_t *off;         // [n + 1] list offsets
    const uint32_t *ent;        // directed entries q = 2k + side, by node, in bond order
    const uint8_t *held;        // per DOF [3 n]: 1 support, 2 prescribed
    int64_t n, nB;
};

// calculatenodalforces.m:25-35 in its serial order (node i gets +f of the bonds
// it starts, -f of those it ends), times cellVolume (driver :111); the residual
// norms of the free and held DOFs go to per-block partial sums.
__global__ void k_static_nodal(SNodes g, const double *__restrict__ f, double V, double *F, double *part)
{
    __shared__ double sh[2][kThreads / 32];
    double rf = 0, rh = 0;
    GRID_STRIDE(i, g.n)
    {
        double a[3] = {0, 0, 0};
        for (int64_t e = g.off[i]; e < g.off[i + 1]; e++) {
            const uint32_t q = g.ent[e];
            const int64_t k = q >> 1;
            for (int c = 0; c < 3; c++) {
                const double v = f[k + c * g.nB];
                a[c] = (q & 1u) ? a[c] - v : a[c] + v;
            }
        }
        for (int c = 0; c < 3; c++) {
            const double v = a[c] * V;
            F[i + c * g.n] = v;
            if (g.held[i + c * g.n]) rh += v * v;
            else rf += v * v;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        rf += __shfl_xor_sync(0xffffffffu, rf, o);
        rh += __shfl_xor_sync(0xffffffffu, rh, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = rf;
        sh[1][threadIdx.x >> 5] = rh;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            s0 += sh[0][w];
            s1 += sh[1][w];
        }
        part[2 * blockIdx.x] = s0;
        part[2 * blockIdx.x + 1] = s1;
    }
}

// y = K p on the free DOFs (held DOFs: y = 0, p taken as 0), and a partial of
// p.y. One warp per node: the lanes take its entries 32 apart and the sums
// meet in a fixed butterfly, so the product is deterministic.
__global__ void k_static_spmv(SNodes g, const uint32_t *__restrict__ a, const uint32_t *__restrict__ b,
                              const double *__restrict__ rig, const double *__restrict__ cv,
                              const double *__restrict__ p, double *y, double *part)
{
    __shared__ double sh[kThreads / 32];
    const int lane = threadIdx.x & 31;
    double acc = 0;
    const int64_t n = g.n, nB = g.nB;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        double pi[3];
        for (int c = 0; c < 3; c++) pi[c] = g.held[i + c * n] ? 0.0 : p[i + c * n];
        double yi[3] = {0, 0, 0};
        for (int64_t e = g.off[i] + lane; e < g.off[i + 1]; e += 32) {
            const uint32_t q = g.ent[e];
            const int64_t k = q >> 1;
            const double r = rig[k];
            if (r == 0) continue;
            const int64_t j = (q & 1u) ? a[k] : b[k];
            const double c0 = cv[k], c1 = cv[k + nB], c2 = cv[k + 2 * nB];
            double dp[3];
            for (int c = 0; c < 3; c++) dp[c] = pi[c] - (g.held[j + c * n] ? 0.0 : p[j + c * n]);
            const double t = r * (c0 * dp[0] + c1 * dp[1] + c2 * dp[2]);
            yi[0] += t * c0;
            yi[1] += t * c1;
            yi[2] += t * c2;
        }
        for (int o = 16; o > 0; o >>= 1)
            for (int c = 0; c < 3; c++) yi[c] += __shfl_xor_sync(0xffffffffu, yi[c], o);
        if (lane == 0)
            for (int c = 0; c < 3; c++) {
                const double v = g.held[i + c * n] ? 0.0 : yi[c];
                y[i + c * n] = v;
                acc += pi[c] * v;
            }
    }
    if (lane == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < kThreads / 32; w++) s += sh[w];
        part[blockIdx.x] = s;
    }
}

// Block-Jacobi preconditioner: the inverse of each node's 3 x 3 diagonal block
// restricted to its free DOFs (symmetric, 6 values); a DOF without stiffness
// (every bond of its node broken) is left out of the solve.
__global__ void k_static_precond(SNodes g, const uint32_t *__restrict__ a, const uint32_t *__restrict__ b,
                                 const double *__restrict__ rig, const double *__restrict__ cv, double *Minv,
                                 uint8_t *skip)
{
    const int64_t n = g.n, nB = g.nB;
    GRID_STRIDE(i, n)
    {
        double D[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int64_t e = g.off[i]; e < g.off[i + 1]; e++) {
            const int64_t k = g.ent[e] >> 1;
            const double r = rig[k];
            if (r == 0) continue;
            const double c[3] = {cv[k], cv[k + nB], cv[k + 2 * nB]};
            for (int u = 0; u < 3; u++)
                for (int v = 0; v < 3; v++) D[u][v] += r * c[u] * c[v];
        }
        bool fr[3];
        for (int u = 0; u < 3; u++) {
            fr[u] = !g.held[i + u * n] && D[u][u] > 0;
            skip[i + u * n] = fr[u] ? 0 : 1;
        }
        for (int u = 0; u < 3; u++)
            for (int v = 0; v < 3; v++)
                if (!fr[u] || !fr[v]) D[u][v] = (u == v) ? 1.0 : 0.0;
        // inverse of the symmetric 3 x 3 block by cofactors
        const double c00 = D[1][1] * D[2][2] - D[1][2] * D[2][1];
        const double c01 = D[1][2] * D[2][0] - D[1][0] * D[2][2];
        const double c02 = D[1][0] * D[2][1] - D[1][1] * D[2][0];
        const double det = D[0][0] * c00 + D[0][1] * c01 + D[0][2] * c02;
        double m[6];
        if (det > 0 && isfinite(det)) {
            const double id = 1.0 / det;
            m[0] = c00 * id;
            m[1] = c01 * id;
            m[2] = c02 * id;
            m[3] = (D[0][0] * D[2][2] - D[0][2] * D[2][0]) * id;
            m[4] = (D[0][2] * D[1][0] - D[0][0] * D[1][2]) * id;
            m[5] = (D[0][0] * D[1][1] - D[0][1] * D[1][0]) * id;
        } else {   // degenerate block: scalar Jacobi
            m[0] = 1.0 / D[0][0];
            m[3] = 1.0 / D[1][1];
            m[5] = 1.0 / D[2][2];
            m[1] = m[2] = m[4] = 0.0;
        }
        for (int q = 0; q < 6; q++) Minv[i + q * n] = m[q];
    }
}

__device__ __forceinline__ void apply_minv(const double *Minv, int64_t i, int64_t n, const double r[3], double z[3])
{
    const double m0 = Minv[i], m1 = Minv[i + n], m2 = Minv[i + 2 * n], m3 = Minv[i + 3 * n], m4 = Minv[i + 4 * n],
                 m5 = Minv[i + 5 * n];
    z[0] = m0 * r[0] + m1 * r[1] + m2 * r[2];
    z[1] = m1 * r[0] + m3 * r[1] + m4 * r[2];
    z[2] = m2 * r[0] + m4 * r[1] + m5 * r[2];
}

// CG start: delta = 0, r = F on the solved DOFs, z = M^-1 r, p = z; partials
// of r.z and r.r
__global__ void k_cg_init(int64_t n, const double *__restrict__ F, const uint8_t *__restrict__ skip,
                          const double *__restrict__ Minv, double *d, double *r, double *z, double *p, double *part)
{
    __shared__ double sh[2][kThreads / 32];
    double rz = 0, rr = 0;
    GRID_STRIDE(i, n)
    {
        double ri[3], zi[3];
        for (int c = 0; c < 3; c++) ri[c] = skip[i + c * n] ? 0.0 : F[i + c * n];
        apply_minv(Minv, i, n, ri, zi);
        for (int c = 0; c < 3; c++) {
            if (skip[i + c * n]) zi[c] = 0.0;
            d[i + c * n] = 0.0;
            r[i + c * n] = ri[c];
            z[i + c * n] = zi[c];
            p[i + c * n] = zi[c];
            rz += ri[c] * zi[c];
            rr += ri[c] * ri[c];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        rz += __shfl_xor_sync(0xffffffffu, rz, o);
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = rz;
        sh[1][threadIdx.x >> 5] = rr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            s0 += sh[0][w];
            s1 += sh[1][w];
        }
        part[2 * blockIdx.x] = s0;
        part[2 * blockIdx.x + 1] = s1;
    }
}

// Sum of `w` interleaved partial streams of `nb` blocks, in block order, to out[0..w)
__global__ void k_reduce(const double *__restrict__ part, int nb, int w, double *out)
{
    if (threadIdx.x < w) {
        double s = 0;
        for (int b = 0; b < nb; b++) s += part[b * w + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// scal: [0] r.z, [1] r.r, [2] p.Kp, [3] alpha
// delta += alpha p, r -= alpha Kp, z = M^-1 r; partials of the new r.z, r.r
__global__ void k_cg_update(int64_t n, const uint8_t *__restrict__ skip, const double *__restrict__ Minv,
                            const double *__restrict__ scal, const double *__restrict__ p,
                            const double *__restrict__ Kp, double *d, double *r, double *z, double *part)
{
    __shared__ double sh[2][kThreads / 32];
    const double alpha = scal[2] != 0 ? scal[0] / scal[2] : 0.0;
    double rz = 0, rr = 0;
    GRID_STRIDE(i, n)
    {
        double ri[3], zi[3];
        for (int c = 0; c < 3; c++) {
            const int64_t e = i + c * n;
            d[e] += alpha * p[e];
            ri[c] = r[e] - alpha * Kp[e];
            if (skip[e]) ri[c] = 0.0;
            r[e] = ri[c];
        }
        apply_minv(Minv, i, n, ri, zi);
        for (int c = 0; c < 3; c++) {
            if (skip[i + c * n]) zi[c] = 0.0;
            z[i + c * n] = zi[c];
            rz += ri[c] * zi[c];
            rr += ri[c] * ri[c];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        rz += __shfl_xor_sync(0xffffffffu, rz, o);
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = rz;
        sh[1][threadIdx.x >> 5] = rr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            s0 += sh[0][w];
            s1 += sh[1][w];
        }
        part[2 * blockIdx.x] = s0;
        part[2 * blockIdx.x + 1] = s1;
    }
}

// p = z + beta p with beta = (new r.z) / (old r.z); rolls r.z forward
__global__ void k_cg_direction(int64_t n, const double *__restrict__ z, double *p, const double *__restrict__ rzn,
                               const double *__restrict__ scal)
{
    const double beta = scal[0] != 0 ? rzn[0] / scal[0] : 0.0;
    GRID_STRIDE(e, 3 * n) p[e] = z[e] + beta * p[e];
}

__global__ void k_roll(double *scal, const double *__restrict__ rzn)
{
    if (threadIdx.x == 0) {
        scal[0] = rzn[0];
        scal[1] = rzn[1];
    }
}

__global__ void k_move(int64_t m, double *x, const double *__restrict__ d) { GRID_STRIDE(e, m) x[e] += d[e]; }

__global__ void k_prescribe(int64_t m, double *x, const uint8_t *__restrict__ held, double inc)
{
    GRID_STRIDE(e, m)
    if (held[e] == 2) x[e] += inc;
}

__global__ void k_iota(uint32_t *v, int64_t n) { GRID_STRIDE(i, n) v[i] = (uint32_t)i; }

__global__ void k_entry_keys(const uint32_t *__restrict__ a, const uint32_t *__restrict__ b, int64_t nB, uint32_t *key)
{
    GRID_STRIDE(q, 2 * nB) key[q] = (q & 1) ? b[q >> 1] : a[q >> 1];
}

__global__ void k_run_bounds(const uint32_t *__restrict__ skey, int64_t m, int64_t *first, int64_t *last)
{
    GRID_STRIDE(r, m)
    {
        const uint32_t p = skey[r];
        if (r == 0 || skey[r - 1] != p) first[p] = r;
        if (r == m - 1 || skey[r + 1] != p) last[p] = r + 1;
    }
}

__global__ void k_counts(const int64_t *__restrict__ first, const int64_t *__restrict__ last, int64_t n, int64_t *cnt)
{
    GRID_STRIDE(i, n + 1) cnt[i] = i < n ? last[i] - first[i] : 0;
}

}  // namespace

struct bbpd_static {
    int device = 0;
    cudaStream_t st = nullptr;
    int64_t n = 0, nB = 0;
    bbpd_params prm{};
    std::vector<void *> allocs;
    double *X = nullptr, *x = nullptr, *F = nullptr, *d = nullptr, *r = nullptr, *z = nullptr, *p = nullptr,
           *Kp = nullptr, *Minv = nullptr, *part = nullptr, *scal = nullptr, *rzn = nullptr, *red = nullptr;
    uint8_t *skip = nullptr;
    SBonds b{};
    SNodes g{};
    cudaGraphExec_t cg_exec = nullptr;   // kCgBlock conjugate-gradient iterations, captured once
    template <class T>
    int alloc(T **q, size_t count)
    {
        BBPD_CUDA_TRY(cudaMalloc((void **)q, sizeof(T) * std::max<size_t>(count, 1)));
        allocs.push_back((void *)*q);
        return BBPD_OK;
    }
    ~bbpd_static()
    {
        if (st) cudaStreamSynchronize(st);
        if (cg_exec) cudaGraphExecDestroy(cg_exec);
        for (void *q : allocs) cudaFree(q);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

constexpr int kCgBlock = 8;   // iterations between convergence checks

// `iters` conjugate-gradient iterations; the step sizes live in device memory,
// so nothing here waits for the host
void enqueue_cg(bbpd_static *S, int iters)
{
    cudaStream_t st = S->st;
    const int64_t n = S->n;
    for (int c = 0; c < iters; c++) {
        k_static_spmv<<<kRedBlocks, kThreads, 0, st>>>(S->g, S->b.a, S->b.b, S->b.rig, S->b.c, S->p, S->Kp, S->part);
        k_reduce<<<1, 32, 0, st>>>(S->part, kRedBlocks, 1, S->scal + 2);
        k_cg_update<<<kRedBlocks, kThreads, 0, st>>>(n, S->skip, S->Minv, S->scal, S->p, S->Kp, S->d, S->r, S->z,
                                                     S->part);
        k_reduce<<<1, 32, 0, st>>>(S->part, kRedBlocks, 2, S->rzn);
        k_cg_direction<<<blocks_for(3 * n), kThreads, 0, st>>>(n, S->z, S->p, S->rzn, S->scal);
        k_roll<<<1, 32, 0, st>>>(S->scal, S->rzn);
    }
}

// kCgBlock iterations as one graph launch (the 6 kernels of an iteration are
// launch-bound on small problems); captured on first use
int run_cg_block(bbpd_static *S)
{
    if (!S->cg_exec) {
        cudaGraph_t gr = nullptr;
        BBPD_CUDA_TRY(cudaStreamBeginCapture(S->st, cudaStreamCaptureModeThreadLocal));
        enqueue_cg(S, kCgBlock);
        cudaError_t e = cudaStreamEndCapture(S->st, &gr);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&S->cg_exec, gr, 0);
        if (gr) cudaGraphDestroy(gr);
        if (e != cudaSuccess) {
            S->cg_exec = nullptr;
            return fail(BBPD_ERR_CUDA, "conjugate-gradient graph: %s", cudaGetErrorString(e));
        }
    }
    BBPD_CUDA_TRY(cudaGraphLaunch(S->cg_exec, S->st));
    return BBPD_OK;
}

int read_scalars(bbpd_static *S, const double *src, int cnt, double *out)
{
    BBPD_CUDA_TRY(cudaMemcpyAsync(out, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost, S->st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(S->st));
    return BBPD_OK;
}

}  // namespace

extern "C" int bbpd_static_create(const bbpd_problem *pb, const bbpd_params *prm, int device, bbpd_static **out)
{
    clear_error();
    if (!pb || !prm || !out) return fail(BBPD_ERR_ARG, "null argument");
    *out = nullptr;
    TRY(require_device());
    const int64_t n = pb->n_nodes, nB = pb->n_bonds;
    if (n < 1 || n >= ((int64_t)1 << 31) || nB < 0 || nB >= ((int64_t)1 << 31))
        return fail(BBPD_ERR_ARG, "need 1 <= n_nodes < 2^31 and 0 <= n_bonds < 2^31");
    if (!pb->undeformed_coordinates || (nB && (!pb->bondlist || !pb->undeformed_length || !pb->bond_stiffness ||
                                               !pb->volume_correction)))
        return fail(BBPD_ERR_ARG, "missing coordinates or bond arrays");
    if (prm->law < 0 || prm->law > 3) return fail(BBPD_ERR_ARG, "bad law");
    if (!(prm->failure_functionality == 0.0 || prm->failure_functionality == 1.0))
        return fail(BBPD_ERR_UNSUPPORTED, "failure_functionality must be 0 or 1");
    if (pb->s0 || pb->s1 || pb->sc) return fail(BBPD_ERR_UNSUPPORTED, "the static solver takes scalar law stretches");
    const double *bl = pb->bondlist;
    std::vector<uint32_t> a(nB), bb(nB);
    std::vector<uint8_t> bt(nB, 0);
    std::vector<double> bfm(nB, 1.0), fl(nB, 1.0);
    for (int64_t k = 0; k < nB; k++) {
        const double ai = bl[k], bj = bl[nB + k];
        if (!(ai >= 1 && bj >= 1 && ai <= (double)n && bj <= (double)n && ai == std::floor(ai) && bj == std::floor(bj)))
            return fail(BBPD_ERR_ARG, "BONDLIST row %lld is not a pair of node ids", (long long)k + 1);
        a[k] = (uint32_t)(ai - 1);
        bb[k] = (uint32_t)(bj - 1);
        if (pb->bond_type) {
            const double t = pb->bond_type[k];
            if (!(t == 0 || t == 1 || t == 2)) return fail(BBPD_ERR_ARG, "BONDTYPE[%lld] = %g", (long long)k, t);
            bt[k] = (uint8_t)t;
            bfm[k] = t == 1 ? 3.0 : 1.0;   // buildbonddata.m:70-71
        }
        if (pb->fail) {
            const double f = pb->fail[k];
            if (!(f == 0 || f == 1)) return fail(BBPD_ERR_ARG, "fail[%lld] = %g", (long long)k, f);
            fl[k] = f;
        }
        if (pb->stretch_plastic && pb->stretch_plastic[k] != 0)
            return fail(BBPD_ERR_UNSUPPORTED, "non-zero stretchPlastic is not on this path");
    }
    std::vector<uint8_t> held(3 * n, 0);
    for (int64_t e = 0; e < 3 * n; e++) {
        const bool cf = pb->constraint_flag && pb->constraint_flag[e] == 1;
        const bool pf = pb->prescribed_flag && pb->prescribed_flag[e] == 1;
        held[e] = cf ? 1 : (pf ? 2 : 0);   // a support holds a DOF even where a load is prescribed
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return fail(BBPD_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    }
    auto *S = new bbpd_static;
    std::unique_ptr<bbpd_static> guard(S);
    S->device = device;
    S->n = n;
    S->nB = nB;
    S->prm = *prm;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    cudaStream_t st = S->st;
    TRY(S->alloc(&S->X, 3 * n));
    TRY(S->alloc(&S->x, 3 * n));
    TRY(staging::upload_copy(S->X, pb->undeformed_coordinates, 3 * n, st));
    BBPD_CUDA_TRY(cudaMemcpyAsync(S->x, S->X, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, st));
    for (double **q : {&S->F, &S->d, &S->r, &S->z, &S->p, &S->Kp}) TRY(S->alloc(q, 3 * n));
    TRY(S->alloc(&S->Minv, 6 * n));
    TRY(S->alloc(&S->skip, 3 * n));
    TRY(S->alloc(&S->part, 2 * kRedBlocks));
    TRY(S->alloc(&S->scal, 4));
    TRY(S->alloc(&S->rzn, 2));
    TRY(S->alloc(&S->red, 2));
    BBPD_CUDA_TRY(cudaMemsetAsync(S->F, 0, sizeof(double) * 3 * n, st));

    SBonds &B = S->b;
    uint32_t *da = nullptr, *db = nullptr;
    uint8_t *dbt = nullptr, *dheld = nullptr;
    double *dL0 = nullptr, *dBS = nullptr, *dV = nullptr, *dBFM = nullptr;
    TRY(S->alloc(&da, nB));
    TRY(S->alloc(&db, nB));
    TRY(S->alloc(&dbt, nB));
    TRY(S->alloc(&dL0, nB));
    TRY(S->alloc(&dBS, nB));
    TRY(S->alloc(&dV, nB));
    TRY(S->alloc(&dBFM, nB));
    TRY(S->alloc(&B.fail, nB));
    TRY(S->alloc(&B.bsf, nB));
    TRY(S->alloc(&B.flag, nB));
    TRY(S->alloc(&B.rig, nB));
    TRY(S->alloc(&B.c, 3 * nB));
    TRY(S->alloc(&B.f, 3 * nB));
    TRY(S->alloc(&dheld, 3 * n));
    TRY(staging::upload_copy(da, a.data(), nB, st));
    TRY(staging::upload_copy(db, bb.data(), nB, st));
    TRY(staging::upload_copy(dbt, bt.data(), nB, st));
    TRY(staging::upload_copy(dBFM, bfm.data(), nB, st));
    TRY(staging::upload_copy(B.fail, fl.data(), nB, st));
    TRY(staging::upload_copy(dheld, held.data(), 3 * n, st));
    if (nB) {
        TRY(staging::upload_copy(dL0, pb->undeformed_length, nB, st));
        TRY(staging::upload_copy(dBS, pb->bond_stiffness, nB, st));
        TRY(staging::upload_copy(dV, pb->volume_correction, nB, st));
    }
    BBPD_CUDA_TRY(cudaMemsetAsync(B.bsf, 0, sizeof(double) * std::max<int64_t>(nB, 1), st));
    BBPD_CUDA_TRY(cudaMemsetAsync(B.flag, 0, std::max<int64_t>(nB, 1), st));
    B.a = da;
    B.b = db;
    B.L0 = dL0;
    B.BS = dBS;
    B.VCF = dV;
    B.BFM = dBFM;
    B.BT = dbt;
    B.nB = nB;
    B.law = prm->law;
    B.V = prm->cell_volume;
    LawScalars &P = B.P;
    P.s0 = prm->s0;
    P.s1 = prm->s1;
    P.sc = prm->sc;
    P.beta = prm->beta_tri;
    const double eta = prm->s1 / prm->s0;
    P.tri_c1 = (eta - P.beta) / (eta - 1);
    P.tri_c2 = (1 - P.beta) / (eta - 1);
    P.k = prm->k_exp;
    P.alpha = prm->alpha_exp;
    P.exp_den = 1 - std::exp(-prm->k_exp);
    P.sc_steel = prm->sc_steel;
    P.ff = prm->failure_functionality;

    // per-node lists of bond ends in bond order: stable sort of q = 2k + side by node
    const int64_t m = 2 * nB;
    int64_t *off = nullptr;
    uint32_t *ent = nullptr;
    TRY(S->alloc(&off, n + 1));
    TRY(S->alloc(&ent, m));
    {
        uint32_t *key = nullptr, *skey = nullptr, *val = nullptr;
        int64_t *first = nullptr, *last = nullptr, *cnt = nullptr;
        uint8_t *tmp = nullptr;
        size_t tb = 0, ts = 0;
        int bits = 1;
        while (bits < 32 && ((int64_t)1 << bits) < n) bits++;
        BBPD_CUDA_TRY(cudaMallocAsync(&key, sizeof(uint32_t) * std::max<int64_t>(m, 1), st));
        BBPD_CUDA_TRY(cudaMallocAsync(&skey, sizeof(uint32_t) * std::max<int64_t>(m, 1), st));
        BBPD_CUDA_TRY(cudaMallocAsync(&val, sizeof(uint32_t) * std::max<int64_t>(m, 1), st));
        BBPD_CUDA_TRY(cudaMallocAsync(&first, sizeof(int64_t) * n, st));
        BBPD_CUDA_TRY(cudaMallocAsync(&last, sizeof(int64_t) * n, st));
        BBPD_CUDA_TRY(cudaMallocAsync(&cnt, sizeof(int64_t) * (n + 1), st));
        BBPD_CUDA_TRY(cudaMemsetAsync(first, 0, sizeof(int64_t) * n, st));
        BBPD_CUDA_TRY(cudaMemsetAsync(last, 0, sizeof(int64_t) * n, st));
        if (m > 0) {
            k_entry_keys<<<blocks_for(m), kThreads, 0, st>>>(da, db, nB, key);
            k_iota<<<blocks_for(m), kThreads, 0, st>>>(val, m);
            BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, skey, val, ent, m, 0, bits, st));
        }
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, ts, cnt, off, n + 1, st));
        BBPD_CUDA_TRY(cudaMallocAsync(&tmp, std::max<size_t>(std::max(tb, ts), 1), st));
        int rc = BBPD_OK;
        if (m > 0) {
            cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tb, key, skey, val, ent, m, 0, bits, st);
            if (e == cudaSuccess) {
                k_run_bounds<<<blocks_for(m), kThreads, 0, st>>>(skey, m, first, last);
                e = cudaGetLastError();
            }
            if (e != cudaSuccess) rc = fail(BBPD_ERR_CUDA, "static solver lists: %s", cudaGetErrorString(e));
        }
        if (rc == BBPD_OK) {
            k_counts<<<blocks_for(n + 1), kThreads, 0, st>>>(first, last, n, cnt);
            size_t t2 = std::max(tb, ts);
            cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, t2, cnt, off, n + 1, st);
            if (e != cudaSuccess) rc = fail(BBPD_ERR_CUDA, "static solver lists: %s", cudaGetErrorString(e));
        }
        for (void *q : {(void *)key, (void *)skey, (void *)val, (void *)first, (void *)last, (void *)cnt, (void *)tmp})
            cudaFreeAsync(q, st);
        TRY(rc);
    }
    S->g.off = off;
    S->g.ent = ent;
    S->g.held = dheld;
    S->g.n = n;
    S->g.nB = nB;
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    *out = guard.release();
    return BBPD_OK;
}

extern "C" int bbpd_static_step(bbpd_static *S, double increment, double tol, int max_newton, double cg_tol,
                                int max_cg, bbpd_static_stats *stats)
{
    if (!S || !stats) return fail(BBPD_ERR_ARG, "null argument");
    if (!(tol > 0) || !(cg_tol > 0) || max_newton < 1 || max_cg < 1 || !std::isfinite(increment))
        return fail(BBPD_ERR_ARG, "need tol > 0, cg_tol > 0, max_newton >= 1, max_cg >= 1, finite increment");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t st = S->st;
    const int64_t n = S->n;
    *stats = bbpd_static_stats{};
    if (increment != 0) k_prescribe<<<blocks_for(3 * n), kThreads, 0, st>>>(3 * n, S->x, S->g.held, increment);
    for (int it = 0;; it++) {
        k_static_bonds<<<blocks_for(S->nB), kThreads, 0, st>>>(S->b, S->x, n);
        k_static_nodal<<<kRedBlocks, kThreads, 0, st>>>(S->g, S->b.f, S->prm.cell_volume, S->F, S->part);
        k_reduce<<<1, 32, 0, st>>>(S->part, kRedBlocks, 2, S->red);
        TRY(launch_check());
        double rr[2];
        TRY(read_scalars(S, S->red, 2, rr));
        stats->residual = std::sqrt(rr[0]);
        stats->reaction = std::sqrt(rr[1]);
        stats->newton_iterations = it;
        if (!std::isfinite(stats->residual) || !std::isfinite(stats->reaction))
            return fail(BBPD_ERR_NONFINITE, "non-finite nodal force");
        if (stats->residual <= tol * stats->reaction || stats->residual == 0) {
            stats->converged = 1;
            return BBPD_OK;
        }
        if (it == max_newton) return BBPD_OK;   // not converged: stats say so
        // K delta = F on the free DOFs by PCG
        k_static_precond<<<blocks_for(n), kThreads, 0, st>>>(S->g, S->b.a, S->b.b, S->b.rig, S->b.c, S->Minv, S->skip);
        k_cg_init<<<kRedBlocks, kThreads, 0, st>>>(n, S->F, S->skip, S->Minv, S->d, S->r, S->z, S->p, S->part);
        k_reduce<<<1, 32, 0, st>>>(S->part, kRedBlocks, 2, S->scal);
        TRY(launch_check());
        double s01[2];
        TRY(read_scalars(S, S->scal, 2, s01));
        const double rr0 = s01[1];
        if (rr0 > 0) {
            for (int done = 0; done < max_cg;) {
                const int blk = std::min(kCgBlock, max_cg - done);
                if (blk == kCgBlock) TRY(run_cg_block(S));
                else enqueue_cg(S, blk);
                TRY(launch_check());
                done += blk;
                stats->cg_iterations += blk;
                double rz[2];
                TRY(read_scalars(S, S->rzn, 2, rz));
                if (!std::isfinite(rz[1])) return fail(BBPD_ERR_NONFINITE, "conjugate gradient diverged");
                if (rz[1] <= cg_tol * cg_tol * rr0) break;
            }
        }
        k_move<<<blocks_for(3 * n), kThreads, 0, st>>>(3 * n, S->x, S->d);
        TRY(launch_check());
    }
}

extern "C" int bbpd_static_get(bbpd_static *S, int field, double *out)
{
    if (!S || !out) return fail(BBPD_ERR_ARG, "null argument");
    BBPD_CUDA_TRY(cudaSetDevice(S->device));
    cudaStream_t st = S->st;
    const int64_t n = S->n, nB = S->nB;
    switch (field) {
    case BBPD_FIELD_DEFORMED: return staging::download_copy(out, S->x, 3 * n, st);
    case BBPD_FIELD_FORCE: return staging::download_copy(out, S->F, 3 * n, st);
    case BBPD_FIELD_DISPLACEMENT: {
        const double *x = S->x;
        TRY(staging::download_copy(out, x, 3 * n, st));
        std::vector<double> X(3 * n);
        TRY(staging::download_copy(X.data(), S->X, 3 * n, st));
        for (int64_t e = 0; e < 3 * n; e++) out[e] = out[e] - X[e];
        return BBPD_OK;
    }
    case BBPD_FIELD_BSF: return staging::download_copy(out, S->b.bsf, nB, st);
    case BBPD_FIELD_FAIL: return staging::download_copy(out, S->b.fail, nB, st);
    case BBPD_FIELD_FLAG: {
        std::vector<uint8_t> f(nB);
        TRY(staging::download_copy(f.data(), S->b.flag, nB, st));
        for (int64_t k = 0; k < nB; k++) out[k] = f[k];
        return BBPD_OK;
    }
    default: return fail(BBPD_ERR_ARG, "field %d not held by the static solver", field);
    }
}

extern "C" int bbpd_static_destroy(bbpd_static *S)
{
    if (!S) return BBPD_OK;
    cudaSetDevice(S->device);
    delete S;
    return BBPD_OK;
}

// ---- buildstiffnessmatrixCSCformat.m as a routine ----

namespace {

struct CooBonds {
    const double *X;            // nodal coordinates, nNodes x NOD
    const double *bl, *VCF, *BS, *BFM, *fail, *BSF;
    int64_t n, nB;
    int NOD;
    double V;
};

// Local stiffness of bond k: its scale rig and bond vector (NOD components);
// false for a failed bond (buildstiffnessmatrixCSCformat.m:72, :110).
__device__ __forceinline__ bool coo_local(const CooBonds &q, int64_t k, double &rig, double c[3], int64_t &i,
                                          int64_t &j)
{
    if (q.fail[k] != 1) return false;
    i = (int64_t)q.bl[k] - 1;
    j = (int64_t)q.bl[q.nB + k] - 1;
    double L2 = 0;
    for (int u = 0; u < q.NOD; u++) {
        c[u] = q.X[j + u * q.n] - q.X[i + u * q.n];
        L2 = u == 0 ? c[u] * c[u] : L2 + c[u] * c[u];
    }
    const double L = sqrt(L2);
    if (q.NOD == 3)   // :116
        rig = q.BFM[k] * ((q.BS[k] / (L * L * L)) * q.VCF[k] * (q.V * q.V)) * (1 - q.BSF[k]);
    else              // :78
        rig = q.BFM[k] * (q.BS[k] / (L * L * L)) * q.VCF[k] * (q.V * q.V);
    return true;
}

// entry (r, s) of the 2 NOD x 2 NOD local matrix rig [A -A; -A A], A = c c^T
__device__ __forceinline__ double coo_entry(double rig, const double *c, int NOD, int r, int s)
{
    const double m = c[r % NOD] * c[s % NOD];
    return ((r < NOD) == (s < NOD)) ? rig * m : rig * (-m);
}

// nonzero count and norm(Klocal) of every bond; norm = 2 |rig| |c|^2, the
// largest singular value of rig [A -A; -A A]
__global__ void k_coo_count(CooBonds q, int64_t *cnt, double *nrm)
{
    GRID_STRIDE(k, q.nB + 1)
    {
        if (k == q.nB) {
            cnt[k] = 0;
            continue;
        }
        double rig, c[3];
        int64_t i, j;
        int64_t z = 0;
        double nm = 0;
        if (coo_local(q, k, rig, c, i, j)) {
            const int D = 2 * q.NOD;
            for (int s = 0; s < D; s++)
                for (int r = 0; r < D; r++) z += coo_entry(rig, c, q.NOD, r, s) != 0;
            double L2 = 0;
            for (int u = 0; u < q.NOD; u++) L2 = u == 0 ? c[u] * c[u] : L2 + c[u] * c[u];
            nm = 2 * fabs(rig) * L2;
        }
        cnt[k] = z;
        nrm[k] = nm;
    }
}

// nonzeros of every bond in MATLAB find order (column-major), with 1-based
// global DOFs NOD (node - 1) + 1 .. NOD node (:91-100, :129-138)
__global__ void k_coo_write(CooBonds q, const int64_t *__restrict__ off, double *rows, double *cols, double *vals)
{
    GRID_STRIDE(k, q.nB)
    {
        double rig, c[3];
        int64_t i, j;
        if (!coo_local(q, k, rig, c, i, j)) continue;
        const int D = 2 * q.NOD;
        int64_t o = off[k];
        for (int s = 0; s < D; s++)
            for (int r = 0; r < D; r++) {
                const double v = coo_entry(rig, c, q.NOD, r, s);
                if (v == 0) continue;
                const int64_t gr = (r < q.NOD ? q.NOD * i : q.NOD * j) + (r % q.NOD) + 1;
                const int64_t gc = (s < q.NOD ? q.NOD * i : q.NOD * j) + (s % q.NOD) + 1;
                rows[o] = (double)gr;
                cols[o] = (double)gc;
                vals[o] = v;
                o++;
            }
    }
}

__global__ void k_node_sum(const int64_t *__restrict__ off, const uint32_t *__restrict__ ent, int64_t n,
                           const double *__restrict__ v, double *out)
{
    GRID_STRIDE(i, n)
    {
        double a = 0;
        for (int64_t e = off[i]; e < off[i + 1]; e++) a = a + v[ent[e] >> 1];
        out[i] = a;
    }
}

__global__ void k_bl_nodes(const double *__restrict__ bl, int64_t nB, int64_t n, uint32_t *a, uint32_t *b, int *bad)
{
    GRID_STRIDE(k, nB)
    {
        const double x = bl[k], y = bl[nB + k];
        if (!(x >= 1 && y >= 1 && x <= (double)n && y <= (double)n)) {
            *bad = 1;
            a[k] = b[k] = 0;
            continue;
        }
        a[k] = (uint32_t)(x - 1);
        b[k] = (uint32_t)(y - 1);
    }
}

}  // namespace

extern "C" int bbpd_dev_buildstiffnessmatrix(const double *X, int64_t nNodes, int NOD, const double *BONDLIST,
        const double *VCF, double VOLUME, const double *BS, const double *BFM, const double *failFlag, const double *BSF,
        int64_t nBonds, int64_t capacity, int64_t *nnz, double *rowIndex, double *columnIndex, double *values,
        double *massVector, void *stream)
{
    if (!nnz) return fail(BBPD_ERR_ARG, "null nnz");
    if (NOD != 2 && NOD != 3) return fail(BBPD_ERR_ARG, "NOD must be 2 or 3");
    if (nNodes < 1 || nNodes >= ((int64_t)1 << 31) || nBonds < 0 || nBonds >= ((int64_t)1 << 31))
        return fail(BBPD_ERR_ARG, "need 1 <= nNodes < 2^31 and 0 <= nBonds < 2^31");
    if (!X || (nBonds && (!BONDLIST || !VCF || !BS || !BFM || !failFlag || !BSF))) return fail(BBPD_ERR_ARG, "null array");
    TRY(require_device());
    cudaStream_t st = as_stream(stream);
    const int64_t n = nNodes, nB = nBonds, m = 2 * nB;
    CooBonds q{X, BONDLIST, VCF, BS, BFM, failFlag, BSF, n, nB, NOD, VOLUME};
    std::vector<void *> tmp;
    auto get = [&](void **p, size_t bytes) -> int {
        BBPD_CUDA_TRY(cudaMallocAsync(p, std::max<size_t>(bytes, 8), st));
        tmp.push_back(*p);
        return BBPD_OK;
    };
    struct Free {
        std::vector<void *> &t;
        cudaStream_t s;
        ~Free()
        {
            for (void *p : t) cudaFreeAsync(p, s);
        }
    } freer{tmp, st};
    uint32_t *a = nullptr, *b = nullptr, *key = nullptr, *skey = nullptr, *val = nullptr, *ent = nullptr;
    int64_t *cnt = nullptr, *off = nullptr, *first = nullptr, *last = nullptr, *ncnt = nullptr, *noff = nullptr;
    double *nrm = nullptr;
    int *bad = nullptr;
    TRY(get((void **)&a, 4 * nB));
    TRY(get((void **)&b, 4 * nB));
    TRY(get((void **)&bad, sizeof(int)));
    TRY(get((void **)&cnt, 8 * (nB + 1)));
    TRY(get((void **)&off, 8 * (nB + 1)));
    TRY(get((void **)&nrm, 8 * nB));
    BBPD_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    k_bl_nodes<<<blocks_for(nB), kThreads, 0, st>>>(BONDLIST, nB, n, a, b, bad);
    k_coo_count<<<blocks_for(nB + 1), kThreads, 0, st>>>(q, cnt, nrm);
    TRY(launch_check());
    size_t tb = 0;
    BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, nB + 1, st));
    void *t1 = nullptr;
    TRY(get(&t1, tb));
    BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(t1, tb, cnt, off, nB + 1, st));
    int64_t total = 0;
    int hbad = 0;
    BBPD_CUDA_TRY(cudaMemcpyAsync(&total, off + nB, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    if (hbad) return fail(BBPD_ERR_ARG, "BONDLIST holds node ids outside [1, nNodes]");
    *nnz = total;
    if (capacity >= total && total > 0 && rowIndex && columnIndex && values) {
        k_coo_write<<<blocks_for(nB), kThreads, 0, st>>>(q, off, rowIndex, columnIndex, values);
        TRY(launch_check());
    }
    if (massVector) {
        // massVector(i) accumulates norm(Klocal) of its intact bonds in bond order
        TRY(get((void **)&key, 4 * m));
        TRY(get((void **)&skey, 4 * m));
        TRY(get((void **)&val, 4 * m));
        TRY(get((void **)&ent, 4 * m));
        TRY(get((void **)&first, 8 * n));
        TRY(get((void **)&last, 8 * n));
        TRY(get((void **)&ncnt, 8 * (n + 1)));
        TRY(get((void **)&noff, 8 * (n + 1)));
        BBPD_CUDA_TRY(cudaMemsetAsync(first, 0, 8 * n, st));
        BBPD_CUDA_TRY(cudaMemsetAsync(last, 0, 8 * n, st));
        int bits = 1;
        while (bits < 32 && ((int64_t)1 << bits) < n) bits++;
        if (m > 0) {
            k_entry_keys<<<blocks_for(m), kThreads, 0, st>>>(a, b, nB, key);
            k_iota<<<blocks_for(m), kThreads, 0, st>>>(val, m);
            BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, skey, val, ent, m, 0, bits, st));
            void *t2 = nullptr;
            TRY(get(&t2, tb));
            BBPD_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t2, tb, key, skey, val, ent, m, 0, bits, st));
            k_run_bounds<<<blocks_for(m), kThreads, 0, st>>>(skey, m, first, last);
        }
        k_counts<<<blocks_for(n + 1), kThreads, 0, st>>>(first, last, n, ncnt);
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, ncnt, noff, n + 1, st));
        void *t3 = nullptr;
        TRY(get(&t3, tb));
        BBPD_CUDA_TRY(cub::DeviceScan::ExclusiveSum(t3, tb, ncnt, noff, n + 1, st));
        k_node_sum<<<blocks_for(n), kThreads, 0, st>>>(noff, ent, n, nrm, massVector);
        TRY(launch_check());
    }
    BBPD_CUDA_TRY(cudaStreamSynchronize(st));
    return BBPD_OK;
}

extern "C" int bbpd_buildstiffnessmatrix(const double *X, int64_t nNodes, int NOD, const double *BONDLIST,
        const double *VCF, double VOLUME, const double *BS, const double *BFM, const double *failFlag, const double *BSF,
        int64_t nBonds, int64_t capacity, int64_t *nnz, double *rowIndex, double *columnIndex, double *values,
        double *massVector)
{
    if (!nnz) return fail(BBPD_ERR_ARG, "null nnz");
    if (NOD != 2 && NOD != 3) return fail(BBPD_ERR_ARG, "NOD must be 2 or 3");
    if (nNodes < 1 || nBonds < 0) return fail(BBPD_ERR_ARG, "bad sizes");
    if (!X || (nBonds && (!BONDLIST || !VCF || !BS || !BFM || !failFlag || !BSF))) return fail(BBPD_ERR_ARG, "null array");
    TRY(require_device());
    cudaStream_t st = nullptr;
    BBPD_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Own {
        cudaStream_t s;
        std::vector<void *> p;
        ~Own()
        {
            for (void *q : p) cudaFreeAsync(q, s);
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } own{st, {}};
    auto up = [&](const double *h, int64_t cnt, double **d) -> int {
        BBPD_CUDA_TRY(cudaMallocAsync((void **)d, sizeof(double) * std::max<int64_t>(cnt, 1), st));
        own.p.push_back(*d);
        return h ? staging::upload_copy(*d, h, cnt, st) : BBPD_OK;
    };
    const int64_t nB = nBonds;
    double *dX, *dbl, *dV, *dBS, *dBFM, *dfail, *dBSF, *dm = nullptr;
    TRY(up(X, NOD * nNodes, &dX));
    TRY(up(BONDLIST, 2 * nB, &dbl));
    TRY(up(VCF, nB, &dV));
    TRY(up(BS, nB, &dBS));
    TRY(up(BFM, nB, &dBFM));
    TRY(up(failFlag, nB, &dfail));
    TRY(up(BSF, nB, &dBSF));
    if (massVector) TRY(up(nullptr, nNodes, &dm));
    TRY(bbpd_dev_buildstiffnessmatrix(dX, nNodes, NOD, dbl, dV, VOLUME, dBS, dBFM, dfail, dBSF, nB, 0, nnz, nullptr,
                                      nullptr, nullptr, dm, st));
    const int64_t total = *nnz;
    if (capacity >= total && total > 0 && rowIndex && columnIndex && values) {
        double *dr, *dc, *dv;
        TRY(up(nullptr, total, &dr));
        TRY(up(nullptr, total, &dc));
        TRY(up(nullptr, total, &dv));
        int64_t again = 0;
        TRY(bbpd_dev_buildstiffnessmatrix(dX, nNodes, NOD, dbl, dV, VOLUME, dBS, dBFM, dfail, dBSF, nB, total, &again,
                                          dr, dc, dv, nullptr, st));
        TRY(staging::download_copy(rowIndex, dr, total, st));
        TRY(staging::download_copy(columnIndex, dc, total, st));
        TRY(staging::download_copy(values, dv, total, st));
    }
    if (dm) TRY(staging::download_copy(massVector, dm, nNodes, st));
    return BBPD_OK;
}
