// Per-routine CUDA kernels: one entry point per reference MEX routine (and per
// MATLAB-only routine of the hot path), with the reference's argument meaning
// and in-place semantics. Bond routines run one thread per bond, node routines
// one thread per node. The nodal force sum is node-centric: a plan holds each
// node's bonds in bond order and the node adds them in the reference's OpenMP
// order, so no atomics are needed and the result is bit-identical.
//
// Host-pointer variants (used by the mexFunction gateways) keep a device
// mirror per host buffer, copy the inputs in, run, copy the outputs back and
// synchronize.
#include "bbpd_internal.h"
#include "physics.cuh"
#include "staging.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <mutex>
#include <unordered_map>
#include <vector>

using namespace bbpd;

namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n)
{
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;  // grid-stride beyond this
    return (int)b;
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_deformedlength(const double *__restrict__ x, const double *__restrict__ bl,
                                 const double *__restrict__ L0, int64_t nB, int64_t nN,
                                 double *L, double *dX, double *dY, double *dZ, double *s)
{
    GRID_STRIDE(k, nB)
    {
        int64_t i = (int64_t)bl[k], j = (int64_t)bl[nB + k];
        double a, b, c, l, st;
        bond_kinematics(x[i - 1], x[i - 1 + nN], x[i - 1 + 2 * nN], x[j - 1], x[j - 1 + nN],
                        x[j - 1 + 2 * nN], L0[k], a, b, c, l, st);
        dX[k] = a; dY[k] = b; dZ[k] = c; L[k] = l; s[k] = st;
    }
}

__global__ void k_bsfexponential(const double *__restrict__ s, const double *__restrict__ s0,
                                 const double *__restrict__ sc, LawScalars P, double *bsf,
                                 double *BSF, const double *__restrict__ BT, double *flag,
                                 int64_t nB)
{
    GRID_STRIDE(k, nB)
    {
        if (BT[k] != 0) continue;
        double B = BSF[k];
        bool f = false;
        double bs = bsf[k];   // caller-zeroed scratch; the reference writes it in place
        double s0k = s0[k], sck = sc[k], sk = s[k];
        if (s0k < sk && sk <= sck) {
            f = true;
            double numerator = 1 - cr_exp(-P.k * (sk - s0k) / (sck - s0k));   // correctly rounded (crexp.cuh)
            double residual = P.alpha * (1 - (sk - s0k) / (sck - s0k));
            bs = 1 - (s0k / sk) * ((1 - (numerator / P.exp_den)) + residual) / (1 + P.alpha);
            bsf[k] = bs;
        } else if (sk > sck) {
            bs = 1;
            bsf[k] = bs;
        }
        if (bs > B) B = bs;
        if (B > 1) B = 1;
        if (B != B) B = 0.0;
        BSF[k] = B;
        if (f) flag[k] = 1;
    }
}

__global__ void k_bsftrilinear(const double *__restrict__ s, LawScalars P, double *BSF,
                               const double *__restrict__ BT, double *flag, int64_t nB)
{
    GRID_STRIDE(k, nB)
    {
        double B = BSF[k];
        bool f = false;
        law_trilinear(s[k], P.s0, P.s1, P.sc, P, false, BT[k] == 0, B, f);
        BSF[k] = B;
        if (f) flag[k] = 1;
    }
}

__global__ void k_bilinear(const double *__restrict__ s, LawScalars P, double *flag,
                           double *BSF, const double *__restrict__ BT, int64_t nB)
{
    GRID_STRIDE(k, nB)
    {
        double B = BSF[k];
        // flag is a double in the reference: a pre-set non-zero value other than 1
        // still multiplies bsf (calculatebondsofteningfactor.m:163)
        double fl = flag[k];
        if (BT[k] == 0 && s[k] > P.s0) fl = 1;
        double bsf = ((s[k] - P.s0) / s[k]) * (P.sc / (P.sc - P.s0));
        B = matlab_max(B, bsf * fl);
        if (B > 1) B = 1;
        if (isnan(B)) B = 0;
        BSF[k] = B;
        flag[k] = fl;
    }
}

__global__ void k_bondfailure(double *fail, LawScalars P, const double *__restrict__ BT,
                              const double *__restrict__ s, int64_t nB)
{
    GRID_STRIDE(k, nB)
    {
        double f = fail[k];
        law_linear(s[k], P.sc, P, (int)BT[k], f);
        fail[k] = f;
    }
}

__global__ void k_bondforces(double *fX, double *fY, double *fZ, const double *__restrict__ fail,
                             const double *__restrict__ dX, const double *__restrict__ dY,
                             const double *__restrict__ dZ, const double *__restrict__ L,
                             const double *__restrict__ s, const double *__restrict__ sp,
                             const double *__restrict__ BS, double V,
                             const double *__restrict__ VCF, const double *__restrict__ BSF,
                             int64_t nB)
{
    GRID_STRIDE(k, nB)
    {
        double t = bond_force_scalar(fail[k], BS[k], BSF[k], s[k], sp[k], V, VCF[k]);
        fX[k] = bond_force_component(t, dX[k], L[k]);
        fY[k] = bond_force_component(t, dY[k], L[k]);
        fZ[k] = bond_force_component(t, dZ[k], L[k]);
    }
}

__global__ void k_eulercromer(double *a, const double *__restrict__ F, double D, double *v,
                              const double *__restrict__ rho, const double *__restrict__ CF,
                              double dt, double *u, double *x, const double *__restrict__ X,
                              int64_t nN, int NOD)
{
    GRID_STRIDE(k, nN)
    {
        for (int d = 0; d < NOD; d++) {
            int64_t e = k + nN * d;
            double ae = (F[e] - D * v[e]) / rho[k];
            if (CF[e] == 1) ae = 0;
            double ve = v[e] + (ae * dt);
            double ue = u[e] + (ve * dt);
            a[e] = ae; v[e] = ve; u[e] = ue;
            x[e] = X[e] + ue;
        }
    }
}

__global__ void k_adr(int64_t it, double dt, double *vh, const double *__restrict__ F,
                      const double *__restrict__ m, double cn, const double *vhp, double *u,
                      const double *__restrict__ CF, int64_t nN)
{
    GRID_STRIDE(k, nN)
    {
        double minv = 1.0 / m[k];
        for (int d = 0; d < 3; d++) {
            int64_t e = k + nN * d;
            double v;
            if (it == 1) v = 0.5 * dt * minv * F[e];
            else v = (((2 - cn * dt) * vhp[e]) + (2 * dt * minv * F[e])) / (2 + cn * dt);
            double ue = u[e] + (dt * v);
            if (CF[e] == 1) { ue = 0; v = 0; }
            u[e] = ue;
            vh[e] = v;
        }
    }
}

// Per-node Rayleigh-quotient terms, xor-butterfly over 32 nodes per warp:
// calculatedampingcoefficient.m:61-85 in the fixed order of the fused solver.
__global__ void k_damping_slices(const double *__restrict__ F, const double *__restrict__ m,
                                 const double *__restrict__ Fp, double dt,
                                 const double *__restrict__ vhp, const double *__restrict__ u,
                                 int64_t nN, int64_t nsl, double *part)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t sl = warp; sl < nsl; sl += nwarps) {
        int64_t i = sl * 32 + lane;
        double c1 = 0, c2 = 0;
        if (i < nN) {
            for (int d = 0; d < 3; d++) {
                int64_t e = i + nN * d;
                if (vhp[e] != 0)
                    c1 = c1 - u[e] * u[e] * ((F[e] / m[i] - Fp[e] / m[i]) / (dt * vhp[e]));
            }
            for (int d = 0; d < 3; d++) {
                int64_t e = i + nN * d;
                c2 = c2 + u[e] * u[e];
            }
        }
        for (int off = 16; off >= 1; off >>= 1) {
            c1 = c1 + __shfl_xor_sync(0xffffffffu, c1, off);
            c2 = c2 + __shfl_xor_sync(0xffffffffu, c2, off);
        }
        if (lane == 0) { part[sl] = c1; part[nsl + sl] = c2; }
    }
}

// Upper levels of the 32-ary tree over the slice partials (groups of 32
// consecutive partials, xor butterfly, missing members 0.0) until one value is
// left; one block of 1024 threads, ping-pong buffers a/b of ceil(nsl/32) each.
// Then the clamp of calculatedampingcoefficient.m:90-112.
__global__ void __launch_bounds__(1024) k_damping_final(const double *part, int64_t nsl, double *a,
                                                        double *b, double *cn_out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double *src = part;
    int64_t cnt = nsl;
    double *dst = a;
    // src holds cnt pairs as [cnt1 ..., cnt2 ...] with stride `sstride`
    int64_t sstride = nsl;
    while (cnt > 1) {
        const int64_t m = (cnt + 31) / 32;
        for (int64_t g = warp; g < m; g += 32) {
            const int64_t idx = g * 32 + lane;
            double c1 = idx < cnt ? src[idx] : 0.0, c2 = idx < cnt ? src[sstride + idx] : 0.0;
            for (int off = 16; off >= 1; off >>= 1) {
                c1 = c1 + __shfl_xor_sync(0xffffffffu, c1, off);
                c2 = c2 + __shfl_xor_sync(0xffffffffu, c2, off);
            }
            if (lane == 0) { dst[g] = c1; dst[m + g] = c2; }
        }
        __syncthreads();
        src = dst;
        sstride = m;
        cnt = m;
        dst = (dst == a) ? b : a;
    }
    if (threadIdx.x == 0) {
        const double c1 = nsl > 0 ? src[0] : 0.0, c2 = nsl > 0 ? src[sstride] : 0.0;
        double cn;
        if (c2 != 0) {
            if ((c1 / c2) > 0) cn = 2 * sqrt(c1 / c2);
            else cn = 0;
        } else {
            cn = 0;
        }
        if (cn > 2) cn = 1.9;
        *cn_out = cn;
    }
}

// calculatedamage.m:34-43: unbroken bonds per node, accumulated into
// damage[] (fail is 0 or 1, so the sums are exact integers in any order).
// Ids outside [1, nN] are skipped and reported through *bad.
__global__ void k_damage_count(const double *__restrict__ bl, const double *__restrict__ fail_,
                               int64_t nB, int64_t nN, double *damage, int *bad)
{
    GRID_STRIDE(k, nB)
    {
        const double di = bl[k], dj = bl[nB + k];
        if (!(di >= 1 && dj >= 1 && di <= (double)nN && dj <= (double)nN)) {
            *bad = 1;
            continue;
        }
        const double f = fail_[k];
        atomicAdd(&damage[(int64_t)di - 1], f);
        atomicAdd(&damage[(int64_t)dj - 1], f);
    }
}

// calculatedamage.m:45: damage = 1 - unbroken / nFAMILYMEMBERS.
__global__ void k_damage_final(const double *__restrict__ nfam, int64_t nN, double *damage)
{
    GRID_STRIDE(i, nN)
    damage[i] = 1 - (damage[i] / nfam[i]);
}

// calculatedamageenergy.m:34-62: energy dissipated by each bond, never
// decreasing. shape = 2k - 2e^k + alpha k - alpha k e^k + 2 and den =
// 2k (e^k - 1)(1 + alpha) are formed once on the host; every product keeps the
// reference's left-to-right order.
__global__ void k_damageenergy(const double *__restrict__ BS, const double *__restrict__ s0,
                               const double *__restrict__ sc, const double *__restrict__ L0,
                               const double *__restrict__ stretch, double shape, double den, double V2,
                               double *energy, int64_t nB)
{
    GRID_STRIDE(k, nB)
    {
        const double s = stretch[k], a = s0[k], c = sc[k];
        double de = 0.0;
        if ((a < s) && (s <= c)) de = (((((BS[k] * a) * L0[k]) * (a - s)) * shape) / den) * V2;
        else if (s > c) de = (((((BS[k] * a) * L0[k]) * (a - c)) * shape) / den) * V2;
        const double e = energy[k];
        energy[k] = isnan(e) ? de : (de > e ? de : e);   // MATLAB's max ignores NaN
    }
}

// ---- nodal force plan ----

__global__ void k_plan_keys(const double *__restrict__ bl, int64_t nB, int64_t nN,
                            int32_t *keys, int64_t *vals, int *bad)
{
    GRID_STRIDE(k, nB)
    {
        double di = bl[k], dj = bl[nB + k];
        int64_t i = (int64_t)di, j = (int64_t)dj;
        if (!(di == (double)i && dj == (double)j && i >= 1 && j >= 1 && i <= nN && j <= nN && i != j)) {
            *bad = 1;
            i = j = 1;
        }
        keys[2 * k] = (int32_t)(i - 1);
        keys[2 * k + 1] = (int32_t)(j - 1);
        vals[2 * k] = 2 * k;          // i end: +f
        vals[2 * k + 1] = 2 * k + 1;  // j end: -f
    }
}

__global__ void k_plan_count(const int32_t *keys, int64_t n, int32_t *cnt)
{
    GRID_STRIDE(p, n) atomicAdd(&cnt[keys[p]], 1);
}

__global__ void k_nodalforces(const int64_t *__restrict__ rp, const int64_t *__restrict__ ent,
                              int64_t nB, int64_t nN, int T, double *F,
                              const double *__restrict__ fX, const double *__restrict__ fY,
                              const double *__restrict__ fZ)
{
    GRID_STRIDE(n, nN)
    {
        // nodalForce[n] += thread partials in thread order (calculatenodalforcesopenmpMex.c:70-80)
        double tx = F[n], ty = F[n + nN], tz = F[n + 2 * nN];
        double ax = 0.0, ay = 0.0, az = 0.0;
        int cur = -1;
        for (int64_t p = rp[n]; p < rp[n + 1]; p++) {
            int64_t v = ent[p], k = v >> 1;
            int c = omp_chunk_of(k, nB, T);
            if (c != cur) {
                if (cur >= 0) { tx = tx + ax; ty = ty + ay; tz = tz + az; }
                ax = ay = az = 0.0;
                cur = c;
            }
            // private partial of the thread owning bond k (:56-63)
            if (v & 1) { ax = ax - fX[k]; ay = ay - fY[k]; az = az - fZ[k]; }
            else       { ax = ax + fX[k]; ay = ay + fY[k]; az = az + fZ[k]; }
        }
        if (cur >= 0) { tx = tx + ax; ty = ty + ay; tz = tz + az; }
        F[n] = tx; F[n + nN] = ty; F[n + 2 * nN] = tz;
    }
}

LawScalars scalars_exp(double k, double alpha)
{
    LawScalars P{};
    P.k = k;
    P.alpha = alpha;
    P.exp_den = 1 - std::exp(-k);   // glibc exp, as the reference computes it
    return P;
}

LawScalars scalars_tri(double s0, double s1, double sc)
{
    LawScalars P{};
    P.s0 = s0; P.s1 = s1; P.sc = sc;
    P.beta = 0.25;
    double eta = s1 / s0;
    P.tri_c1 = (eta - P.beta) / (eta - 1);
    P.tri_c2 = (1 - P.beta) / (eta - 1);
    return P;
}

int launch_check()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return BBPD_OK;
}

}  // namespace

struct bbpd_nodal_plan {
    int64_t nB, nN;
    int T;
    int64_t *rp = nullptr;   // nN + 1
    int64_t *ent = nullptr;  // 2 nB
};

// ---- device-pointer entry points ----

extern "C" int bbpd_dev_calculatedeformedlength(const double *x, const double *bl,
        const double *L0, int64_t nB, int64_t nN, double *L, double *dX, double *dY,
        double *dZ, double *s, void *stream)
{
    if (nB < 0 || nN < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    k_deformedlength<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(x, bl, L0, nB, nN, L, dX, dY, dZ, s);
    return launch_check();
}

extern "C" int bbpd_dev_calculatebsfexponential(const double *s, const double *s0,
        const double *sc, double k, double alpha, double *bsf, double *BSF,
        const double *BT, double *flag, int64_t nB, void *stream)
{
    if (nB < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    k_bsfexponential<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(s, s0, sc, scalars_exp(k, alpha), bsf, BSF, BT, flag, nB);
    return launch_check();
}

extern "C" int bbpd_dev_calculatebsftrilinear(const double *s, double s0, double s1,
        double sc, double *BSF, const double *BT, double *flag, int64_t nB, void *stream)
{
    if (nB < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    k_bsftrilinear<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(s, scalars_tri(s0, s1, sc), BSF, BT, flag, nB);
    return launch_check();
}

extern "C" int bbpd_dev_calculatebondsofteningfactor(const double *s, double s0,
        double sc, double *flag, double *BSF, const double *BT, int64_t nB, void *stream)
{
    if (nB < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    LawScalars P{};
    P.s0 = s0; P.sc = sc;
    k_bilinear<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(s, P, flag, BSF, BT, nB);
    return launch_check();
}

extern "C" int bbpd_dev_calculatebondfailure(double *fail_, double ff, const double *BT,
        const double *s, double csc, double css, int64_t nB, void *stream)
{
    if (nB < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    LawScalars P{};
    P.sc = csc; P.sc_steel = css; P.ff = ff;
    k_bondfailure<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(fail_, P, BT, s, nB);
    return launch_check();
}

extern "C" int bbpd_dev_calculatedamage(const double *bl, const double *fail_, const double *nfam,
        int64_t nB, int64_t nN, double *damage, void *stream)
{
    if (nB < 0 || nN < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nN == 0) return BBPD_OK;
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    int *bad = nullptr;
    BBPD_CUDA_TRY(cudaMallocAsync(&bad, sizeof(int), st));
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(damage, 0, sizeof(double) * (size_t)nN, st);
    if (e == cudaSuccess && nB > 0) {
        k_damage_count<<<blocks_for(nB), kThreads, 0, st>>>(bl, fail_, nB, nN, damage, bad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_damage_final<<<blocks_for(nN), kThreads, 0, st>>>(nfam, nN, damage);
        e = cudaGetLastError();
    }
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(bad, st);
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "damage: %s", cudaGetErrorString(e));
    if (h) return fail(BBPD_ERR_ARG, "BONDLIST holds node ids outside [1, nNodes]");
    return BBPD_OK;
}

extern "C" int bbpd_dev_calculatedamageenergy(const double *BS, const double *s0, const double *sc,
        const double *L0, const double *stretch, double k, double alpha, double cellVolume,
        double *damageEnergy, int64_t nB, void *stream)
{
    if (nB < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    int rc = require_device();
    if (rc) return rc;
    const double ek = std::exp(k);
    const double den = 2 * k * (ek - 1) * (1 + alpha);
    const double shape = (2 * k) - (2 * ek) + (alpha * k) - (alpha * k * ek) + 2;
    k_damageenergy<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(BS, s0, sc, L0, stretch, shape, den,
                                                                        cellVolume * cellVolume, damageEnergy, nB);
    return launch_check();
}

extern "C" int bbpd_dev_calculatebondforces(double *fX, double *fY, double *fZ,
        const double *fail_, const double *dX, const double *dY, const double *dZ,
        const double *L, const double *s, const double *sp, const double *BS, double V,
        const double *VCF, const double *BSF, int64_t nB, void *stream)
{
    if (nB < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nB == 0) return BBPD_OK;
    k_bondforces<<<blocks_for(nB), kThreads, 0, as_stream(stream)>>>(fX, fY, fZ, fail_, dX, dY, dZ, L, s, sp, BS, V, VCF, BSF, nB);
    return launch_check();
}

extern "C" int bbpd_dev_timeintegrationeulercromer(double *a, const double *F, double D,
        double *v, const double *rho, const double *CF, double dt, double *u, double *x,
        const double *X, int64_t nN, int NOD, void *stream)
{
    if (nN < 0 || NOD < 1 || NOD > 3) return fail(BBPD_ERR_ARG, "bad size");
    if (nN == 0) return BBPD_OK;
    k_eulercromer<<<blocks_for(nN), kThreads, 0, as_stream(stream)>>>(a, F, D, v, rho, CF, dt, u, x, X, nN, NOD);
    return launch_check();
}

extern "C" int bbpd_dev_timeintegrationADR(int64_t it, double dt, double *vh, const double *F,
        const double *m, double cn, const double *vhp, double *u, const double *CF,
        int64_t nN, void *stream)
{
    if (nN < 0) return fail(BBPD_ERR_ARG, "negative size");
    if (nN == 0) return BBPD_OK;
    k_adr<<<blocks_for(nN), kThreads, 0, as_stream(stream)>>>(it, dt, vh, F, m, cn, vhp, u, CF, nN);
    return launch_check();
}

extern "C" int bbpd_dev_calculatedampingcoefficient(const double *F, const double *m,
        const double *Fp, double dt, const double *vhp, const double *u, int64_t nN,
        double *cn, void *stream)
{
    if (nN < 0 || !cn) return fail(BBPD_ERR_ARG, "bad argument");
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    int64_t nsl = (nN + 31) / 32;
    const int64_t lv = 2 * ((nsl + 31) / 32) + 2;   // one level of the tree, both sums
    double *scratch = nullptr;   // 2 * nsl slice partials, 2 level buffers, 1 result
    BBPD_CUDA_TRY(cudaMallocAsync(&scratch, sizeof(double) * (size_t)(2 * nsl + 2 * lv + 1), st));
    double *res = scratch + 2 * nsl + 2 * lv;
    if (nsl > 0)
        k_damping_slices<<<blocks_for(nsl * 32), kThreads, 0, st>>>(F, m, Fp, dt, vhp, u, nN, nsl, scratch);
    k_damping_final<<<1, 1024, 0, st>>>(scratch, nsl, scratch + 2 * nsl, scratch + 2 * nsl + lv, res);
    rc = launch_check();
    double h = 0;
    if (rc == BBPD_OK) {
        cudaError_t e = cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(BBPD_ERR_CUDA, "damping coefficient: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(scratch, st);
    if (rc == BBPD_OK) *cn = h;
    return rc;
}

extern "C" int bbpd_nodal_plan_create(const double *bl, int64_t nB, int64_t nN, int nChunks,
                                      void *stream, bbpd_nodal_plan **out)
{
    if (!out || nB < 0 || nN < 0 || nChunks < 1 || nN >= (int64_t)1 << 31)
        return fail(BBPD_ERR_ARG, "bad plan arguments");
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    auto *p = new bbpd_nodal_plan;
    p->nB = nB; p->nN = nN; p->T = nChunks;
    int64_t ne = 2 * nB;
    int32_t *keys = nullptr, *keys2 = nullptr, *cnt = nullptr;
    int64_t *vals = nullptr;
    int *bad = nullptr;
    void *tmp = nullptr;
    size_t tmpb = 0, tmpb2 = 0;
    cudaError_t e = cudaSuccess;
#define PLAN_TRY(x) do { e = (x); if (e != cudaSuccess) goto fail_; } while (0)
    PLAN_TRY(cudaMalloc(&p->rp, sizeof(int64_t) * (size_t)(nN + 1)));
    PLAN_TRY(cudaMalloc(&p->ent, sizeof(int64_t) * (size_t)(ne > 0 ? ne : 1)));
    PLAN_TRY(cudaMalloc(&cnt, sizeof(int32_t) * (size_t)(nN + 1)));
    PLAN_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nN + 1), st));
    PLAN_TRY(cudaMalloc(&bad, sizeof(int)));
    PLAN_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    if (ne > 0) {
        PLAN_TRY(cudaMalloc(&keys, sizeof(int32_t) * (size_t)ne));
        PLAN_TRY(cudaMalloc(&keys2, sizeof(int32_t) * (size_t)ne));
        PLAN_TRY(cudaMalloc(&vals, sizeof(int64_t) * (size_t)ne));
        k_plan_keys<<<blocks_for(nB), kThreads, 0, st>>>(bl, nB, nN, keys, vals, bad);
        // stable radix sort by node keeps each node's entries in bond order
        PLAN_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys, keys2, vals, p->ent, ne, 0, 32, st));
        PLAN_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmpb2, cnt, cnt, nN + 1, st));
        if (tmpb2 > tmpb) tmpb = tmpb2;
        PLAN_TRY(cudaMalloc(&tmp, tmpb));
        PLAN_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmpb, keys, keys2, vals, p->ent, ne, 0, 32, st));
        k_plan_count<<<blocks_for(ne), kThreads, 0, st>>>(keys, ne, cnt);
    }
    {
        // row pointers: exclusive scan of the counts (64-bit)
        std::vector<int32_t> hc((size_t)nN + 1);
        PLAN_TRY(cudaMemcpyAsync(hc.data(), cnt, sizeof(int32_t) * (size_t)(nN + 1), cudaMemcpyDeviceToHost, st));
        int hbad = 0;
        PLAN_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
        PLAN_TRY(cudaStreamSynchronize(st));
        if (hbad) {
            cudaFree(keys); cudaFree(keys2); cudaFree(vals); cudaFree(cnt); cudaFree(bad); cudaFree(tmp);
            bbpd_nodal_plan_destroy(p);
            return fail(BBPD_ERR_ARG, "BONDLIST holds a node id that is not an integer in [1, nNodes] or a self-bond");
        }
        std::vector<int64_t> hr((size_t)nN + 1);
        int64_t acc = 0;
        for (int64_t i = 0; i < nN; i++) { hr[i] = acc; acc += hc[i]; }
        hr[nN] = acc;
        PLAN_TRY(cudaMemcpyAsync(p->rp, hr.data(), sizeof(int64_t) * (size_t)(nN + 1), cudaMemcpyHostToDevice, st));
        PLAN_TRY(cudaStreamSynchronize(st));
    }
    cudaFree(keys); cudaFree(keys2); cudaFree(vals); cudaFree(cnt); cudaFree(bad); cudaFree(tmp);
    *out = p;
    return BBPD_OK;
fail_:
    cudaFree(keys); cudaFree(keys2); cudaFree(vals); cudaFree(cnt); cudaFree(bad); cudaFree(tmp);
    bbpd_nodal_plan_destroy(p);
    return fail(e == cudaErrorMemoryAllocation ? BBPD_ERR_OOM : BBPD_ERR_CUDA, "nodal plan: %s",
                cudaGetErrorString(e));
#undef PLAN_TRY
}

extern "C" int bbpd_nodal_plan_destroy(bbpd_nodal_plan *p)
{
    if (!p) return BBPD_OK;
    cudaFree(p->rp);
    cudaFree(p->ent);
    delete p;
    return BBPD_OK;
}

extern "C" int bbpd_dev_calculatenodalforces(const bbpd_nodal_plan *p, double *F,
        const double *fX, const double *fY, const double *fZ, void *stream)
{
    if (!p) return fail(BBPD_ERR_ARG, "null plan");
    if (p->nN == 0) return BBPD_OK;
    k_nodalforces<<<blocks_for(p->nN), kThreads, 0, as_stream(stream)>>>(p->rp, p->ent, p->nB, p->nN, p->T, F, fX, fY, fZ);
    return launch_check();
}

// ---- host-pointer variants: device mirrors keyed by host address ----

namespace {

struct Mirror { void *dev; size_t bytes; };
std::mutex g_mu;
std::unordered_map<const void *, Mirror> g_mirrors;

struct Plans {
    const void *host_bl = nullptr;
    int64_t nB = -1, nN = -1;
    int T = 0;
    uint64_t hash = 0;
    bbpd_nodal_plan *plan = nullptr;
} g_plan;

// Device buffer mirroring a host buffer of `bytes`; uploaded if `in`.
int mirror(const void *h, size_t bytes, bool in, double **d)
{
    if (!h) { *d = nullptr; return BBPD_OK; }
    auto it = g_mirrors.find(h);
    if (it == g_mirrors.end() || it->second.bytes < bytes) {
        if (it != g_mirrors.end()) { cudaFree(it->second.dev); g_mirrors.erase(it); }
        void *p = nullptr;
        BBPD_CUDA_TRY(cudaMalloc(&p, bytes > 0 ? bytes : 8));
        g_mirrors[h] = Mirror{p, bytes};
        it = g_mirrors.find(h);
    }
    *d = (double *)it->second.dev;
    if (in && bytes) return staging::upload_copy((char *)*d, (const char *)h, (int64_t)bytes, 0);
    return BBPD_OK;
}

int download(void *h, const double *d, size_t bytes)
{
    if (bytes) return staging::download_copy((char *)h, (const char *)d, (int64_t)bytes, 0);
    return BBPD_OK;
}

int finish()
{
    BBPD_CUDA_TRY(cudaDeviceSynchronize());
    return BBPD_OK;
}

uint64_t fnv1a(const void *p, size_t n)
{
    const uint64_t *w = (const uint64_t *)p;
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n / 8; i++) { h ^= w[i]; h *= 1099511628211ull; }
    return h;
}

}  // namespace

#define MIRROR_IN(h, n, d) do { int r_ = mirror((h), (n), true, &(d)); if (r_) return r_; } while (0)
#define MIRROR_OUT(h, n, d) do { int r_ = mirror((h), (n), false, &(d)); if (r_) return r_; } while (0)
#define TRY(x) do { int r_ = (x); if (r_) return r_; } while (0)

extern "C" int bbpd_release_mirrors(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &kv : g_mirrors) cudaFree(kv.second.dev);
    g_mirrors.clear();
    if (g_plan.plan) bbpd_nodal_plan_destroy(g_plan.plan);
    g_plan = Plans{};
    return BBPD_OK;
}

extern "C" int bbpd_calculatedeformedlength(const double *x, const double *bl, const double *L0,
        int64_t nB, int64_t nN, double *L, double *dX, double *dY, double *dZ, double *s)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *dx_, *dbl, *dL0, *dL, *ddX, *ddY, *ddZ, *ds;
    MIRROR_IN(x, sizeof(double) * 3 * (size_t)nN, dx_);
    MIRROR_IN(bl, 2 * b, dbl);
    MIRROR_IN(L0, b, dL0);
    MIRROR_OUT(L, b, dL); MIRROR_OUT(dX, b, ddX); MIRROR_OUT(dY, b, ddY); MIRROR_OUT(dZ, b, ddZ);
    MIRROR_OUT(s, b, ds);
    TRY(bbpd_dev_calculatedeformedlength(dx_, dbl, dL0, nB, nN, dL, ddX, ddY, ddZ, ds, nullptr));
    TRY(finish());
    TRY(download(L, dL, b)); TRY(download(dX, ddX, b)); TRY(download(dY, ddY, b));
    TRY(download(dZ, ddZ, b)); TRY(download(s, ds, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatebsfexponential(const double *s, const double *s0, const double *sc,
        double k, double alpha, double *bsf, double *BSF, const double *BT, double *flag, int64_t nB)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *ds, *ds0, *dsc, *dbsf, *dB, *dBT, *dfl;
    MIRROR_IN(s, b, ds); MIRROR_IN(s0, b, ds0); MIRROR_IN(sc, b, dsc);
    MIRROR_IN(bsf, b, dbsf); MIRROR_IN(BSF, b, dB); MIRROR_IN(BT, b, dBT); MIRROR_IN(flag, b, dfl);
    TRY(bbpd_dev_calculatebsfexponential(ds, ds0, dsc, k, alpha, dbsf, dB, dBT, dfl, nB, nullptr));
    TRY(finish());
    TRY(download(bsf, dbsf, b)); TRY(download(BSF, dB, b)); TRY(download(flag, dfl, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatebsftrilinear(const double *s, double s0, double s1, double sc,
        double *BSF, const double *BT, double *flag, int64_t nB)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *ds, *dB, *dBT, *dfl;
    MIRROR_IN(s, b, ds); MIRROR_IN(BSF, b, dB); MIRROR_IN(BT, b, dBT); MIRROR_IN(flag, b, dfl);
    TRY(bbpd_dev_calculatebsftrilinear(ds, s0, s1, sc, dB, dBT, dfl, nB, nullptr));
    TRY(finish());
    TRY(download(BSF, dB, b)); TRY(download(flag, dfl, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatebondsofteningfactor(const double *s, double s0, double sc,
        double *flag, double *BSF, const double *BT, int64_t nB)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *ds, *dB, *dBT, *dfl;
    MIRROR_IN(s, b, ds); MIRROR_IN(BSF, b, dB); MIRROR_IN(BT, b, dBT); MIRROR_IN(flag, b, dfl);
    TRY(bbpd_dev_calculatebondsofteningfactor(ds, s0, sc, dfl, dB, dBT, nB, nullptr));
    TRY(finish());
    TRY(download(BSF, dB, b)); TRY(download(flag, dfl, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatebondfailure(double *fail_, double ff, const double *BT,
        const double *s, double csc, double css, int64_t nB)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *df, *dBT, *ds;
    MIRROR_IN(fail_, b, df); MIRROR_IN(BT, b, dBT); MIRROR_IN(s, b, ds);
    TRY(bbpd_dev_calculatebondfailure(df, ff, dBT, ds, csc, css, nB, nullptr));
    TRY(finish());
    TRY(download(fail_, df, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatebondforces(double *fX, double *fY, double *fZ, const double *fail_,
        const double *dX, const double *dY, const double *dZ, const double *L, const double *s,
        const double *sp, const double *BS, double V, const double *VCF, const double *BSF,
        int64_t nB)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *dfX, *dfY, *dfZ, *dfa, *ddX, *ddY, *ddZ, *dL, *ds, *dsp, *dBS, *dV, *dB;
    MIRROR_OUT(fX, b, dfX); MIRROR_OUT(fY, b, dfY); MIRROR_OUT(fZ, b, dfZ);
    MIRROR_IN(fail_, b, dfa); MIRROR_IN(dX, b, ddX); MIRROR_IN(dY, b, ddY); MIRROR_IN(dZ, b, ddZ);
    MIRROR_IN(L, b, dL); MIRROR_IN(s, b, ds); MIRROR_IN(sp, b, dsp); MIRROR_IN(BS, b, dBS);
    MIRROR_IN(VCF, b, dV); MIRROR_IN(BSF, b, dB);
    TRY(bbpd_dev_calculatebondforces(dfX, dfY, dfZ, dfa, ddX, ddY, ddZ, dL, ds, dsp, dBS, V, dV, dB, nB, nullptr));
    TRY(finish());
    TRY(download(fX, dfX, b)); TRY(download(fY, dfY, b)); TRY(download(fZ, dfZ, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatedamage(const double *bl, const double *fail_, const double *nfam,
        int64_t nB, int64_t nN, double *damage)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    const size_t b = sizeof(double) * (size_t)nB, n = sizeof(double) * (size_t)nN;
    double *dbl, *dfa, *dnf, *ddm;
    MIRROR_IN(bl, 2 * b, dbl); MIRROR_IN(fail_, b, dfa); MIRROR_IN(nfam, n, dnf); MIRROR_OUT(damage, n, ddm);
    TRY(bbpd_dev_calculatedamage(dbl, dfa, dnf, nB, nN, ddm, nullptr));
    TRY(finish());
    TRY(download(damage, ddm, n));
    return BBPD_OK;
}

extern "C" int bbpd_calculatedamageenergy(const double *BS, const double *s0, const double *sc,
        const double *L0, const double *stretch, double k, double alpha, double cellVolume,
        double *damageEnergy, int64_t nB)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    const size_t b = sizeof(double) * (size_t)nB;
    double *dBS, *ds0, *dsc, *dL, *ds, *dE;
    MIRROR_IN(BS, b, dBS); MIRROR_IN(s0, b, ds0); MIRROR_IN(sc, b, dsc); MIRROR_IN(L0, b, dL);
    MIRROR_IN(stretch, b, ds); MIRROR_IN(damageEnergy, b, dE);
    TRY(bbpd_dev_calculatedamageenergy(dBS, ds0, dsc, dL, ds, k, alpha, cellVolume, dE, nB, nullptr));
    TRY(finish());
    TRY(download(damageEnergy, dE, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatenodalforces(const double *bl, int64_t nB, int64_t nN, double *F,
        const double *fX, const double *fY, const double *fZ, int nChunks)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nB;
    double *dbl, *dF, *dfX, *dfY, *dfZ;
    MIRROR_IN(bl, 2 * b, dbl);
    uint64_t h = fnv1a(bl, 2 * b);
    if (!g_plan.plan || g_plan.host_bl != bl || g_plan.nB != nB || g_plan.nN != nN ||
        g_plan.T != nChunks || g_plan.hash != h) {
        if (g_plan.plan) bbpd_nodal_plan_destroy(g_plan.plan);
        g_plan = Plans{};
        TRY(bbpd_nodal_plan_create(dbl, nB, nN, nChunks, nullptr, &g_plan.plan));
        g_plan.host_bl = bl; g_plan.nB = nB; g_plan.nN = nN; g_plan.T = nChunks; g_plan.hash = h;
    }
    MIRROR_IN(F, sizeof(double) * 3 * (size_t)nN, dF);
    MIRROR_IN(fX, b, dfX); MIRROR_IN(fY, b, dfY); MIRROR_IN(fZ, b, dfZ);
    TRY(bbpd_dev_calculatenodalforces(g_plan.plan, dF, dfX, dfY, dfZ, nullptr));
    TRY(finish());
    TRY(download(F, dF, sizeof(double) * 3 * (size_t)nN));
    return BBPD_OK;
}

extern "C" int bbpd_timeintegrationeulercromer(double *a, const double *F, double D, double *v,
        const double *rho, const double *CF, double dt, double *u, double *x, const double *X,
        int64_t nN, int NOD)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * (size_t)nN * (size_t)(NOD > 0 ? NOD : 0);
    double *da, *dF, *dv, *drho, *dCF, *du, *dx_, *dX;
    MIRROR_OUT(a, b, da); MIRROR_IN(F, b, dF); MIRROR_IN(v, b, dv);
    MIRROR_IN(rho, sizeof(double) * (size_t)nN, drho); MIRROR_IN(CF, b, dCF);
    MIRROR_IN(u, b, du); MIRROR_OUT(x, b, dx_); MIRROR_IN(X, b, dX);
    TRY(bbpd_dev_timeintegrationeulercromer(da, dF, D, dv, drho, dCF, dt, du, dx_, dX, nN, NOD, nullptr));
    TRY(finish());
    TRY(download(a, da, b)); TRY(download(v, dv, b)); TRY(download(u, du, b)); TRY(download(x, dx_, b));
    return BBPD_OK;
}

extern "C" int bbpd_timeintegrationADR(int64_t it, double dt, double *vh, const double *F,
        const double *m, double cn, const double *vhp, double *u, const double *CF, int64_t nN)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * 3 * (size_t)nN;
    double *dvh, *dF, *dm, *dvhp, *du, *dCF;
    bool alias = (vh == vhp);
    MIRROR_IN(vh, b, dvh); MIRROR_IN(F, b, dF); MIRROR_IN(m, sizeof(double) * (size_t)nN, dm);
    if (alias) dvhp = dvh; else MIRROR_IN(vhp, b, dvhp);
    MIRROR_IN(u, b, du); MIRROR_IN(CF, b, dCF);
    TRY(bbpd_dev_timeintegrationADR(it, dt, dvh, dF, dm, cn, dvhp, du, dCF, nN, nullptr));
    TRY(finish());
    TRY(download(vh, dvh, b)); TRY(download(u, du, b));
    return BBPD_OK;
}

extern "C" int bbpd_calculatedampingcoefficient(const double *F, const double *m, const double *Fp,
        double dt, const double *vhp, const double *u, int64_t nN, double *cn)
{
    TRY(require_device());
    std::lock_guard<std::mutex> lk(g_mu);
    size_t b = sizeof(double) * 3 * (size_t)nN;
    double *dF, *dm, *dFp, *dvhp, *du;
    MIRROR_IN(F, b, dF); MIRROR_IN(m, sizeof(double) * (size_t)nN, dm); MIRROR_IN(Fp, b, dFp);
    MIRROR_IN(vhp, b, dvhp); MIRROR_IN(u, b, du);
    return bbpd_dev_calculatedampingcoefficient(dF, dm, dFp, dt, dvhp, du, nN, cn, nullptr);
}
