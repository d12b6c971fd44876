// ADR damping coefficient without any device allocation
// (bbpd_dev_calculatedampingcoefficient_noalloc). It computes the same sums as
// bbpd_dev_calculatedampingcoefficient (calculatedampingcoefficient.m:59-112 in
// the fixed 32-ary tree order), but its scratch is a fixed array in this file
// instead of a stream-ordered allocation per call, and the result stays on the
// device. It serves callers that must not allocate device memory per call: a
// time loop that has handed the device's memory to its own fixed pool, or one
// held to a fixed HBM budget, where a per-step allocation could fail or grow
// the pool in the middle of a run.
//
// Limits and rules of use:
//  * at most BBPD_DAMPING_NOALLOC_MAX_NODES nodes (2^24); the scratch holds the
//    level-2 partials of the tree, 2 * 2^14 doubles = 256 KiB per device. Larger
//    inputs are rejected with BBPD_ERR_ARG before anything is launched;
//  * the first call on each device looks up the scratch address with
//    cudaGetSymbolAddress (which may load this library's device code); make that
//    first call before any stream capture;
//  * nothing in the scratch has to start at zero: every call writes each partial
//    before it reads it;
//  * there is one scratch array per device, so calls that overlap on the same
//    device (different streams, or different host threads, with no ordering
//    between them) race on it; order them on one stream or with events.
#include "bbpd_internal.h"

#include <mutex>

using namespace bbpd;

namespace {

constexpr int64_t kMaxNodes = BBPD_DAMPING_NOALLOC_MAX_NODES;
constexpr int64_t kMaxGroups = kMaxNodes / 1024;  // level-2 partials (32 slices of 32 nodes)
constexpr int kMaxDevices = 64;

// Level-2 partials of both sums: [0, m2) for cn1, [m2, 2 m2) for cn2.
static __device__ __align__(256) double g_damping_scratch[2 * kMaxGroups];

std::mutex g_mu;
double *g_scratch[kMaxDevices];  // per-device address of g_damping_scratch, set once

// Levels 1 and 2 of the tree in one pass. Warp w owns group g (slices 32g ..
// 32g+31): for each slice it forms the per-node terms of
// calculatedampingcoefficient.m:61-85 for the slice's 32 nodes (lane = node)
// and folds them with the xor butterfly (offsets 16..1); after the butterfly
// every lane holds the same bits, so lane q keeps slice q's sums. A second
// butterfly folds the group. Missing nodes and slices contribute 0.0, as in the
// allocating routine, so the partials are bit-identical to its level 2.
__global__ void k_damping_groups(const double *__restrict__ F, const double *__restrict__ m,
                                 const double *__restrict__ Fp, double dt,
                                 const double *__restrict__ vhp, const double *__restrict__ u,
                                 int64_t nN, int64_t nsl, int64_t m2, double *part)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = warp; g < m2; g += nwarps) {
        double k1 = 0.0, k2 = 0.0;
        for (int q = 0; q < 32; q++) {
            const int64_t sl = g * 32 + q;
            double c1 = 0, c2 = 0;
            const int64_t i = sl * 32 + lane;
            if (sl < nsl && i < nN) {
                for (int d = 0; d < 3; d++) {
                    const int64_t e = i + nN * d;
                    if (vhp[e] != 0)
                        c1 = c1 - u[e] * u[e] * ((F[e] / m[i] - Fp[e] / m[i]) / (dt * vhp[e]));
                }
                for (int d = 0; d < 3; d++) {
                    const int64_t e = i + nN * d;
                    c2 = c2 + u[e] * u[e];
                }
            }
            for (int off = 16; off >= 1; off >>= 1) {
                c1 = c1 + __shfl_xor_sync(0xffffffffu, c1, off);
                c2 = c2 + __shfl_xor_sync(0xffffffffu, c2, off);
            }
            if (lane == q) { k1 = c1; k2 = c2; }
        }
        for (int off = 16; off >= 1; off >>= 1) {
            k1 = k1 + __shfl_xor_sync(0xffffffffu, k1, off);
            k2 = k2 + __shfl_xor_sync(0xffffffffu, k2, off);
        }
        if (lane == 0) { part[g] = k1; part[m2 + g] = k2; }
    }
}

// Levels 3 and up (groups of 32 consecutive partials, xor butterfly, missing
// members 0.0) in shared memory, one block of 1024 threads, then the clamp of
// calculatedampingcoefficient.m:90-112; the coefficient goes to cn_out (device).
__global__ void __launch_bounds__(1024) k_damping_top(const double *part, int64_t m2,
                                                      double *cn_out)
{
    __shared__ double sa[2 * (kMaxGroups / 32)], sb[2 * (kMaxGroups / 32)];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double *src = part;
    int64_t cnt = m2, sstride = m2;
    double *dst = sa;
    while (cnt > 1) {
        const int64_t mm = (cnt + 31) / 32;
        for (int64_t g = warp; g < mm; g += 32) {
            const int64_t idx = g * 32 + lane;
            double c1 = idx < cnt ? src[idx] : 0.0, c2 = idx < cnt ? src[sstride + idx] : 0.0;
            for (int off = 16; off >= 1; off >>= 1) {
                c1 = c1 + __shfl_xor_sync(0xffffffffu, c1, off);
                c2 = c2 + __shfl_xor_sync(0xffffffffu, c2, off);
            }
            if (lane == 0) { dst[g] = c1; dst[mm + g] = c2; }
        }
        __syncthreads();
        src = dst;
        sstride = mm;
        cnt = mm;
        dst = (dst == sa) ? sb : sa;
    }
    if (threadIdx.x == 0) {
        const double c1 = m2 > 0 ? src[0] : 0.0, c2 = m2 > 0 ? src[sstride] : 0.0;
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

// Address of this device's scratch; looked up once per device.
int scratch_for_current_device(double **out)
{
    int dev = 0;
    BBPD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(BBPD_ERR_UNSUPPORTED, "device ordinal %d beyond the %d this routine tracks", dev, kMaxDevices);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[dev]) {
        double *p = nullptr;
        BBPD_CUDA_TRY(cudaGetSymbolAddress((void **)&p, g_damping_scratch));
        g_scratch[dev] = p;
    }
    *out = g_scratch[dev];
    return BBPD_OK;
}

}  // namespace

extern "C" int bbpd_dev_calculatedampingcoefficient_noalloc(const double *F, const double *m,
        const double *Fp, double dt, const double *vhp, const double *u, int64_t nN,
        double *cn, void *stream)
{
    if (nN < 0 || !cn) return fail(BBPD_ERR_ARG, "bad argument");
    if (nN > kMaxNodes)
        return fail(BBPD_ERR_ARG,
                    "nNodes = %lld exceeds the %lld-node limit of the no-allocation damping "
                    "coefficient (256 KiB of static scratch); use bbpd_dev_calculatedampingcoefficient",
                    (long long)nN, (long long)kMaxNodes);
    int rc = require_device();
    if (rc) return rc;
    double *part = nullptr;
    rc = scratch_for_current_device(&part);
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    const int64_t nsl = (nN + 31) / 32;
    const int64_t m2 = (nsl + 31) / 32;
    if (m2 > 0) {
        const int64_t threads = 256, blocks = (m2 * 32 + threads - 1) / threads;
        k_damping_groups<<<(unsigned)blocks, (unsigned)threads, 0, st>>>(F, m, Fp, dt, vhp, u, nN, nsl, m2, part);
    }
    k_damping_top<<<1, 1024, 0, st>>>(part, m2, cn);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return BBPD_OK;
}
