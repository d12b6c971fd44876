// Device self-tests of the arithmetic the kernels rely on.
#include "bbpd_internal.h"
#include "crexp.cuh"
#include "divide.cuh"

#include <algorithm>
#include <cstring>

using namespace bbpd;

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// double with random significand and the given unbiased exponent
__device__ __forceinline__ double make_double(uint64_t h, int e)
{
    const uint64_t bits = ((uint64_t)(e + 1023) << 52) | (h & 0x000FFFFFFFFFFFFFull);
    return __longlong_as_double((long long)bits);
}

struct Counts {
    unsigned long long recip_bad, quot_bad, skipped, samples;
    unsigned long long rcp_err_bits;  // max |rcp.approx - 1/b| / (1/b), as ordered bits
};

// Divisors over [2^-100, 2^100] (and often near the bond lengths of a beam);
// numerators zero, exact multiples, random and close to rounding midpoints.
__global__ void division_selftest_kernel(int64_t n, uint64_t seed, Counts *c)
{
    unsigned long long rb = 0, qb = 0, sk = 0, cnt = 0;
    double maxerr = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t h1 = mix64(seed ^ (uint64_t)t * 0xD1B54A32D192ED03ull);
        const uint64_t h2 = mix64(h1), h3 = mix64(h2), h4 = mix64(h3);
        int eb = (h1 >> 60) < 10 ? (int)((h2 >> 55) % 31) - 20   // 2^-20 .. 2^10
                                 : (int)((h2 >> 55) % 201) - 100; // 2^-100 .. 2^100
        double b = make_double(h3, eb);
        if ((h1 & 0xFF) == 7) b = make_double(0xFFFFFFFFFFFFFull, eb);   // all-ones significand
        bool ok;
        const double y = recip_rn(b, ok);
        const double ya = rcp_approx(b);
        const double rel = fabs(ya * b - 1.0);
        maxerr = fmax(maxerr, rel);
        if (!ok) { sk++; continue; }
        cnt++;
        if (__double_as_longlong(y) != __double_as_longlong(1.0 / b)) rb++;
        double a;
        const int kind = (int)((h1 >> 8) & 7);
        const int ea = eb + (int)((h4 >> 58) % 9) - 6;   // |a| within 2^-6 .. 2^2 of |b|
        if (kind == 0) a = 0.0;
        else if (kind == 1) a = b * (double)((h4 & 0xFF) + 1);          // exact quotient
        else if (kind <= 4) a = make_double(h4, ea);                    // random
        else {                                                          // near a rounding midpoint
            const double q = make_double(h4, (int)((h2 >> 40) % 9) - 6);
            const double ulp = make_double(0, ((int)((__double_as_longlong(q) >> 52) & 0x7FF) - 1023) - 52);
            a = __fma_rn(q, b, (0.5 * ulp) * b);   // RN((q + ulp/2) b): a / b sits next to a midpoint
        }
        if (((h4 >> 63) & 1) && a != 0.0) a = -a;   // -0 is outside the precondition
        const double q = quot_rn(a, b, y);
        if (__double_as_longlong(q) != __double_as_longlong(a / b)) qb++;
    }
    atomicAdd(&c->recip_bad, rb);
    atomicAdd(&c->quot_bad, qb);
    atomicAdd(&c->skipped, sk);
    atomicAdd(&c->samples, cnt);
    atomicMax(&c->rcp_err_bits, (unsigned long long)__double_as_longlong(maxerr));
}

// Uniform doubles in [lo, hi) from a counter (splitmix64), the sampler of the
// host-side check of the same exp code.
__device__ __forceinline__ double exp_sample(uint64_t seed, uint64_t i, double lo, double hi)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return __dadd_rn(lo, __dmul_rn(__dsub_rn(hi, lo), __dmul_rn((double)(z >> 11), 0x1p-53)));
}

// cr_exp on n samples: results whose fast step differs from the accurate
// step, and the sum (mod 2^64) of the results' bit patterns.
__global__ void exp_selftest_kernel(double lo, double hi, int64_t n, uint64_t seed, unsigned long long *out)
{
    unsigned long long bad = 0, sum = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const double x = exp_sample(seed, (uint64_t)t, lo, hi);
        const double c = cr_exp(x);
        sum += (unsigned long long)__double_as_longlong(c);
        if (fabs(x) >= 0x1p-60 && x >= -745.2 && x <= 709.8) {
            const double a = crexp_detail::accurate(x, (int)rint(x * crexp_tab::INV_LN2_N));
            if (__double_as_longlong(a) != __double_as_longlong(c)) bad++;
        }
    }
    atomicAdd(&out[0], bad);
    atomicAdd(&out[1], sum);
}

// FP64 issue rate: every thread runs 8 independent chains of dependent
// fused multiply-adds (enough to cover the pipe's latency at 8 warps per
// SMSP); the result is written so that nothing is optimised away.
__global__ void fp64_peak_kernel(int64_t iters, double seed, double *out)
{
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + k * 1e-3 + threadIdx.x * 1e-9;
    const double m = 0.999999999, c = 1e-12;
    for (int64_t it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __fma_rn(a[k], m, c);
    }
    double t = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) t += a[k];
    if (t == 42.0) out[0] = t;   // practically never; keeps the chains live
}

}  // namespace

extern "C" int bbpd_selftest_fp64_peak(double seconds_target, double *fma_lanes_per_s)
{
    int rc = require_device();
    if (rc) return rc;
    if (!fma_lanes_per_s || !(seconds_target > 0)) return fail(BBPD_ERR_ARG, "bad argument");
    int nsm = 0, dev = 0;
    BBPD_CUDA_TRY(cudaGetDevice(&dev));
    BBPD_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double *dout = nullptr;
    BBPD_CUDA_TRY(cudaMalloc(&dout, sizeof(double)));
    cudaEvent_t e0, e1;
    BBPD_CUDA_TRY(cudaEventCreate(&e0));
    BBPD_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = nsm * 8, threads = 256;
    int64_t iters = 1 << 14;
    float ms = 0;
    cudaError_t e = cudaSuccess;
    for (int round = 0; round < 6 && e == cudaSuccess; round++) {   // grow until the target time
        cudaEventRecord(e0);
        fp64_peak_kernel<<<blocks, threads>>>(iters, 1.0, dout);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess || ms >= 1e3 * seconds_target) break;
        iters = (int64_t)(iters * std::max(2.0, 1e3 * seconds_target / std::max(ms, 0.01f)));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "fp64 peak: %s", cudaGetErrorString(e));
    *fma_lanes_per_s = (double)blocks * threads * 8.0 * (double)iters / (ms * 1e-3);
    return BBPD_OK;
}

extern "C" int bbpd_selftest_exp(double lo, double hi, int64_t n, uint64_t seed, int64_t *fast_vs_accurate,
                                 uint64_t *bits_sum)
{
    int rc = require_device();
    if (rc) return rc;
    if (n < 0 || !fast_vs_accurate || !bits_sum || !(lo <= hi)) return fail(BBPD_ERR_ARG, "bad argument");
    unsigned long long *dc = nullptr;
    BBPD_CUDA_TRY(cudaMalloc(&dc, 2 * sizeof(unsigned long long)));
    BBPD_CUDA_TRY(cudaMemset(dc, 0, 2 * sizeof(unsigned long long)));
    exp_selftest_kernel<<<148 * 8, 256>>>(lo, hi, n, seed, dc);
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, dc, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(dc);
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "exp selftest: %s", cudaGetErrorString(e));
    *fast_vs_accurate = (int64_t)h[0];
    *bits_sum = (uint64_t)h[1];
    return BBPD_OK;
}

extern "C" int bbpd_selftest_division(int64_t n, uint64_t seed, int64_t *recip_mismatches,
                                      int64_t *quot_mismatches, int64_t *samples,
                                      double *rcp_approx_max_relerr)
{
    int rc = require_device();
    if (rc) return rc;
    if (n < 0 || !recip_mismatches || !quot_mismatches || !samples || !rcp_approx_max_relerr)
        return fail(BBPD_ERR_ARG, "bad argument");
    Counts *dc = nullptr;
    BBPD_CUDA_TRY(cudaMalloc(&dc, sizeof(Counts)));
    BBPD_CUDA_TRY(cudaMemset(dc, 0, sizeof(Counts)));
    division_selftest_kernel<<<148 * 8, 256>>>(n, seed, dc);
    Counts h{};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&h, dc, sizeof(Counts), cudaMemcpyDeviceToHost);
    cudaFree(dc);
    if (e != cudaSuccess) return fail(BBPD_ERR_CUDA, "division selftest: %s", cudaGetErrorString(e));
    *recip_mismatches = (int64_t)h.recip_bad;
    *quot_mismatches = (int64_t)h.quot_bad;
    *samples = (int64_t)h.samples;
    double m;
    std::memcpy(&m, &h.rcp_err_bits, 8);
    *rcp_approx_max_relerr = m;
    return BBPD_OK;
}
