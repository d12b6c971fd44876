// Test harness: the device's correctly rounded exp (bb_pd_b200/csrc/crexp.cuh)
// compiled for the host, beside glibc's exp, for tests/test_crexp.py and the
// device comparison in tests/test_gpu_routines.py.
#include <cmath>
#include <cstdint>

#include "crexp.cuh"

namespace {
// splitmix64: uniform doubles in [lo, hi) from a counter (the device
// self-test draws the same samples)
inline double sample(uint64_t seed, uint64_t i, double lo, double hi)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return lo + (hi - lo) * ((double)(z >> 11) * 0x1p-53);
}
inline uint64_t bits(double d)
{
    uint64_t u;
    __builtin_memcpy(&u, &d, 8);
    return u;
}
}  // namespace

extern "C" {

void crexp_many(const double *x, double *y, long n)
{
    for (long i = 0; i < n; i++) y[i] = bbpd::cr_exp(x[i]);
}

void crexp_accurate_many(const double *x, double *y, long n)
{
    for (long i = 0; i < n; i++) {
        const double m = ::rint(x[i] * bbpd::crexp_tab::INV_LN2_N);
        y[i] = bbpd::crexp_detail::accurate(x[i], (int)m);
    }
}

void glibc_exp_many(const double *x, double *y, long n)
{
    for (long i = 0; i < n; i++) y[i] = std::exp(x[i]);
}

// n samples uniform in [lo, hi): counts of results that differ from glibc's
// exp (and by more than one unit in the last place), and of fast-step results
// that differ from the accurate step's.
void crexp_survey(double lo, double hi, long n, uint64_t seed, long *diff_glibc, long *diff_glibc_gt1ulp,
                  long *diff_accurate)
{
    long dg = 0, dg1 = 0, da = 0;
#pragma omp parallel for reduction(+ : dg, dg1, da) schedule(static)
    for (long i = 0; i < n; i++) {
        const double x = sample(seed, (uint64_t)i, lo, hi);
        const double c = bbpd::cr_exp(x), g = std::exp(x);
        if (bits(c) != bits(g)) {
            dg++;
            const int64_t d = (int64_t)bits(c) - (int64_t)bits(g);
            if (d > 1 || d < -1) dg1++;
        }
        if (::fabs(x) >= 0x1p-60) {
            const double m = ::rint(x * bbpd::crexp_tab::INV_LN2_N);
            if (bits(bbpd::crexp_detail::accurate(x, (int)m)) != bits(c)) da++;
        }
    }
    *diff_glibc = dg;
    *diff_glibc_gt1ulp = dg1;
    *diff_accurate = da;
}

// Sum (mod 2^64) of the bit patterns of cr_exp over the same samples as the
// device self-test bbpd_selftest_exp.
uint64_t crexp_bits_sum(double lo, double hi, long n, uint64_t seed)
{
    uint64_t sum = 0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
    for (long i = 0; i < n; i++) sum += bits(bbpd::cr_exp(sample(seed, (uint64_t)i, lo, hi)));
    return sum;
}

}  // extern "C"
