// Device arithmetic of one bond, shared by the per-routine kernels and the
// fused time-step kernel. Every expression keeps the reference's operation
// order; the translation units that include this file are compiled with
// -fmad=false, so no multiply-add is fused and each double operation rounds
// exactly as the reference MEX code does on x86-64. CUDA's double-precision
// `/` and sqrt() are IEEE correctly rounded, like the host's.
#pragma once

#include <cstdint>

#include "crexp.cuh"

namespace bbpd {

// Law parameters that are scalars in the reference calls.
struct LawScalars {
    double s0, s1, sc;     // stretches when no per-bond array is given
    double beta;           // trilinear beta (calculatebsftrilinear.m:41)
    double tri_c1, tri_c2; // (eta-beta)/(eta-1), (1-beta)/(eta-1) for scalar s0/s1
    double k, alpha;       // exponential law
    double exp_den;        // 1 - exp(-k), computed once (calculatebsfexponentialMex.c:45)
    double sc_steel;       // brittle law, steel bonds
    double ff;             // failureFunctionality (0 or 1)
};

// Deformed bond vector, length and stretch: calculatedeformedlengthMex.c:37-43.
__device__ __forceinline__ void bond_kinematics(double xi, double yi, double zi,
                                                double xj, double yj, double zj,
                                                double l0, double &dX, double &dY,
                                                double &dZ, double &L, double &s)
{
    dX = xj - xi;
    dY = yj - yi;
    dZ = zj - zi;
    L = sqrt(dX * dX + dY * dY + dZ * dZ);
    s = (L - l0) / l0;
}

// Trilinear softening, calculatebsftrilinear.m:82-104 and :112 for one bond.
// eta-derived constants come precomputed when s0/s1 are scalars (percb=false).
__device__ __forceinline__ void law_trilinear(double s, double s0, double s1, double sc,
                                              const LawScalars &P, bool percb,
                                              bool concrete, double &BSF, bool &flag)
{
    double bsf = 0;
    if (concrete) {
        if (s > s0 && s <= s1) {
            double c1, c2;
            if (percb) {
                double eta = s1 / s0;
                c1 = (eta - P.beta) / (eta - 1);
                c2 = (1 - P.beta) / (eta - 1);
            } else {
                c1 = P.tri_c1;
                c2 = P.tri_c2;
            }
            bsf = 1 - (c1 * (s0 / s)) + c2;
            flag = true;
        } else if (s > s1 && s <= sc) {
            bsf = 1 - ((s0 * P.beta) / s) * ((sc - s) / (sc - s1));
        } else if (s > sc) {
            bsf = 1;
        }
        if (bsf > BSF) BSF = bsf;
    }
    if (isnan(BSF)) BSF = 0;
}

// MATLAB max(a, b) on scalars (NaN operands ignored).
__device__ __forceinline__ double matlab_max(double a, double b)
{
    if (isnan(b)) return a;
    if (isnan(a)) return b;
    return (b > a) ? b : a;
}

// Bilinear softening, calculatebondsofteningfactor.m:42-48 for one bond.
__device__ __forceinline__ void law_bilinear(double s, double s0, double sc,
                                             bool concrete, double &BSF, bool &flag)
{
    if (concrete && s > s0) flag = true;
    double bsf = ((s - s0) / s) * (sc / (sc - s0));
    BSF = matlab_max(BSF, bsf * (flag ? 1.0 : 0.0));
    if (BSF > 1) BSF = 1;
    if (isnan(BSF)) BSF = 0;
}

// Decaying-exponential softening, calculatebsfexponentialMex.c:36-58. bsf is the
// per-step scratch value, zero when no branch assigns it (solver :86).
__device__ __forceinline__ void law_exponential(double s, double s0, double sc,
                                                const LawScalars &P, bool concrete,
                                                double &BSF, bool &flag)
{
    if (!concrete) return;
    double bsf = 0.0;
    if (s0 < s && s <= sc) {
        flag = true;
        // exp correctly rounded (crexp.cuh); glibc's exp agrees on all but
        // about 8 in 10^4 arguments of the law's range
        double numerator = 1 - cr_exp(-P.k * (s - s0) / (sc - s0));
        double residual = P.alpha * (1 - (s - s0) / (sc - s0));
        bsf = 1 - (s0 / s) * ((1 - (numerator / P.exp_den)) + residual) / (1 + P.alpha);
    } else if (s > sc) {
        bsf = 1;
    }
    if (bsf > BSF) BSF = bsf;
    if (BSF > 1) BSF = 1;
    if (BSF != BSF) BSF = 0.0;
}

// Brittle failure, calculatebondfailureMex.c:36-38 (fail is 1 or ff).
__device__ __forceinline__ void law_linear(double s, double sc, const LawScalars &P,
                                           int bt, double &fail)
{
    if (fail == 1 && bt == 0 && s > sc) fail = P.ff;
    if (fail == 1 && bt == 1 && s > 3 * sc) fail = P.ff;
    if (fail == 1 && bt == 2 && s > P.sc_steel) fail = P.ff;
}

// Scalar part of the bond force, calculatebondforcesMex.c:34 read left to right:
// fail * BONDSTIFFNESS * (1 - BSF) * (stretch - stretchPlastic) * cellVolume * VCF.
__device__ __forceinline__ double bond_force_scalar(double fail, double bs, double BSF,
                                                    double s, double sp, double V,
                                                    double vcf)
{
    return fail * bs * (1 - BSF) * (s - sp) * V * vcf;
}

// One component: scalar * (d / L), NaN replaced by 0 (calculatebondforcesMex.c:34-40).
__device__ __forceinline__ double bond_force_component(double t, double d, double L)
{
    double f = t * (d / L);
    if (f != f) f = 0.0;
    return f;
}

// libgomp static schedule without chunk size: n iterations over T threads,
// q = n / T each and the first n % T threads one more. Chunk of iteration k.
__device__ __forceinline__ int omp_chunk_of(int64_t k, int64_t n, int T)
{
    int64_t q = n / T, r = n % T;
    int64_t big = r * (q + 1);
    if (k < big) return (int)(k / (q + 1));
    return (int)(r + (k - big) / q);
}

}  // namespace bbpd
