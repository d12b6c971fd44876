/*
 * bbpd_oracle.c -- TEST INFRASTRUCTURE ONLY (see bbpd_oracle.h).
 *
 * Plain-C restatement of the BB_PD hot path. Build: oracle/Makefile
 * (-O2 -ffp-contract=off). Every function follows the reference lines cited
 * above it, with the reference's evaluation order kept operation by operation.
 */
#include "bbpd_oracle.h"

#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* calculatedeformedlengthMex.c:27-47 */
void orc_deformedlength(const double *x, const double *bl, const double *L0,
                        int64_t nBonds, int64_t nNodes, double *L,
                        double *dX, double *dY, double *dZ, double *s)
{
    for (int64_t k = 0; k < nBonds; k++) {
        int64_t i = (int64_t)bl[k];           /* BONDLIST(k,1), 1-based */
        int64_t j = (int64_t)bl[nBonds + k];  /* BONDLIST(k,2) */
        dX[k] = x[j - 1] - x[i - 1];
        dY[k] = x[j + nNodes - 1] - x[i + nNodes - 1];
        dZ[k] = x[j + 2 * nNodes - 1] - x[i + 2 * nNodes - 1];
        L[k] = sqrt(dX[k] * dX[k] + dY[k] * dY[k] + dZ[k] * dZ[k]);
        s[k] = (L[k] - L0[k]) / L0[k];
    }
}

/* The exp of the exponential law's numerator: libm's (the reference's
 * call), or, after orc_use_cr_exp(1), a correctly rounded one (the host build
 * of the device's, oracle/crexp_shim.cpp) to tell the device's arithmetic
 * apart from libm's occasional misrounding. */
double orc_cr_exp(double x);
static double (*law_exp)(double) = exp;
void orc_use_cr_exp(int on) { law_exp = on ? orc_cr_exp : exp; }

/* calculatebsfexponentialMex.c:26-66 */
void orc_bsf_exponential(const double *s, const double *s0, int s0_stride,
                         const double *sc, int sc_stride, double k, double alpha,
                         double *bsf, double *BSF, const double *BT,
                         double *flag, int64_t nBonds)
{
    for (int64_t b = 0; b < nBonds; b++) {
        if (BT ? BT[b] == 0 : 1) {
            double s0b = s0[b * s0_stride], scb = sc[b * sc_stride];
            if (s0b < s[b] && s[b] <= scb) {
                flag[b] = 1;
                double numerator = 1 - law_exp(-k * (s[b] - s0b) / (scb - s0b));
                double denominator = 1 - exp(-k);
                double residual = alpha * (1 - (s[b] - s0b) / (scb - s0b));
                bsf[b] = 1 - (s0b / s[b]) * ((1 - (numerator / denominator)) + residual) / (1 + alpha);
            } else if (s[b] > scb) {
                bsf[b] = 1;
            }
            if (bsf[b] > BSF[b]) BSF[b] = bsf[b];
            if (BSF[b] > 1) BSF[b] = 1;
            if (BSF[b] != BSF[b]) BSF[b] = 0.0;
        }
    }
}

/* calculatebsftrilinear.m:40-112 (eta = s1/s0, beta = 0.25 at :41-42; per-bond
 * s1/sc as in the commented variant :46-77) */
void orc_bsf_trilinear(const double *s, const double *s0, int s0_stride,
                       const double *s1, int s1_stride, const double *sc,
                       int sc_stride, double beta, double *BSF, const double *BT,
                       double *flag, int64_t nBonds)
{
    for (int64_t b = 0; b < nBonds; b++) {
        double s0b = s0[b * s0_stride], s1b = s1[b * s1_stride], scb = sc[b * sc_stride];
        double eta = s1b / s0b;
        double bsf = 0;
        if (BT ? BT[b] == 0 : 1) {
            if (s[b] > s0b && s[b] <= s1b) {
                bsf = 1 - ((eta - beta) / (eta - 1) * (s0b / s[b])) + ((1 - beta) / (eta - 1));
                flag[b] = 1;
            } else if (s[b] > s1b && s[b] <= scb) {
                bsf = 1 - ((s0b * beta) / s[b]) * ((scb - s[b]) / (scb - s1b));
            } else if (s[b] > scb) {
                bsf = 1;
            }
            if (bsf > BSF[b]) BSF[b] = bsf;
        }
        if (isnan(BSF[b])) BSF[b] = 0;   /* :112, applied to every bond */
    }
}

/* MATLAB max(a, b) for scalars: NaN operands are ignored. */
static double matlab_max(double a, double b)
{
    if (isnan(b)) return a;
    if (isnan(a)) return b;
    return (b > a) ? b : a;
}

/* calculatebondsofteningfactor.m:42-48 */
void orc_bsf_bilinear(const double *s, const double *s0, int s0_stride,
                      const double *sc, int sc_stride, double *BSF,
                      const double *BT, double *flag, int64_t nBonds)
{
    for (int64_t b = 0; b < nBonds; b++) {
        double s0b = s0[b * s0_stride], scb = sc[b * sc_stride];
        if ((BT ? BT[b] == 0 : 1) && s[b] > s0b) flag[b] = 1;          /* :159 */
        double bsf = ((s[b] - s0b) / s[b]) * (scb / (scb - s0b));        /* :161 */
        BSF[b] = matlab_max(BSF[b], bsf * flag[b]);                      /* :163 */
        if (BSF[b] > 1) BSF[b] = 1;                                      /* :164 */
        if (isnan(BSF[b])) BSF[b] = 0;                                   /* :165 */
    }
}

/* calculatebondfailureMex.c:26-44 */
void orc_bondfailure(double *fail, double failureFunctionality, const double *BT,
                     const double *s, const double *sc, int sc_stride,
                     double scSteel, int64_t nBonds)
{
    for (int64_t b = 0; b < nBonds; b++) {
        double bt = BT ? BT[b] : 0.0, scb = sc[b * sc_stride];
        if (fail[b] == 1 && bt == 0 && s[b] > scb) fail[b] = failureFunctionality;
        if (fail[b] == 1 && bt == 1 && s[b] > 3 * scb) fail[b] = failureFunctionality;
        if (fail[b] == 1 && bt == 2 && s[b] > scSteel) fail[b] = failureFunctionality;
    }
}

/* calculatebondforcesMex.c:26-45 */
void orc_bondforces(double *fX, double *fY, double *fZ, const double *fail,
                    const double *dX, const double *dY, const double *dZ,
                    const double *L, const double *s, const double *sp,
                    const double *BS, double V, const double *VCF,
                    const double *BSF, int64_t nBonds)
{
    for (int64_t k = 0; k < nBonds; k++) {
        double spk = sp ? sp[k] : 0.0;
        fX[k] = fail[k] * BS[k] * (1 - BSF[k]) * (s[k] - spk) * V * VCF[k] * (dX[k] / L[k]);
        fY[k] = fail[k] * BS[k] * (1 - BSF[k]) * (s[k] - spk) * V * VCF[k] * (dY[k] / L[k]);
        fZ[k] = fail[k] * BS[k] * (1 - BSF[k]) * (s[k] - spk) * V * VCF[k] * (dZ[k] / L[k]);
        if (fX[k] != fX[k]) fX[k] = 0.0;
        if (fY[k] != fY[k]) fY[k] = 0.0;
        if (fZ[k] != fZ[k]) fZ[k] = 0.0;
    }
}

/* libgomp's static schedule without a chunk size: q = n / T iterations each,
 * the first n % T threads take one more (checked against libgomp in tests). */
void orc_chunk_range(int64_t n, int nChunks, int c, int64_t *lo, int64_t *hi)
{
    int64_t q = n / nChunks, r = n % nChunks, t = r;
    if (c < r) { t = 0; q++; }
    *lo = q * c + t;
    *hi = *lo + q;
}

static void nodalforces_scratch(int64_t nB, int64_t nN, const double *bl,
                                double *F, const double *fX, const double *fY,
                                const double *fZ, double *nfX, double *nfY,
                                double *nfZ, int nChunks)
{
    /* calculatenodalforcesopenmpMex.c:50-66: private partial per thread */
    for (int c = 0; c < nChunks; c++) {
        int64_t lo, hi;
        orc_chunk_range(nB, nChunks, c, &lo, &hi);
        for (int64_t k = lo; k < hi; k++) {
            int64_t i = (int64_t)bl[k], j = (int64_t)bl[nB + k];
            nfX[(i - 1) + nN * c] += fX[k];
            nfX[(j - 1) + nN * c] -= fX[k];
            nfY[(i - 1) + nN * c] += fY[k];
            nfY[(j - 1) + nN * c] -= fY[k];
            nfZ[(i - 1) + nN * c] += fZ[k];
            nfZ[(j - 1) + nN * c] -= fZ[k];
        }
    }
    /* :69-81: per-node sum over threads in thread order */
    for (int64_t n = 0; n < nN; n++) {
        for (int c = 0; c < nChunks; c++) {
            F[n] += nfX[n + nN * c];
            F[n + nN] += nfY[n + nN * c];
            F[n + 2 * nN] += nfZ[n + nN * c];
        }
    }
}

void orc_nodalforces_chunked(int64_t nBonds, int64_t nNodes, const double *bl,
                             double *F, const double *fX, const double *fY,
                             const double *fZ, int nChunks)
{
    double *scr = (double *)calloc((size_t)(3 * nNodes * nChunks), sizeof(double));
    nodalforces_scratch(nBonds, nNodes, bl, F, fX, fY, fZ, scr,
                        scr + nNodes * nChunks, scr + 2 * nNodes * nChunks, nChunks);
    free(scr);
}

/* timeintegrationeulercromerMex.c:26-53 */
void orc_eulercromer(double *a, const double *F, double D, double *v,
                     const double *rho, const double *CF, double dt, double *u,
                     double *x, const double *X, int64_t nNodes, int NOD)
{
    for (int64_t k = 0; k < nNodes; k++) {
        for (int d = 0; d < NOD; d++) {
            int64_t e = k + nNodes * d;
            a[e] = (F[e] - D * v[e]) / rho[k];
            if (CF[e] == 1) a[e] = 0;
            v[e] = v[e] + (a[e] * dt);
            u[e] = u[e] + (v[e] * dt);
            x[e] = X[e] + u[e];
        }
    }
}

/* Per-node Rayleigh-quotient terms of calculatedampingcoefficient.m:61-85. */
static void damping_terms(const double *F, const double *m, const double *Fp,
                          double dt, const double *vhp, const double *u,
                          int64_t nN, int64_t i, double *t1, double *t2)
{
    double c1 = 0, c2 = 0;
    for (int d = 0; d < 3; d++) {
        int64_t e = i + nN * d;
        if (vhp[e] != 0)
            c1 = c1 - u[e] * u[e] * ((F[e] / m[i] - Fp[e] / m[i]) / (dt * vhp[e]));
    }
    for (int d = 0; d < 3; d++) {
        int64_t e = i + nN * d;
        c2 = c2 + u[e] * u[e];
    }
    *t1 = c1;
    *t2 = c2;
}

/* calculatedampingcoefficient.m:90-112 */
double orc_cn_from_sums(double cn1, double cn2)
{
    double cn;
    if (cn2 != 0) {
        if ((cn1 / cn2) > 0) cn = 2 * sqrt(cn1 / cn2);
        else cn = 0;
    } else {
        cn = 0;
    }
    if (cn > 2) cn = 1.9;
    return cn;
}

/* calculatedampingcoefficient.m:59-112, sums in the literal node/dof order. */
double orc_damping_coefficient_seq(const double *F, const double *m,
                                   const double *Fp, double dt,
                                   const double *vhp, const double *u,
                                   int64_t nN)
{
    double cn1 = 0, cn2 = 0;
    for (int64_t i = 0; i < nN; i++) {
        for (int d = 0; d < 3; d++) {
            int64_t e = i + nN * d;
            if (vhp[e] != 0)
                cn1 = cn1 - u[e] * u[e] * ((F[e] / m[i] - Fp[e] / m[i]) / (dt * vhp[e]));
        }
        for (int d = 0; d < 3; d++) {
            int64_t e = i + nN * d;
            cn2 = cn2 + u[e] * u[e];
        }
    }
    return orc_cn_from_sums(cn1, cn2);
}

/* xor butterfly over 32 values (offsets 16, 8, 4, 2, 1); value of lane 0 */
static double butterfly32(double v[32])
{
    double w[32];
    for (int off = 16; off >= 1; off /= 2) {
        for (int l = 0; l < 32; l++) w[l] = v[l] + v[l ^ off];
        memcpy(v, w, sizeof(w));
    }
    return v[0];
}

double orc_tree_sum(const double *t, int64_t n)
{
    if (n <= 0) return 0.0;
    int64_t m = (n + 31) / 32;
    double *p = (double *)malloc(sizeof(double) * (size_t)m);
    const double *src = t;
    int64_t cnt = n;
    /* level 1 reduces the terms, every further level the previous partials,
     * 32 consecutive values at a time, until one value is left */
    for (;;) {
        m = (cnt + 31) / 32;
        for (int64_t g = 0; g < m; g++) {
            double v[32];
            for (int l = 0; l < 32; l++) {
                int64_t idx = g * 32 + l;
                v[l] = (idx < cnt) ? src[idx] : 0.0;
            }
            p[g] = butterfly32(v);   /* g < m <= index of src being read: in place is safe */
        }
        if (m == 1) break;
        src = p;
        cnt = m;
    }
    double r = p[0];
    free(p);
    return r;
}

double orc_damping_coefficient_tree(const double *F, const double *m,
                                    const double *Fp, double dt,
                                    const double *vhp, const double *u,
                                    int64_t nN)
{
    double *t = (double *)malloc((size_t)(2 * nN) * sizeof(double));
    for (int64_t i = 0; i < nN; i++)
        damping_terms(F, m, Fp, dt, vhp, u, nN, i, &t[i], &t[nN + i]);
    double cn1 = orc_tree_sum(t, nN), cn2 = orc_tree_sum(t + nN, nN);
    free(t);
    return orc_cn_from_sums(cn1, cn2);
}

/* timeintegrationADR.m:53-80; vh and vhp may alias (element-wise update). */
void orc_adr_integrate(int64_t iTimeStep, double dt, double *vh, const double *F,
                       const double *m, double cn, const double *vhp, double *u,
                       const double *CF, int64_t nN)
{
    for (int64_t k = 0; k < nN; k++) {
        double minv = 1.0 / m[k];   /* massVector(kNode,1)^-1 */
        for (int d = 0; d < 3; d++) {
            int64_t e = k + nN * d;
            if (iTimeStep == 1)
                vh[e] = 0.5 * dt * minv * F[e];
            else
                vh[e] = (((2 - cn * dt) * vhp[e]) + (2 * dt * minv * F[e])) / (2 + cn * dt);
            u[e] = u[e] + (dt * vh[e]);
        }
    }
    for (int64_t e = 0; e < 3 * nN; e++) {     /* :196-197 */
        if (CF[e] == 1) { u[e] = 0; vh[e] = 0; }
    }
}

/* smoothstepdata.m:40-42 (xi^3 taken as (xi*xi)*xi, xi^2 as xi*xi) */
/* calculatedamage.m:29-45: unbroken bonds counted per node in bond order,
 * then damage = 1 - unbroken / nFAMILYMEMBERS. */
void orc_damage(const double *bl, const double *fail, const double *nFamily,
                int64_t nBonds, int64_t nNodes, double *damage)
{
    for (int64_t i = 0; i < nNodes; i++) damage[i] = 0.0;
    for (int64_t k = 0; k < nBonds; k++) {
        const int64_t i = (int64_t)bl[k] - 1, j = (int64_t)bl[nBonds + k] - 1;
        damage[i] = damage[i] + fail[k];
        damage[j] = damage[j] + fail[k];
    }
    for (int64_t i = 0; i < nNodes; i++) damage[i] = 1 - (damage[i] / nFamily[i]);
}

void orc_damageenergy(const double *BS, const double *s0, const double *sc, const double *L0,
                      const double *stretch, double k, double alpha, double cellVolume,
                      double *damageEnergy, int64_t nBonds)
{
    const double denominator = 2 * k * (exp(k) - 1) * (1 + alpha);                         /* :36 */
    const double shape = (2 * k) - (2 * exp(k)) + (alpha * k) - (alpha * k * exp(k)) + 2;  /* :47, :54 */
    const double V2 = cellVolume * cellVolume;
    for (int64_t b = 0; b < nBonds; b++) {
        const double s = stretch[b];
        double de = 0.0;
        if ((s0[b] < s) && (s <= sc[b])) {                                                  /* :43 */
            const double numerator = BS[b] * s0[b] * L0[b] * (s0[b] - s) * shape;
            de = (numerator / denominator) * V2;
        } else if (s > sc[b]) {                                                             /* :50 */
            const double numerator = BS[b] * s0[b] * L0[b] * (s0[b] - sc[b]) * shape;
            de = (numerator / denominator) * V2;
        }
        /* :61 max(damageEnergy, de), NaN entries ignored as MATLAB's max does */
        const double e = damageEnergy[b];
        damageEnergy[b] = (e != e) ? de : ((de > e) ? de : e);
    }
}

/* calculatecontactforce.m:29-80 (literal: distances from the positions at
 * entry, then the nodes inside the radius in family order). */
double orc_contact(const orc_penetrator *pen, double *cz, const double *X,
                   double *x, double *u, double *v, double dt, double V,
                   const double *rho, int64_t nNodes)
{
    const int64_t nN = nNodes;
    *cz = *cz + pen->increment;                                  /* :41 */
    double fz = 0.0;
    for (int64_t f = 0; f < pen->nFamily; f++) {
        const int64_t i = (int64_t)pen->family[f] - 1;
        const double dX = x[i] - pen->cx, dZ = x[i + 2 * nN] - *cz;   /* :43-45 */
        const double dist = sqrt((dX * dX) + (dZ * dZ));
        if (dist < pen->radius) {                                /* :49 */
            const double ux = dX / dist, uz = dZ / dist;         /* :58-61 */
            const double uxs = ux * pen->radius, uzs = uz * pen->radius;
            x[i] = pen->cx + uxs;                                /* :69-71 */
            x[i + 2 * nN] = *cz + uzs;
            double un[3], vn[3];
            for (int c = 0; c < 3; c++) {
                const int64_t e = i + c * nN;
                un[c] = x[e] - X[e];                             /* :74 */
                vn[c] = (un[c] - u[e]) / dt;                     /* :77 */
            }
            const double dpz = -1 * rho[i] * (vn[2] - v[i + 2 * nN]) / dt * V;   /* :80-82 */
            fz = fz + dpz;                                       /* :88 sum in family order */
            for (int c = 0; c < 3; c++) {
                u[i + c * nN] = un[c];
                v[i + c * nN] = vn[c];
            }
        }
    }
    return fz;
}

double orc_smoothstep(double t, double t0, double t1, double v0, double v1)
{
    double xi = (t - t0) / (t1 - t0);
    return v0 + (v1 - v0) * ((xi * xi) * xi) * (10 - 15 * xi + 6 * (xi * xi));
}

double orc_prescribed(const orc_problem *p, int64_t n)
{
    if (p->amplitude == ORC_AMP_SMOOTHSTEP)
        return orc_smoothstep((double)n, 1.0, (double)p->nTimeSteps, 0.0, p->appliedFinal);
    return p->rate * (double)n;
}

void orc_init_state(const orc_problem *p, orc_state *st)
{
    int64_t nN = p->nNodes, nB = p->nBonds;
    st->step = 1;
    st->cn = 0;
    memset(st->u, 0, sizeof(double) * 3 * nN);
    memset(st->v, 0, sizeof(double) * 3 * nN);
    memset(st->a, 0, sizeof(double) * 3 * nN);
    memset(st->F, 0, sizeof(double) * 3 * nN);
    memset(st->Fp, 0, sizeof(double) * 3 * nN);
    for (int64_t b = 0; b < nB; b++) { st->fail[b] = 1; st->BSF[b] = 0; st->flag[b] = 0; }
    double U1 = orc_prescribed(p, 1);
    for (int64_t e = 0; e < 3 * nN; e++) {
        if (p->PF && p->PF[e] == 1) st->u[e] = U1;
        st->x[e] = p->X[e] + st->u[e];
    }
    for (int q = 0; q < 4; q++) st->penCz[q] = q < p->nPen ? p->pen[q].cz : 0.0;
    st->reaction = 0.0;
}

/* ---- kernel tables ---- */

static void k_nodalforces_restated(int64_t nB, int64_t nN, const double *bl,
                                   double *F, const double *fX, const double *fY,
                                   const double *fZ, double *nfX, double *nfY,
                                   double *nfZ, int nChunks)
{
    nodalforces_scratch(nB, nN, bl, F, fX, fY, fZ, nfX, nfY, nfZ, nChunks);
}

static const orc_kernels restated = {
    orc_deformedlength, orc_bsf_exponential, orc_bondfailure, orc_bondforces,
    k_nodalforces_restated, orc_eulercromer,
};

const orc_kernels *orc_restated_kernels(void) { return &restated; }

/* Reference MEX computational routines, renamed at compile time by
 * oracle/Makefile (their original names clash between files). */
typedef void (*ref_dl_t)(double *, double *, double *, int, int, double *, double *, double *, double *, double *);
typedef void (*ref_exp_t)(double *, double *, double *, double, double, double *, double *, double *, double *, int);
typedef void (*ref_bf_t)(double *, double *, double *, double *, double *, double *, double *, double *, double *, double *, double *, double, double *, double *, int);
typedef void (*ref_nf_t)(int, int, double *, double *, double *, double *, double *, double *, double *, double *);
typedef void (*ref_ec_t)(double *, double *, double, double *, double *, double *, double, double *, double *, double *, int, int);
typedef void (*ref_fail_t)(double *, double, double *, double *, double, double, int);

static struct {
    ref_dl_t dl; ref_exp_t ex; ref_bf_t bf; ref_nf_t nf; ref_ec_t ec; ref_fail_t fl;
    double *ones_s0, *ones_sc, *zeros_sp, *zeros_bt; int64_t cap;
} R;

/* Expand a scalar (stride 0) parameter to a per-bond array: the MEX takes arrays. */
static double *expand(double **buf, const double *p, int stride, int64_t n)
{
    if (stride) return (double *)p;
    *buf = (double *)realloc(*buf, sizeof(double) * (size_t)n);
    for (int64_t k = 0; k < n; k++) (*buf)[k] = p[0];
    return *buf;
}

static void r_dl(const double *x, const double *bl, const double *L0, int64_t nB,
                 int64_t nN, double *L, double *dX, double *dY, double *dZ, double *s)
{
    R.dl((double *)x, (double *)bl, (double *)L0, (int)nB, (int)nN, L, dX, dY, dZ, s);
}

static void r_exp(const double *s, const double *s0, int s0s, const double *sc,
                  int scs, double k, double alpha, double *bsf, double *BSF,
                  const double *BT, double *flag, int64_t nB)
{
    double *a0 = expand(&R.ones_s0, s0, s0s, nB);
    double *ac = expand(&R.ones_sc, sc, scs, nB);
    double *bt = (double *)BT;
    if (!bt) { double z = 0; bt = expand(&R.zeros_bt, &z, 0, nB); }
    R.ex((double *)s, a0, ac, k, alpha, bsf, BSF, bt, flag, (int)nB);
}

static void r_fail(double *fail, double ff, const double *BT, const double *s,
                   const double *sc, int scs, double scSteel, int64_t nB)
{
    if (scs) { orc_bondfailure(fail, ff, BT, s, sc, scs, scSteel, nB); return; }
    double *bt = (double *)BT;
    if (!bt) { double z = 0; bt = expand(&R.zeros_bt, &z, 0, nB); }
    R.fl(fail, ff, bt, (double *)s, sc[0], scSteel, (int)nB);
}

static void r_bf(double *fX, double *fY, double *fZ, const double *fail,
                 const double *dX, const double *dY, const double *dZ,
                 const double *L, const double *s, const double *sp,
                 const double *BS, double V, const double *VCF, const double *BSF,
                 int64_t nB)
{
    double *spp = (double *)sp;
    if (!spp) { double z = 0; spp = expand(&R.zeros_sp, &z, 0, nB); }
    R.bf(fX, fY, fZ, (double *)fail, (double *)dX, (double *)dY, (double *)dZ,
         (double *)L, (double *)s, spp, (double *)BS, V, (double *)VCF,
         (double *)BSF, (int)nB);
}

static void r_nf(int64_t nB, int64_t nN, const double *bl, double *F,
                 const double *fX, const double *fY, const double *fZ,
                 double *nfX, double *nfY, double *nfZ, int nChunks)
{
    (void)nChunks; /* the reference forces 8 threads (calculatenodalforcesopenmpMex.c:39) */
    R.nf((int)nB, (int)nN, (double *)bl, F, (double *)fX, (double *)fY,
         (double *)fZ, nfX, nfY, nfZ);
}

static void r_ec(double *a, const double *F, double D, double *v, const double *rho,
                 const double *CF, double dt, double *u, double *x, const double *X,
                 int64_t nN, int NOD)
{
    R.ec(a, (double *)F, D, v, (double *)rho, (double *)CF, dt, u, x, (double *)X,
         (int)nN, NOD);
}

static const orc_kernels reference = { r_dl, r_exp, r_fail, r_bf, r_nf, r_ec };

const orc_kernels *orc_load_reference(const char *so_path, char *err, int errlen)
{
    void *h = dlopen(so_path, RTLD_NOW | RTLD_LOCAL);
    if (!h) { snprintf(err, (size_t)errlen, "%s", dlerror()); return NULL; }
    R.dl = (ref_dl_t)dlsym(h, "ref_calculatedeformedlength");
    R.ex = (ref_exp_t)dlsym(h, "ref_calculatebsfexponential");
    R.bf = (ref_bf_t)dlsym(h, "ref_calculatebondforces");
    R.nf = (ref_nf_t)dlsym(h, "ref_calculatenodalforces_omp");
    R.ec = (ref_ec_t)dlsym(h, "ref_timeintegrationeulercromer");
    R.fl = (ref_fail_t)dlsym(h, "ref_calculatebondfailure");
    if (!R.dl || !R.ex || !R.bf || !R.nf || !R.ec || !R.fl) {
        snprintf(err, (size_t)errlen, "missing symbol in %s", so_path);
        return NULL;
    }
    return &reference;
}

/* ---- the time loop ---- */

void orc_run(const orc_problem *p, orc_state *st, const orc_kernels *k,
             int64_t nsteps)
{
    int64_t nN = p->nNodes, nB = p->nBonds;
    /* Prescribed DOFs are held like constrained ones during integration and
     * then set to the amplitude of the next step. */
    double *CFe = (double *)malloc(sizeof(double) * (size_t)(3 * nN));
    for (int64_t e = 0; e < 3 * nN; e++)
        CFe[e] = (p->CF[e] == 1 || (p->PF && p->PF[e] == 1)) ? 1.0 : 0.0;
    const double *s0 = p->s0 ? p->s0 : &p->s0v;
    const double *s1 = p->s1 ? p->s1 : &p->s1v;
    const double *sc = p->sc ? p->sc : &p->scv;
    int s0s = p->s0 ? 1 : 0, s1s = p->s1 ? 1 : 0, scs = p->sc ? 1 : 0;
    int nCh = p->nChunks > 0 ? p->nChunks : 8;

    for (int64_t it = 0; it < nsteps; it++) {
        int64_t n = st->step;
        /* dynamicsolverdisplacementcontrolled.m:79 */
        k->deformedlength(st->x, p->bl, p->L0, nB, nN, st->L, st->dX, st->dY, st->dZ, st->s);
        /* :82-91 (law chosen by the problem) */
        switch (p->law) {
        case ORC_LAW_EXPONENTIAL:
            memset(st->bsf, 0, sizeof(double) * (size_t)nB);   /* :86 */
            k->bsfexponential(st->s, s0, s0s, sc, scs, p->kexp, p->alphaexp,
                              st->bsf, st->BSF, p->BT, st->flag, nB);
            break;
        case ORC_LAW_TRILINEAR:
            orc_bsf_trilinear(st->s, s0, s0s, s1, s1s, sc, scs, p->beta,
                              st->BSF, p->BT, st->flag, nB);
            break;
        case ORC_LAW_BILINEAR:
            orc_bsf_bilinear(st->s, s0, s0s, sc, scs, st->BSF, p->BT, st->flag, nB);
            break;
        default:
            k->bondfailure(st->fail, p->failureFunctionality, p->BT, st->s, sc,
                           scs, p->scSteel, nB);
            break;
        }
        /* :94 */
        k->bondforces(st->fX, st->fY, st->fZ, st->fail, st->dX, st->dY, st->dZ,
                      st->L, st->s, p->sp, p->BS, p->V, p->VCF, st->BSF, nB);
        /* :97-101 */
        memset(st->F, 0, sizeof(double) * (size_t)(3 * nN));
        memset(st->nfX, 0, sizeof(double) * (size_t)(nN * nCh));
        memset(st->nfY, 0, sizeof(double) * (size_t)(nN * nCh));
        memset(st->nfZ, 0, sizeof(double) * (size_t)(nN * nCh));
        k->nodalforces(nB, nN, p->bl, st->F, st->fX, st->fY, st->fZ, st->nfX,
                       st->nfY, st->nfZ, nCh);
        double Un = orc_prescribed(p, n + 1);
        if (p->scheme == ORC_SCHEME_EULERCROMER) {
            /* :105 */
            k->eulercromer(st->a, st->F, p->damping, st->v, p->rho, CFe, p->dt,
                           st->u, st->x, p->X, nN, 3);
            if (p->PF)
                for (int64_t e = 0; e < 3 * nN; e++)
                    if (p->PF[e] == 1) { st->u[e] = Un; st->x[e] = p->X[e] + st->u[e]; }
        } else {
            /* dynamicsolverdisplacementcontrolledADR.m:137,142,153-155 */
            st->cn = p->cnOrder ? orc_damping_coefficient_seq(st->F, p->mass, st->Fp, p->dt, st->v, st->u, nN)
                                : orc_damping_coefficient_tree(st->F, p->mass, st->Fp, p->dt, st->v, st->u, nN);
            orc_adr_integrate(n, p->dt, st->v, st->F, p->mass, st->cn, st->v, st->u, CFe, nN);
            for (int64_t e = 0; e < 3 * nN; e++) {
                if (p->PF && p->PF[e] == 1) { st->u[e] = Un; st->v[e] = 0; }
                st->x[e] = p->X[e] + st->u[e];
            }
            memcpy(st->Fp, st->F, sizeof(double) * (size_t)(3 * nN));
        }
        /* contact bodies after the integration (dynamicsolverdisplacementcontrolled.m:107-115) */
        if (p->nPen > 0) {
            double r = 0.0;
            int first = 1;
            for (int q = 0; q < p->nPen; q++) {
                const double fz = orc_contact(&p->pen[q], &st->penCz[q], p->X, st->x, st->u, st->v,
                                              p->dt, p->V, p->rho, nN);
                if (p->pen[q].reaction) {
                    r = first ? fz : r + fz;
                    first = 0;
                }
            }
            st->reaction = r;
        }
        st->step = n + 1;
    }
    free(CFe);
}

/* ---- input builder ---- */

int64_t orc_buildhorizons(const double *X, int64_t nNodes, double horizon, int64_t capacity,
                          double *nFamily, double *famPtr, double *family, double *bl,
                          double *L0)
{
    const int64_t n = nNodes;
    int64_t nb = 0, nf = 0;
    for (int64_t i = 0; i < n; i++) {
        int64_t c = 0;
        for (int64_t j = 0; j < n; j++) {
            if (j == i) continue;
            const double e0 = X[i] - X[j], e1 = X[i + n] - X[j + n], e2 = X[i + 2 * n] - X[j + 2 * n];
            if (sqrt(e0 * e0 + e1 * e1 + e2 * e2) <= horizon) {
                c++;
                if (j > i) nb++;
            }
        }
        if (nFamily) nFamily[i] = (double)c;
        if (famPtr) famPtr[i] = (double)(nf + 1);     /* buildhorizons.m:36-44 */
        nf += c;
    }
    if (capacity < nb) return nb;
    int64_t k = 0, f = 0;
    for (int64_t i = 0; i < n; i++)
        for (int64_t j = 0; j < n; j++) {
            if (j == i) continue;
            const double e0 = X[i] - X[j], e1 = X[i + n] - X[j + n], e2 = X[i + 2 * n] - X[j + 2 * n];
            const double L = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
            if (L > horizon) continue;
            if (family) family[f++] = (double)(j + 1);
            if (j > i) {                                /* :64-76 */
                bl[k] = (double)(i + 1);
                bl[k + nb] = (double)(j + 1);
                L0[k] = L;                              /* :88-97 */
                k++;
            }
        }
    return nb;
}

void orc_volumecorrection(const double *L0, int64_t nBonds, double horizon, double radij,
                          double *VCF)
{
    for (int64_t k = 0; k < nBonds; k++) {
        const double UL = L0[k];
        if (UL <= (horizon - radij)) VCF[k] = 1;                                   /* :23-25 */
        else if ((UL > (horizon - radij)) && (UL <= horizon)) VCF[k] = (horizon + radij - UL) / (2 * radij);
        else VCF[k] = 0;
    }
}

int orc_bonddata(const double *bl, int64_t nBonds, const double *nFamily,
                 const double *materialFlag, double bsConcrete, double bsSteel,
                 double cellVolume, double neighbourhoodVolume, double *BS, double *BT,
                 double *BFM, double *stiffening)
{
    for (int64_t k = 0; k < nBonds; k++) {
        const int64_t i = (int64_t)bl[k] - 1, j = (int64_t)bl[nBonds + k] - 1;
        const double mi = materialFlag ? materialFlag[i] : 0.0, mj = materialFlag ? materialFlag[j] : 0.0;
        double bst;
        if (mi == 0 && mj == 0) { bst = bsConcrete; BT[k] = 0; }                 /* :33-38 */
        else if (mi == 0 && mj == 1) { bst = bsConcrete; BT[k] = 1; }            /* :40-45 */
        else if (mi == 1 && mj == 0) { bst = bsConcrete; BT[k] = 1; }            /* :47-52 */
        else if (mi == 1 && mj == 1) { bst = bsSteel; BT[k] = 2; }               /* :54-59 */
        else return -1;
        const double vi = nFamily[i] * cellVolume, vj = nFamily[j] * cellVolume;    /* :62-63 */
        const double sf = (2 * neighbourhoodVolume) / ((vi + vj));                /* :64 */
        if (stiffening) stiffening[k] = sf;
        BS[k] = sf * bst;                                                          /* :65 */
        BFM[k] = BT[k] == 1 ? 3 : 1;                                               /* :70-71 */
    }
    return 0;
}

void orc_massmatrix(int64_t nNodes, double dx, double bsConcrete, double dt,
                    const double *nFamily, double *mass)
{
    for (int64_t i = 0; i < nNodes; i++) {
        const double Kij = (nFamily[i] * (dx * dx)) * (bsConcrete / dx);              /* :36 */
        mass[i] = 0.25 * (dt * dt) * Kij;                                          /* :37-38 */
    }
}

static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* determineintersection.m:59-86 with plane_line_intersect :126-150 */
static int notch_hit(const double *A, const double *B, const double *D, const double *nrm,
                     const double *P0, const double *P1)
{
    double AB[3], AD[3], u[3], w[3], I[3];
    for (int c = 0; c < 3; c++) {
        AB[c] = B[c] - A[c];
        AD[c] = D[c] - A[c];
        u[c] = P1[c] - P0[c];
        w[c] = P0[c] - A[c];
    }
    const double Dn = dot3(nrm, u), N = -dot3(nrm, w);
    if (fabs(Dn) < 1e-7) return 0;                 /* parallel: check 2 or 0, no hit */
    const double sI = N / Dn;
    for (int c = 0; c < 3; c++) I[c] = P0[c] + (sI * u[c]);
    if (sI < 0 || sI > 1) return 0;                /* check 3 */
    return (dot3(A, AB) <= dot3(I, AB)) && (dot3(I, AB) <= dot3(B, AB)) && (dot3(A, AD) <= dot3(I, AD)) &&
           (dot3(I, AD) <= dot3(D, AD));
}

int64_t orc_buildnotch(const double *X, int64_t nNodes, const double *bl, const double *L0,
                       int64_t nBonds, double DX, double xlocation, double depth,
                       double *blOut, double *L0Out, double *nFamily, double *famPtr,
                       double *family)
{
    const int64_t n = nNodes;
    double lo[3], hi[3];
    for (int c = 0; c < 3; c++) {
        lo[c] = hi[c] = X[c * n];
        for (int64_t i = 1; i < n; i++) {
            const double v = X[i + c * n];
            if (v < lo[c]) lo[c] = v;
            if (v > hi[c]) hi[c] = v;
        }
    }
    const double A[3] = {xlocation * DX, lo[1], lo[2]}, B[3] = {xlocation * DX, hi[1], lo[2]};   /* :52-55 */
    const double D[3] = {xlocation * DX, lo[1], depth * DX};
    double AB[3], AD[3], cr[3], nrm[3];
    for (int c = 0; c < 3; c++) {
        AB[c] = B[c] - A[c];
        AD[c] = D[c] - A[c];
    }
    cross3(AB, AD, cr);
    const double len = sqrt(dot3(cr, cr));
    for (int c = 0; c < 3; c++) nrm[c] = cr[c] / len;
    char *keep = (char *)malloc((size_t)(nBonds > 0 ? nBonds : 1));
    int64_t m = 0;
    for (int64_t k = 0; k < nBonds; k++) {
        const int64_t i = (int64_t)bl[k] - 1, j = (int64_t)bl[nBonds + k] - 1;
        const double P0[3] = {X[i], X[i + n], X[i + 2 * n]}, P1[3] = {X[j], X[j + n], X[j + 2 * n]};
        keep[k] = !notch_hit(A, B, D, nrm, P0, P1);
        m += keep[k];
    }
    int64_t r = 0;
    for (int64_t k = 0; k < nBonds; k++)
        if (keep[k]) {
            blOut[r] = bl[k];
            blOut[r + m] = bl[nBonds + k];
            L0Out[r] = L0[k];
            r++;
        }
    free(keep);
    /* :90-119 families from the reduced list, in bond order */
    for (int64_t i = 0; i < n; i++) nFamily[i] = 0;
    for (int64_t k = 0; k < m; k++) {
        nFamily[(int64_t)blOut[k] - 1] += 1;
        nFamily[(int64_t)blOut[k + m] - 1] += 1;
    }
    double acc = 1;
    for (int64_t i = 0; i < n; i++) {
        famPtr[i] = acc;
        acc += nFamily[i];
    }
    if (family) {
        double *cnt = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
        for (int64_t k = 0; k < m; k++) {
            const int64_t i = (int64_t)blOut[k] - 1, j = (int64_t)blOut[k + m] - 1;
            family[(int64_t)(famPtr[i] + cnt[i]) - 1] = (double)(j + 1);
            family[(int64_t)(famPtr[j] + cnt[j]) - 1] = (double)(i + 1);
            cnt[i] += 1;
            cnt[j] += 1;
        }
        free(cnt);
    }
    return m;
}

int64_t orc_stiffness_coo(const double *X, int64_t nNodes, int NOD, const double *bl,
                          const double *VCF, double V, const double *BS, const double *BFM,
                          const double *fail, const double *BSF, int64_t nBonds,
                          int64_t capacity, double *rows, double *cols, double *vals,
                          double *mass)
{
    const int64_t n = nNodes;
    if (mass)
        for (int64_t i = 0; i < n; i++) mass[i] = 0.0;
    int64_t cnt = 0;
    for (int64_t k = 0; k < nBonds; k++) {
        if (fail[k] != 1) continue;                                      /* :72, :110 */
        const int64_t i = (int64_t)bl[k] - 1, j = (int64_t)bl[nBonds + k] - 1;
        double c[3], L2 = 0;
        for (int u = 0; u < NOD; u++) {
            c[u] = X[j + u * n] - X[i + u * n];                          /* :76-77, :114-116 */
            L2 = u == 0 ? c[u] * c[u] : L2 + c[u] * c[u];
        }
        const double L = sqrt(L2);
        const double rig = NOD == 3 ? BFM[k] * ((BS[k] / (L * L * L)) * VCF[k] * (V * V)) * (1 - BSF[k])   /* :118 */
                                    : BFM[k] * (BS[k] / (L * L * L)) * VCF[k] * (V * V);                     /* :79 */
        const int D = 2 * NOD;
        for (int s = 0; s < D; s++)                                      /* find: column-major */
            for (int r = 0; r < D; r++) {
                const double m = c[r % NOD] * c[s % NOD];
                const double v = ((r < NOD) == (s < NOD)) ? rig * m : rig * (-m);
                if (v == 0) continue;
                if (cnt < capacity) {
                    rows[cnt] = (double)((r < NOD ? NOD * i : NOD * j) + (r % NOD) + 1);
                    cols[cnt] = (double)((s < NOD ? NOD * i : NOD * j) + (s % NOD) + 1);
                    vals[cnt] = v;
                }
                cnt++;
            }
        if (mass) {
            const double nm = 2 * fabs(rig) * L2;                        /* norm(Klocal) */
            mass[i] = mass[i] + nm;
            mass[j] = mass[j] + nm;
        }
    }
    return cnt;
}
