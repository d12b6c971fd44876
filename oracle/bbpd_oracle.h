/*
 * bbpd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the BB_PD bond-force chain and
 * the explicit / ADR time step that drives it. It exists so that tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg can check the CUDA
 * path. Nothing in the product (bb_pd_b200/) links, loads or calls it.
 *
 * Every routine cites the reference file:line it restates (paths inside the
 * mark-hobbs/BB_PD tree). Arrays use the reference's MATLAB conventions:
 * column-major, node-major SoA (x of node k at [k], y at [k + nNodes], ...),
 * 1-based node ids stored as doubles in BONDLIST (nBonds x 2).
 *
 * Floating-point contract: compiled without FMA contraction (-ffp-contract=off),
 * every expression evaluated in the order the reference writes it, so that the
 * results are bit-identical to the reference MEX routines compiled with gcc
 * on x86-64 (checked against them in tests/). The ADR Rayleigh-quotient sums
 * (MATLAB-only in the reference) are offered twice: literally sequential, and in
 * the fixed blocked-tree order that the CUDA kernels reproduce bit for bit.
 *
 * Parity pinning: the reference ships no tests, fixtures or golden vectors.
 * The restatement is pinned against the reference's own MEX routines compiled
 * from their sources (oracle/Makefile -> oracle/_ref/libbbpd_ref.so) and against
 * golden vectors generated from them (tests/golden/). The MATLAB-only pieces
 * (trilinear and bilinear laws, ADR, smooth step) have no compiled reference;
 * they are restated from the .m sources and pinned by known-answer tests.
 */
#ifndef BBPD_ORACLE_H
#define BBPD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- per-routine restatements (reference layouts, in place) ---- */

/* calculatedeformedlengthMex.c:27-47 */
void orc_deformedlength(const double *x, const double *bl, const double *L0,
                        int64_t nBonds, int64_t nNodes, double *L,
                        double *dX, double *dY, double *dZ, double *s);

/* Numerator exp of the restated exponential law: libm's (0, the default) or a
 * correctly rounded one (1). The compiled reference routines always use libm. */
void orc_use_cr_exp(int on);
/* calculatebsfexponentialMex.c:26-66. bsf is the caller-zeroed scratch
 * (dynamicsolverdisplacementcontrolled.m:86). s0/sc strides: 1 = per bond, 0 = scalar. */
void orc_bsf_exponential(const double *s, const double *s0, int s0_stride,
                         const double *sc, int sc_stride, double k, double alpha,
                         double *bsf, double *BSF, const double *BT,
                         double *flag, int64_t nBonds);

/* calculatebsftrilinear.m:40-112 (MATLAB only). Strides as above. */
void orc_bsf_trilinear(const double *s, const double *s0, int s0_stride,
                       const double *s1, int s1_stride, const double *sc,
                       int sc_stride, double beta, double *BSF, const double *BT,
                       double *flag, int64_t nBonds);

/* calculatebondsofteningfactor.m:42-48 (MATLAB only, bilinear). */
void orc_bsf_bilinear(const double *s, const double *s0, int s0_stride,
                      const double *sc, int sc_stride, double *BSF,
                      const double *BT, double *flag, int64_t nBonds);

/* calculatebondfailureMex.c:26-44 (brittle "linear" law; interface bonds 3x sc). */
void orc_bondfailure(double *fail, double failureFunctionality, const double *BT,
                     const double *s, const double *sc, int sc_stride,
                     double scSteel, int64_t nBonds);

/* calculatebondforcesMex.c:26-45 */
void orc_bondforces(double *fX, double *fY, double *fZ, const double *fail,
                    const double *dX, const double *dY, const double *dZ,
                    const double *L, const double *s, const double *sp,
                    const double *BS, double V, const double *VCF,
                    const double *BSF, int64_t nBonds);

/* calculatenodalforcesopenmpMex.c:29-85 with its OpenMP static schedule made
 * explicit: nChunks contiguous bond ranges (libgomp rule), one private partial
 * per chunk summed in bond order, then summed over chunks in chunk order.
 * nChunks = 8 is the reference's forced team (line 39); nChunks = 1 is the
 * serial calculatenodalforcesMex.c:19-46. F is accumulated into (caller zeroes). */
void orc_nodalforces_chunked(int64_t nBonds, int64_t nNodes, const double *bl,
                             double *F, const double *fX, const double *fY,
                             const double *fZ, int nChunks);

/* Bond range [*lo, *hi) of chunk c under libgomp's static schedule. */
void orc_chunk_range(int64_t n, int nChunks, int c, int64_t *lo, int64_t *hi);

/* timeintegrationeulercromerMex.c:26-53 */
void orc_eulercromer(double *a, const double *F, double D, double *v,
                     const double *rho, const double *CF, double dt, double *u,
                     double *x, const double *X, int64_t nNodes, int NOD);

/* calculatedampingcoefficient.m:59-112, literal sequential sums. */
double orc_damping_coefficient_seq(const double *F, const double *m,
                                   const double *Fp, double dt,
                                   const double *vhp, const double *u,
                                   int64_t nNodes);

/* Same coefficient, with cn1 and cn2 summed in the fixed blocked-tree order
 * used by the CUDA kernels (see orc_tree_sum). */
double orc_damping_coefficient_tree(const double *F, const double *m,
                                    const double *Fp, double dt,
                                    const double *vhp, const double *u,
                                    int64_t nNodes);

/* Clamp of calculatedampingcoefficient.m:90-112 applied to two sums. */
double orc_cn_from_sums(double cn1, double cn2);

/* Fixed reduction order over per-node terms t[0..n): a 32-ary tree. Level 1
 * takes slices of 32 consecutive nodes, every further level groups of 32
 * consecutive partials of the level below; each group is folded by an xor
 * butterfly (offsets 16, 8, 4, 2, 1; lane l adds lane l^off; the result is
 * lane 0's), missing members count as 0.0; levels repeat until one value is
 * left. */
double orc_tree_sum(const double *t, int64_t n);

/* timeintegrationADR.m:53-80 (ADR central-difference half-step update). */
void orc_adr_integrate(int64_t iTimeStep, double dt, double *vh, const double *F,
                       const double *m, double cn, const double *vhp, double *u,
                       const double *CF, int64_t nNodes);

/* calculatedamage.m:29-45 (damage per node, nNodes entries). */
void orc_damage(const double *bl, const double *fail, const double *nFamily,
                int64_t nBonds, int64_t nNodes, double *damage);

/* calculatedamageenergy.m:34-62 (energy dissipated by every bond, never
 * decreasing; k and alpha as the drivers pass them, 25 and 0.25). */
void orc_damageenergy(const double *BS, const double *s0, const double *sc, const double *L0,
                      const double *stretch, double k, double alpha, double cellVolume,
                      double *damageEnergy, int64_t nBonds);

/* ---- input builder (the reference's input module) ---- */

/* buildhorizons.m:13-97 by brute force: node j is in node i's family when
 * sqrt(((xi - xj)^2 + (yi - yj)^2) + (zi - zj)^2) <= horizon, j != i. Families
 * are listed by ascending node id (the reference's rangesearch lists them by
 * distance); BONDLIST rows (i, j), i < j, by i then j, 1-based doubles.
 * Returns nBonds; the arrays are written when capacity >= nBonds
 * (NODEFAMILY then needs 2 nBonds entries). */
int64_t orc_buildhorizons(const double *X, int64_t nNodes, double horizon, int64_t capacity,
                          double *nFamily, double *famPtr, double *family, double *bl,
                          double *L0);

/* calculatevolumecorrectionfactors.m:16-34 */
void orc_volumecorrection(const double *L0, int64_t nBonds, double horizon, double radij,
                          double *VCF);

/* buildbonddata.m:16-66 (materialFlag null: every node concrete). Returns 0,
 * or -1 when a material flag is neither 0 nor 1. */
int orc_bonddata(const double *bl, int64_t nBonds, const double *nFamily,
                 const double *materialFlag, double bsConcrete, double bsSteel,
                 double cellVolume, double neighbourhoodVolume, double *BS, double *BT,
                 double *BFM, double *stiffening);

/* buildmassmatrix.m:32-40 */
void orc_massmatrix(int64_t nNodes, double dx, double bsConcrete, double dt,
                    const double *nFamily, double *mass);

/* buildnotch.m:13-119 with determineintersection.m:59-150: bonds whose segment
 * meets the rectangle x = xlocation DX, y in [min y, max y], z in [min z,
 * depth DX] are removed, families rebuilt from the reduced list. Writes the
 * kept rows (col-major with leading dimension = the returned count) and
 * returns the number kept. */
int64_t orc_buildnotch(const double *X, int64_t nNodes, const double *bl, const double *L0,
                       int64_t nBonds, double DX, double xlocation, double depth,
                       double *blOut, double *L0Out, double *nFamily, double *famPtr,
                       double *family);

/* buildstiffnessmatrixCSCformat.m:57-150 (NOD 2 or 3), literal: the
 * nonzeros of every intact bond's local matrix in MATLAB find order and
 * massVector += norm(Klocal) at both ends, the norm taken as 2 |rig| |c|^2.
 * Returns the triplet count; writes the triplets when capacity allows. */
int64_t orc_stiffness_coo(const double *X, int64_t nNodes, int NOD, const double *bl,
                          const double *VCF, double V, const double *BS, const double *BFM,
                          const double *fail, const double *BSF, int64_t nBonds,
                          int64_t capacity, double *rows, double *cols, double *vals,
                          double *mass);

/* smoothstepdata.m:40-42 */
double orc_smoothstep(double t, double t0, double t1, double v0, double v1);

/* ---- the time loop (dynamicsolverdisplacementcontrolled.m:71-105, ADR per
 *      dynamicsolverdisplacementcontrolledADR.m:91-155 with the ADR calls the
 *      reference leaves commented at :137 and :142 switched on) ---- */

enum { ORC_LAW_LINEAR = 0, ORC_LAW_BILINEAR = 1, ORC_LAW_TRILINEAR = 2,
       ORC_LAW_EXPONENTIAL = 3 };
enum { ORC_SCHEME_EULERCROMER = 0, ORC_SCHEME_ADR = 1 };
enum { ORC_AMP_LINEAR = 0, ORC_AMP_SMOOTHSTEP = 1 };

/* A rigid cylinder (axis along y) pushed into the body: the penetrator and
 * supports of calculatecontactforce.m. */
typedef struct orc_penetrator {
    double cx, cz;          /* centre before step 1 */
    double radius;
    double increment;       /* centre z change per step (0 for a support) */
    const double *family;   /* 1-based node ids checked for contact, in order */
    int64_t nFamily;
    int reaction;           /* its force counts toward the reaction */
} orc_penetrator;

/* calculatecontactforce.m:29-80: moves the centre by `increment` (*cz), pushes
 * family nodes inside the radius back onto the surface, updates their
 * displacement, velocity and deformed position, and returns the z force on
 * the cylinder (sum over the family in order). */
double orc_contact(const orc_penetrator *pen, double *cz, const double *X,
                   double *x, double *u, double *v, double dt, double V,
                   const double *rho, int64_t nNodes);

typedef struct orc_problem {
    int64_t nNodes, nBonds;
    const double *X;        /* nNodes x 3 */
    const double *bl;       /* nBonds x 2, 1-based */
    const double *L0, *BS, *VCF, *BT; /* nBonds (BT may be NULL: all concrete) */
    const double *sp;       /* nBonds or NULL (zeros) */
    const double *s0, *s1, *sc; /* per-bond arrays or NULL (use scalars) */
    double s0v, s1v, scv, scSteel, kexp, alphaexp, beta, failureFunctionality;
    double V, dt, damping;
    const double *rho;      /* nNodes, Euler-Cromer density */
    const double *mass;     /* nNodes, ADR fictitious mass */
    const double *CF;       /* nNodes x 3, constraint flags */
    const double *PF;       /* nNodes x 3 prescribed-displacement flags or NULL */
    int law, scheme, amplitude, nChunks;
    double rate;            /* linear amplitude: U(n) = rate * n */
    double appliedFinal;    /* smooth-step amplitude final value */
    int64_t nTimeSteps;     /* smooth-step final step */
    int cnOrder;            /* 0 = fixed tree (GPU order), 1 = literal sequential */
    int nPen;               /* contact bodies applied after each integration, in order */
    orc_penetrator pen[4];
} orc_problem;

typedef struct orc_state {
    int64_t step;           /* next time step to run, 1-based */
    double cn;              /* last ADR damping coefficient */
    double *x, *u, *v, *a, *F, *Fp; /* nNodes x 3 (v = v_half for ADR) */
    double *fail, *BSF, *flag;      /* nBonds */
    double *L, *dX, *dY, *dZ, *s, *fX, *fY, *fZ, *bsf; /* nBonds scratch */
    double *nfX, *nfY, *nfZ;        /* nNodes x nChunks scratch (nodal-force partials) */
    double penCz[4];                /* current centre z of each contact body */
    double reaction;                /* reactionForce of the last step (contact runs) */
} orc_state;

/* Prescribed displacement at step n for the chosen amplitude. */
double orc_prescribed(const orc_problem *p, int64_t n);

/* Initial state (arraypreallocation.m:25-56): zeros, fail = 1, x = X + u with
 * prescribed DOFs at U(1). Arrays must be allocated by the caller. */
void orc_init_state(const orc_problem *p, orc_state *st);

/* Function table of the bond/node routines; orc_run calls through it, so the
 * loop can run either this restatement or the reference's compiled MEX
 * routines (loaded by orc_load_reference). */
typedef struct orc_kernels {
    void (*deformedlength)(const double *x, const double *bl, const double *L0,
                           int64_t nB, int64_t nN, double *L, double *dX,
                           double *dY, double *dZ, double *s);
    void (*bsfexponential)(const double *s, const double *s0, int s0s,
                           const double *sc, int scs, double k, double alpha,
                           double *bsf, double *BSF, const double *BT,
                           double *flag, int64_t nB);
    void (*bondfailure)(double *fail, double ff, const double *BT,
                        const double *s, const double *sc, int scs,
                        double scSteel, int64_t nB);
    void (*bondforces)(double *fX, double *fY, double *fZ, const double *fail,
                       const double *dX, const double *dY, const double *dZ,
                       const double *L, const double *s, const double *sp,
                       const double *BS, double V, const double *VCF,
                       const double *BSF, int64_t nB);
    void (*nodalforces)(int64_t nB, int64_t nN, const double *bl, double *F,
                        const double *fX, const double *fY, const double *fZ,
                        double *nfX, double *nfY, double *nfZ, int nChunks);
    void (*eulercromer)(double *a, const double *F, double D, double *v,
                        const double *rho, const double *CF, double dt,
                        double *u, double *x, const double *X, int64_t nN,
                        int NOD);
} orc_kernels;

/* The restatement's own kernels. */
const orc_kernels *orc_restated_kernels(void);

/* dlopen the reference MEX routines built by oracle/Makefile and return a
 * table that calls them (NULL and a message in err if unavailable). The
 * reference's nodal-force routine always runs 8 OpenMP threads. */
const orc_kernels *orc_load_reference(const char *so_path, char *err, int errlen);

/* Run nsteps time steps. */
void orc_run(const orc_problem *p, orc_state *st, const orc_kernels *k,
             int64_t nsteps);

#ifdef __cplusplus
}
#endif

#endif
