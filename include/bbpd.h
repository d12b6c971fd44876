/*
 * bbpd.h -- C ABI of libbbpd, a B200 (sm_100a) implementation of the BB_PD
 * bond-based peridynamics hot path: per-bond deformed length and stretch,
 * constitutive law with irreversible damage, bond force, fixed-order nodal
 * force sum, and the Euler-Cromer / adaptive-dynamic-relaxation (ADR) time step.
 *
 * Conventions (identical to the reference's MEX routines):
 *   - arrays are double precision, column-major (MATLAB): a node array of
 *     nNodes x 3 stores x of node k at [k], y at [k + nNodes], z at [k + 2 nNodes];
 *   - BONDLIST is nBonds x 2, node ids 1-based and stored as doubles;
 *   - "in place" arguments are read and overwritten, as the MEX files do.
 * Every function returns a bbpd_status; nothing long-jumps or aborts.
 * Plain pointers and sizes only: no C++ or framework types cross this ABI.
 *
 * Numerics: the FP64 paths evaluate each expression in the reference's order
 * with no fused multiply-add, and sum nodal forces in the reference's OpenMP
 * order, so their results are bit-identical to the reference MEX chain on the
 * same inputs (the exponential law's exp() aside, which may differ from glibc's
 * in the last bit).
 */
#ifndef BBPD_H
#define BBPD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BBPD_ABI_VERSION 1

typedef enum bbpd_status {
    BBPD_OK = 0,
    BBPD_ERR_ARG = 1,          /* invalid argument, size or value */
    BBPD_ERR_CUDA = 2,         /* CUDA runtime error (message in bbpd_last_error) */
    BBPD_ERR_OOM = 3,          /* device allocation failed */
    BBPD_ERR_TIMEOUT = 4,      /* a device-side wait gave up (kernel returned early) */
    BBPD_ERR_NONFINITE = 5,    /* a displacement or velocity became NaN/Inf */
    BBPD_ERR_UNSUPPORTED = 6,  /* valid input outside what this library implements */
    BBPD_ERR_NO_DEVICE = 7     /* no CUDA device (this library has no CPU path) */
} bbpd_status;

enum { BBPD_LAW_LINEAR = 0,       /* brittle: calculatebondfailureMex.c:26-44 */
       BBPD_LAW_BILINEAR = 1,     /* calculatebondsofteningfactor.m:42-48 */
       BBPD_LAW_TRILINEAR = 2,    /* calculatebsftrilinear.m:80-112 */
       BBPD_LAW_EXPONENTIAL = 3   /* calculatebsfexponentialMex.c:26-66 */ };
enum { BBPD_SCHEME_EULERCROMER = 0, BBPD_SCHEME_ADR = 1 };
enum { BBPD_PREC_FP64 = 0,        /* plain form: bit-identical to the reference chain */
       BBPD_PREC_FP32 = 1         /* FP32 stretch/force, FP64 sums, FP64 guard band; inputs
                                     whose FP32 bond-vector dictionary exceeds 65 535
                                     entries run the FP64 kernel */ };
enum { BBPD_AMP_LINEAR = 0,       /* U(n) = rate * n */
       BBPD_AMP_SMOOTHSTEP = 1    /* smoothstepdata.m:40-42 from step 1 to nTimeSteps */ };
enum { BBPD_ORDER_INPUT = 0,      /* input node order, neighbours gathered from HBM/L2
                                     with L2 prefetch of the bond streams; the default */
       BBPD_ORDER_MORTON = 1,     /* Morton node order, neighbours gathered from HBM/L2 */
       BBPD_ORDER_TILED = 2,      /* Morton order in 512-node tiles whose neighbours are
                                     staged in shared memory (falls back to MORTON when a
                                     tile's neighbourhood does not fit) */
       BBPD_ORDER_LATTICE = 3     /* lattice form: nodes on a regular lattice in x-fastest
                                     order (buildmaterialpointcoordinates.m) with a bond
                                     list ordered by first node and one common family
                                     order (buildbonddata.m): neighbours addressed by the
                                     stencil, one state slot per bond, tiles of positions
                                     staged in shared memory. FP64 form; other inputs and
                                     the FP32 form fall back to INPUT */ };

/* Message of the last failing call on this thread ("" if none). */
const char *bbpd_last_error(void);
const char *bbpd_status_string(int status);
int bbpd_abi_version(void);
/* Number of visible CUDA devices (0 when there is none). */
int bbpd_device_count(void);

/* ===================================================================== *
 *  Per-routine entry points: one per reference MEX routine.             *
 *  _dev_ variants take device pointers and a cudaStream_t (as void*,    *
 *  NULL = legacy default stream) and return after enqueueing.           *
 *  Host-pointer variants copy in, run, copy out and synchronize; they   *
 *  are what the mexFunction gateways call.                              *
 * ===================================================================== */

/* replaces calculatedeformedlength, calculatedeformedlengthMex.c:27 */
int bbpd_dev_calculatedeformedlength(const double *deformedCoordinates,
        const double *bondlist, const double *undeformedLength, int64_t nBonds,
        int64_t nNodes, double *deformedLength, double *deformedX,
        double *deformedY, double *deformedZ, double *stretch, void *stream);
int bbpd_calculatedeformedlength(const double *deformedCoordinates,
        const double *bondlist, const double *undeformedLength, int64_t nBonds,
        int64_t nNodes, double *deformedLength, double *deformedX,
        double *deformedY, double *deformedZ, double *stretch);

/* replaces calculatebsfexponential, calculatebsfexponentialMex.c:26 (s0, sc per bond) */
int bbpd_dev_calculatebsfexponential(const double *stretch, const double *s0,
        const double *sc, double k, double alpha, double *bsf,
        double *bondSofteningFactor, const double *BONDTYPE,
        double *flagBondSoftening, int64_t nBonds, void *stream);
int bbpd_calculatebsfexponential(const double *stretch, const double *s0,
        const double *sc, double k, double alpha, double *bsf,
        double *bondSofteningFactor, const double *BONDTYPE,
        double *flagBondSoftening, int64_t nBonds);

/* replaces calculatebsftrilinear.m:1 (scalar s0, s1, sc; beta = 0.25 at :41) */
int bbpd_dev_calculatebsftrilinear(const double *stretch, double s0, double s1,
        double sc, double *bondSofteningFactor, const double *BONDTYPE,
        double *flagBondSoftening, int64_t nBonds, void *stream);
int bbpd_calculatebsftrilinear(const double *stretch, double s0, double s1,
        double sc, double *bondSofteningFactor, const double *BONDTYPE,
        double *flagBondSoftening, int64_t nBonds);

/* replaces calculatebondsofteningfactor.m:1 (bilinear; scalar s0, sc) */
int bbpd_dev_calculatebondsofteningfactor(const double *stretch, double s0,
        double sc, double *flagBondSoftening, double *bondSofteningFactor,
        const double *BONDTYPE, int64_t nBonds, void *stream);
int bbpd_calculatebondsofteningfactor(const double *stretch, double s0,
        double sc, double *flagBondSoftening, double *bondSofteningFactor,
        const double *BONDTYPE, int64_t nBonds);

/* replaces calculatebondfailure, calculatebondfailureMex.c:26 */
int bbpd_dev_calculatebondfailure(double *fail, double failureFunctionality,
        const double *BONDTYPE, const double *stretch,
        double criticalStretchConcrete, double criticalStretchSteel,
        int64_t nBonds, void *stream);
int bbpd_calculatebondfailure(double *fail, double failureFunctionality,
        const double *BONDTYPE, const double *stretch,
        double criticalStretchConcrete, double criticalStretchSteel,
        int64_t nBonds);

/* replaces calculatebondforces, calculatebondforcesMex.c:26 */
int bbpd_dev_calculatebondforces(double *bForceX, double *bForceY,
        double *bForceZ, const double *fail, const double *deformedX,
        const double *deformedY, const double *deformedZ,
        const double *deformedLength, const double *stretch,
        const double *stretchPlastic, const double *BONDSTIFFNESS,
        double cellVolume, const double *VOLUMECORRECTIONFACTORS,
        const double *bondSofteningFactor, int64_t nBonds, void *stream);
int bbpd_calculatebondforces(double *bForceX, double *bForceY,
        double *bForceZ, const double *fail, const double *deformedX,
        const double *deformedY, const double *deformedZ,
        const double *deformedLength, const double *stretch,
        const double *stretchPlastic, const double *BONDSTIFFNESS,
        double cellVolume, const double *VOLUMECORRECTIONFACTORS,
        const double *bondSofteningFactor, int64_t nBonds);

/* Nodal force sum. The reference scatters with per-thread private arrays
 * (calculatenodalforcesopenmpMex.c:29-85); here a plan holds the per-node
 * bond lists (bond order) once, and each node sums its bonds in the
 * reference's order: nChunks contiguous bond ranges under OpenMP's static
 * schedule (8 = the reference's forced team, 1 = the serial
 * calculatenodalforcesMex.c), chunk partials added in chunk order.
 * The plan owns device memory; create it once per bond list. */
typedef struct bbpd_nodal_plan bbpd_nodal_plan;
int bbpd_nodal_plan_create(const double *bondlist_dev, int64_t nBonds,
        int64_t nNodes, int nChunks, void *stream, bbpd_nodal_plan **plan);
int bbpd_nodal_plan_destroy(bbpd_nodal_plan *plan);
/* replaces calculatenodalforces, calculatenodalforcesopenmpMex.c:29; adds into nodalForce */
int bbpd_dev_calculatenodalforces(const bbpd_nodal_plan *plan,
        double *nodalForce, const double *bForceX, const double *bForceY,
        const double *bForceZ, void *stream);
int bbpd_calculatenodalforces(const double *bondlist, int64_t nBonds,
        int64_t nNodes, double *nodalForce, const double *bForceX,
        const double *bForceY, const double *bForceZ, int nChunks);

/* replaces timeintegrationeulercromer, timeintegrationeulercromerMex.c:26 */
int bbpd_dev_timeintegrationeulercromer(double *nodalAcceleration,
        const double *nodalForce, double DAMPING, double *nodalVelocity,
        const double *DENSITY, const double *constraintFlag, double DT,
        double *nodalDisplacement, double *deformedCoordinates,
        const double *undeformedCoordinates, int64_t nNodes, int NOD,
        void *stream);
int bbpd_timeintegrationeulercromer(double *nodalAcceleration,
        const double *nodalForce, double DAMPING, double *nodalVelocity,
        const double *DENSITY, const double *constraintFlag, double DT,
        double *nodalDisplacement, double *deformedCoordinates,
        const double *undeformedCoordinates, int64_t nNodes, int NOD);

/* replaces calculatedampingcoefficient.m:1 (NOD = 3). The Rayleigh-quotient
 * sums use a fixed blocked-tree order (slices of 32 nodes, then 1024 strands),
 * so the result is deterministic; *cn is written to host memory. Uses a
 * scratch buffer of 2 * ceil(nNodes / 32) doubles that it allocates. */
int bbpd_dev_calculatedampingcoefficient(const double *nodalForce,
        const double *massVector, const double *nodalForcePrevious, double DT,
        const double *nodalVelocityPreviousHalf, const double *nodalDisplacement,
        int64_t nNodes, double *cn, void *stream);
int bbpd_calculatedampingcoefficient(const double *nodalForce,
        const double *massVector, const double *nodalForcePrevious, double DT,
        const double *nodalVelocityPreviousHalf, const double *nodalDisplacement,
        int64_t nNodes, double *cn);

/* No counterpart in the reference. The damping coefficient above without any
 * device allocation, for callers that must not allocate device memory per call
 * (a time loop that has handed the device's memory to its own fixed pool, or
 * one held to a fixed HBM budget, where a per-step allocation could fail or grow
 * the pool mid-run). Same sums in the same tree order; the result is written to
 * *cn in DEVICE memory (one double), stream-ordered, with no host
 * synchronisation. Scratch is a fixed 256 KiB array per device inside the
 * library, so nNodes <= BBPD_DAMPING_NOALLOC_MAX_NODES (larger: BBPD_ERR_ARG).
 * The first call on each device looks up that array's address: make it before
 * any stream capture. The address is kept for the life of the process, so
 * after cudaDeviceReset on a device, unload and reload the library before the
 * next call there. Nothing needs zeroing beforehand. Calls that overlap on
 * one device (unordered streams or host threads) race on the shared scratch. */
#define BBPD_DAMPING_NOALLOC_MAX_NODES 16777216
int bbpd_dev_calculatedampingcoefficient_noalloc(const double *nodalForce,
        const double *massVector, const double *nodalForcePrevious, double DT,
        const double *nodalVelocityPreviousHalf, const double *nodalDisplacement,
        int64_t nNodes, double *cn, void *stream);

/* replaces calculatedamage.m:1 (damage = fraction of broken bonds per node,
 * :34-45): damage[i] = 1 - (sum of fail over node i's bonds) / nFAMILYMEMBERS[i].
 * fail holds 0 or 1, so the sums are exact whatever their order. */
int bbpd_dev_calculatedamage(const double *bondlist, const double *fail,
        const double *nFAMILYMEMBERS, int64_t nBonds, int64_t nNodes,
        double *damage, void *stream);
int bbpd_calculatedamage(const double *bondlist, const double *fail,
        const double *nFAMILYMEMBERS, int64_t nBonds, int64_t nNodes, double *damage);

/* replaces calculatedamageenergy.m:1 (energy dissipated by every bond,
 * :34-62): for s0 < stretch <= sc the bond's energy is BONDSTIFFNESS s0
 * UNDEFORMEDLENGTH (s0 - stretch) shape / den cellVolume^2, above sc the same
 * with sc in place of the stretch, else 0, with shape = 2k - 2e^k + alpha k -
 * alpha k e^k + 2 and den = 2k (e^k - 1)(1 + alpha); damageEnergy keeps the
 * larger of its value and this one (damageEnergy in place, nBonds entries).
 * The drivers pass k = 25, alpha = 0.25
 * (dynamicsolverdisplacementcontrolled.m:121). */
int bbpd_dev_calculatedamageenergy(const double *BONDSTIFFNESS, const double *s0,
        const double *sc, const double *UNDEFORMEDLENGTH, const double *stretch,
        double k, double alpha, double cellVolume, double *damageEnergy,
        int64_t nBonds, void *stream);
int bbpd_calculatedamageenergy(const double *BONDSTIFFNESS, const double *s0,
        const double *sc, const double *UNDEFORMEDLENGTH, const double *stretch,
        double k, double alpha, double cellVolume, double *damageEnergy, int64_t nBonds);

/* ---- input builder (the reference's input module, on the GPU) ----
 * Host-pointer calls copy their inputs to the device and their outputs back;
 * the bbpd_dev_ forms take device pointers and a stream (NULL: the default
 * stream) and return once their results are complete. Arrays follow the
 * reference's layouts: column-major, node ids 1-based doubles. */

/* replaces buildhorizons.m:1 (families and bond list, :13-97). Node j is in
 * node i's family when sqrt(((xi-xj)^2 + (yi-yj)^2) + (zi-zj)^2) <= horizon,
 * j != i (found with a cell list instead of rangesearch; families are listed
 * by ascending node id, rangesearch lists them by distance). BONDLIST rows are
 * (i, j) with i < j, by i then j; UNDEFORMEDLENGTH is the same square root.
 * *nBonds always receives the bond count; nFAMILYMEMBERS and
 * NODEFAMILYPOINTERS (nNodes entries, 1-based) are written when not NULL;
 * BONDLIST (nBonds x 2), UNDEFORMEDLENGTH and NODEFAMILY (2 nBonds entries) are
 * written when capacity >= nBonds (call with capacity 0 to size them). */
int bbpd_buildhorizons(const double *undeformedCoordinates, int64_t nNodes,
        double horizonRadius, int64_t capacity, int64_t *nBonds,
        double *nFAMILYMEMBERS, double *NODEFAMILYPOINTERS, double *NODEFAMILY,
        double *BONDLIST, double *UNDEFORMEDLENGTH);
int bbpd_dev_buildhorizons(const double *undeformedCoordinates, int64_t nNodes,
        double horizonRadius, int64_t capacity, int64_t *nBonds,
        double *nFAMILYMEMBERS, double *NODEFAMILYPOINTERS, double *NODEFAMILY,
        double *BONDLIST, double *UNDEFORMEDLENGTH, void *stream);

/* replaces buildnotch.m:1 (:13-119 with determineintersection.m:59-150): the
 * bonds whose segment meets the rectangle x = xlocation DX, y from the least
 * to the largest y coordinate, z from the least z coordinate to depth DX are
 * removed; the kept rows keep their order. *nBondsOut receives their count;
 * BONDLISTout (written nBondsOut x 2, room for nBonds x 2), UNDEFORMEDLENGTHout
 * (room for nBonds), nFAMILYMEMBERS and NODEFAMILYPOINTERS (nNodes) and
 * NODEFAMILY (room for 2 nBonds; every family in bond order of the reduced
 * list) may each be NULL. */
int bbpd_buildnotch(const double *undeformedCoordinates, int64_t nNodes,
        const double *BONDLIST, const double *UNDEFORMEDLENGTH, int64_t nBonds,
        double DX, double xlocation, double depth, int64_t *nBondsOut,
        double *BONDLISTout, double *UNDEFORMEDLENGTHout, double *nFAMILYMEMBERS,
        double *NODEFAMILYPOINTERS, double *NODEFAMILY);
int bbpd_dev_buildnotch(const double *undeformedCoordinates, int64_t nNodes,
        const double *BONDLIST, const double *UNDEFORMEDLENGTH, int64_t nBonds,
        double DX, double xlocation, double depth, int64_t *nBondsOut,
        double *BONDLISTout, double *UNDEFORMEDLENGTHout, double *nFAMILYMEMBERS,
        double *NODEFAMILYPOINTERS, double *NODEFAMILY, void *stream);

/* replaces calculatevolumecorrectionfactors.m:1 (:16-34): 1 for L <= horizon -
 * RADIJ, (horizon + RADIJ - L) / (2 RADIJ) up to the horizon, else 0. */
int bbpd_calculatevolumecorrectionfactors(const double *UNDEFORMEDLENGTH,
        int64_t nBonds, double horizon, double RADIJ, double *VOLUMECORRECTIONFACTORS);
int bbpd_dev_calculatevolumecorrectionfactors(const double *UNDEFORMEDLENGTH,
        int64_t nBonds, double horizon, double RADIJ, double *VOLUMECORRECTIONFACTORS,
        void *stream);

/* replaces buildbonddata.m:1 (:16-71): BONDTYPE 0 concrete-concrete, 1
 * concrete-steel (either way), 2 steel-steel from MATERIALFLAG (NULL: all
 * concrete; values other than 0 or 1 are rejected); stiffeningFactor =
 * 2 neighbourhoodVolume / (nFAM_i cellVolume + nFAM_j cellVolume);
 * BONDSTIFFNESS = stiffeningFactor x the concrete or steel constant;
 * BFMULTIPLIER 3 for BONDTYPE 1, else 1. BONDTYPE, BFMULTIPLIER and
 * stiffeningFactor may be NULL. The reference's VOLUMECORRECTIONFACTORS
 * argument is unused there and absent here. */
int bbpd_buildbonddata(const double *BONDLIST, int64_t nBonds, int64_t nNodes,
        const double *nFAMILYMEMBERS, const double *MATERIALFLAG,
        double bondStiffnessConcrete, double bondStiffnessSteel, double cellVolume,
        double neighbourhoodVolume, double *BONDSTIFFNESS, double *BONDTYPE,
        double *BFMULTIPLIER, double *stiffeningFactor);
int bbpd_dev_buildbonddata(const double *BONDLIST, int64_t nBonds, int64_t nNodes,
        const double *nFAMILYMEMBERS, const double *MATERIALFLAG,
        double bondStiffnessConcrete, double bondStiffnessSteel, double cellVolume,
        double neighbourhoodVolume, double *BONDSTIFFNESS, double *BONDTYPE,
        double *BFMULTIPLIER, double *stiffeningFactor, void *stream);

/* replaces buildmassmatrix.m:1 (:32-40): the ADR mass of every node,
 * 0.25 DT^2 (nFAM DX^2)(bondStiffnessConcrete / DX). */
int bbpd_buildmassmatrix(int64_t nNodes, double DX, double bondStiffnessConcrete,
        double DT, const double *nFAMILYMEMBERS, double *massVector);
int bbpd_dev_buildmassmatrix(int64_t nNodes, double DX, double bondStiffnessConcrete,
        double DT, const double *nFAMILYMEMBERS, double *massVector, void *stream);

/* Free the device mirrors and cached plan of the host-pointer entry points
 * (the gateways register it with mexAtExit). */
int bbpd_release_mirrors(void);

/* replaces timeintegrationADR.m:1 (NOD = 3) */
int bbpd_dev_timeintegrationADR(int64_t iTimeStep, double DT,
        double *nodalVelocityForwardHalf, const double *nodalForce,
        const double *massVector, double cn,
        const double *nodalVelocityPreviousHalf, double *nodalDisplacement,
        const double *CONSTRAINTFLAG, int64_t nNodes, void *stream);
int bbpd_timeintegrationADR(int64_t iTimeStep, double DT,
        double *nodalVelocityForwardHalf, const double *nodalForce,
        const double *massVector, double cn,
        const double *nodalVelocityPreviousHalf, double *nodalDisplacement,
        const double *CONSTRAINTFLAG, int64_t nNodes);

/* ===================================================================== *
 *  Fused solver: the whole time loop of                                  *
 *  dynamicsolverdisplacementcontrolled.m:71-105 (Euler-Cromer) or its    *
 *  ADR form (dynamicsolverdisplacementcontrolledADR.m:91-155 with the    *
 *  ADR calls at :137, :142 switched on), one persistent kernel per call  *
 *  of bbpd_step, state resident on the device between calls.            *
 * ===================================================================== */

typedef struct bbpd_params {
    int32_t law;              /* BBPD_LAW_* */
    int32_t scheme;           /* BBPD_SCHEME_* */
    int32_t precision;        /* BBPD_PREC_* */
    int32_t n_chunks;         /* nodal-force summation chunks (8 = reference) */
    int32_t amplitude;        /* BBPD_AMP_* for prescribed DOFs */
    int32_t node_order;       /* BBPD_ORDER_*: device-side node ordering */
    double cell_volume;       /* cellVolume */
    double dt;                /* simulation.DT */
    double damping;           /* simulation.DAMPING (Euler-Cromer) */
    double s0, s1, sc;        /* law stretches when the per-bond arrays are NULL */
    double sc_steel;          /* brittle law, steel bonds (BONDTYPE 2) */
    double k_exp, alpha_exp;  /* exponential law (25, 0.25 at dynamicsolverdisplacementcontrolled.m:87) */
    double beta_tri;          /* trilinear beta (0.25 at calculatebsftrilinear.m:41) */
    double failure_functionality; /* value fail takes on breaking (0: failure on) */
    double rate;              /* BBPD_AMP_LINEAR: displacement per step */
    double applied_final;     /* BBPD_AMP_SMOOTHSTEP: final displacement */
    int64_t n_time_steps;     /* BBPD_AMP_SMOOTHSTEP: final step */
    double guard_band;        /* BBPD_PREC_FP32: FP64 recheck when |s - sc| < guard_band */
    double barrier_timeout_s; /* device grid-barrier wait limit (0 = 2 s) */
} bbpd_params;

/* Fill params with the reference defaults (law exponential k=25 alpha=0.25,
 * beta=0.25, 8 chunks, failure on, FP64, Euler-Cromer, guard band 1e-5). */
void bbpd_params_default(bbpd_params *p);

typedef struct bbpd_problem {
    int64_t n_nodes, n_bonds;
    const double *undeformed_coordinates; /* nNodes x 3 */
    const double *bondlist;               /* nBonds x 2, 1-based */
    const double *undeformed_length;      /* nBonds */
    const double *bond_stiffness;         /* nBonds (BONDSTIFFNESS) */
    const double *volume_correction;      /* nBonds (VOLUMECORRECTIONFACTORS) */
    const double *bond_type;              /* nBonds in {0,1,2}, or NULL = all 0 */
    const double *fail;                   /* nBonds in {0,1}, or NULL = all 1 */
    const double *stretch_plastic;        /* nBonds (must be 0), or NULL */
    const double *s0, *s1, *sc;           /* nBonds each, or NULL = params scalars */
    const double *density;                /* nNodes (Euler-Cromer), or NULL */
    const double *mass;                   /* nNodes (ADR massVector), or NULL */
    const double *constraint_flag;        /* nNodes x 3 in {0,1}, or NULL */
    const double *prescribed_flag;        /* nNodes x 3 in {0,1}, or NULL */
} bbpd_problem;

/* ---- static (implicit) solver ----
 * replaces the displacement-controlled Newton-Raphson of
 * solvers/scripts/static/newtonraphsondisplacementcontrolled.m:56-160 with its
 * tangent from buildstiffnessmatrixCSCformat.m (NOD = 3). Each step moves the
 * prescribed DOFs (prescribed_flag) by `increment`; supports
 * (constraint_flag) stay; then Newton iterations update every bond
 * (calculatedeformedlength, the law of params.law with params.s0/s1/sc,
 * calculatebondfailure with params.sc and params.sc_steel), form the bond
 * forces of calculatebondforces.m (BFMULTIPLIER from BONDTYPE: 3 for type 1)
 * and their nodal sum in bond order times cellVolume, and move the free nodes
 * by the solution of K delta = F. K is the sum over intact bonds of
 * BFM (BS / L^3) VCF cellVolume^2 (1 - BSF) [c c^T, -c c^T; -c c^T, c c^T].
 * The linear solves are a block-Jacobi preconditioned conjugate gradient to a
 * relative residual of cg_tol (the reference calls MATLAB's bicgstabl and
 * lsqr). A step ends when ||F on free DOFs|| <= tol ||F on held DOFs|| (the
 * reference uses 0.5 % of the net internal force), or after max_newton
 * solves with stats->converged = 0. Per-bond s0/s1/sc arrays are rejected. */
typedef struct bbpd_static bbpd_static;
typedef struct bbpd_static_stats {
    int32_t newton_iterations;   /* linear solves of the step */
    int32_t cg_iterations;       /* conjugate-gradient iterations, all solves */
    double residual;             /* ||nodal force on free DOFs|| at the end */
    double reaction;             /* ||nodal force on held DOFs|| at the end */
    int32_t converged;           /* 1 when residual <= tol * reaction */
    int32_t reserved;
} bbpd_static_stats;
int bbpd_static_create(const bbpd_problem *problem, const bbpd_params *params, int device,
        bbpd_static **out);
int bbpd_static_step(bbpd_static *solver, double increment, double tol, int max_newton,
        double cg_tol, int max_cg, bbpd_static_stats *stats);
/* BBPD_FIELD_DISPLACEMENT, _DEFORMED, _FORCE (nodal force times cellVolume,
 * as the driver forms it), _BSF, _FLAG, _FAIL */
int bbpd_static_get(bbpd_static *solver, int field, double *out);
int bbpd_static_destroy(bbpd_static *solver);

/* replaces buildstiffnessmatrixCSCformat.m:1 (NOD 2 or 3): the triplets of the
 * global stiffness matrix, bond by bond (intact bonds only, fail == 1), each
 * bond's nonzeros in MATLAB find order (column-major over its local matrix
 * rig [c c^T, -c c^T; -c c^T, c c^T], rows and columns its 1-based global
 * DOFs), with rig = BFMULTIPLIER ((BONDSTIFFNESS / L^3) VCF VOLUME^2)
 * (1 - bondSofteningFactor) for NOD = 3 and without the softening factor for
 * NOD = 2, c the bond vector at the given coordinates and L its length (L^3 is
 * formed as L L L). massVector (nNodes, or NULL) accumulates norm(Klocal) =
 * 2 |rig| |c|^2 of every intact bond at both ends, in bond order (MATLAB's
 * norm computes the same value by an SVD, to rounding). *nnz always receives
 * the triplet count; the triplets are written when capacity >= *nnz. The
 * reference's UNDEFORMEDLENGTH argument is unused there and absent here. */
int bbpd_buildstiffnessmatrix(const double *nodalCoordinates, int64_t nNodes, int NOD,
        const double *BONDLIST, const double *VOLUMECORRECTIONFACTORS, double VOLUME,
        const double *BONDSTIFFNESS, const double *BFMULTIPLIER, const double *fail,
        const double *bondSofteningFactor, int64_t nBonds, int64_t capacity, int64_t *nnz,
        double *globalRowIndex, double *globalColumnIndex, double *globalNonZeroValues,
        double *massVector);
int bbpd_dev_buildstiffnessmatrix(const double *nodalCoordinates, int64_t nNodes, int NOD,
        const double *BONDLIST, const double *VOLUMECORRECTIONFACTORS, double VOLUME,
        const double *BONDSTIFFNESS, const double *BFMULTIPLIER, const double *fail,
        const double *bondSofteningFactor, int64_t nBonds, int64_t capacity, int64_t *nnz,
        double *globalRowIndex, double *globalColumnIndex, double *globalNonZeroValues,
        double *massVector, void *stream);

typedef struct bbpd_solver bbpd_solver;

/* Validate, lay out (per-node bond lists in bond order, sliced by 32 nodes)
 * and upload a problem; the state starts at step 1 (arraypreallocation.m). */
int bbpd_create(const bbpd_problem *problem, const bbpd_params *params,
                int device, bbpd_solver **out);
/* Run nsteps time steps in one persistent-kernel launch; blocks until done. */
int bbpd_step(bbpd_solver *s, int64_t nsteps);
/* Enqueue nsteps on the solver's stream without waiting (status of the
 * previous work is returned by bbpd_sync). */
int bbpd_step_async(bbpd_solver *s, int64_t nsteps);
int bbpd_sync(bbpd_solver *s);
int bbpd_destroy(bbpd_solver *s);

enum { BBPD_FIELD_DISPLACEMENT = 0,  /* nodalDisplacement, nNodes x 3 */
       BBPD_FIELD_VELOCITY = 1,      /* nodalVelocity (ADR: forward half step) */
       BBPD_FIELD_FORCE = 2,         /* nodalForce of the last step */
       BBPD_FIELD_DEFORMED = 3,      /* deformedCoordinates */
       BBPD_FIELD_FORCE_PREV = 4,    /* nodalForcePrevious (ADR) */
       BBPD_FIELD_ACCELERATION = 5,  /* nodalAcceleration (Euler-Cromer) */
       BBPD_FIELD_BSF = 16,          /* bondSofteningFactor, nBonds */
       BBPD_FIELD_FLAG = 17,         /* flagBondSoftening, nBonds */
       BBPD_FIELD_FAIL = 18,         /* fail, nBonds */
       BBPD_FIELD_DAMAGE_ENERGY = 19 /* damageEnergy, nBonds (after bbpd_track_damage_energy) */ };

/* Copy a field to host memory (reference layout and node order). */
int bbpd_get(bbpd_solver *s, int field, double *host_out);
/* Overwrite a field from host memory (restoring a checkpoint; FORCE and
 * FORCE_PREV included). Bond fields set both directed copies of each bond. */
int bbpd_set(bbpd_solver *s, int field, const double *host_in);
/* Next step to run (1-based) and last ADR damping coefficient. */
/* replaces the per-step calculatedamageenergy.m call of the drivers
 * (dynamicsolverdisplacementcontrolled.m:121, :34-62 of the function) for the
 * fused solver. From this call on, every launch records the largest stretch
 * of each concrete bond (BONDTYPE 0) once it exceeds s0, and
 * bbpd_get(BBPD_FIELD_DAMAGE_ENERGY) returns the energy dissipated per bond:
 * the formula evaluated at that stretch, which equals the reference's running
 * maximum over steps because the energy never decreases with the stretch. k
 * and alpha come from params.k_exp and params.alpha_exp (25 and 0.25, the
 * values the drivers pass); other bonds report 0. Softening laws only (the
 * linear law: BBPD_ERR_UNSUPPORTED). A second call starts the record afresh;
 * the record takes 8 bytes per directed entry and is not part of a checkpoint.
 * The FP32 form records its FP32 stretch outside the guard band. */
int bbpd_track_damage_energy(bbpd_solver *s);

int bbpd_get_step(bbpd_solver *s, int64_t *step, double *cn);
int bbpd_set_step(bbpd_solver *s, int64_t step, double cn);

typedef struct bbpd_info {
    int64_t n_nodes, n_bonds, n_entries;  /* entries: directed slots incl. padding */
    int64_t n_slices;
    int32_t grid_blocks, block_threads;
    int64_t device_bytes;                 /* device memory held by the solver */
    double bytes_per_step;                /* algorithmic DRAM bytes of one step */
    int32_t layout;                       /* 1 = 16-bit dictionary ids, 2 = 32-bit ids
                                             (irregular input), 3 = FP32 dictionary of bond
                                             vectors; +16 when the tiled kernel runs,
                                             +32 when the lattice form runs */
    int32_t reserved;                     /* dictionary entries */
} bbpd_info;
int bbpd_get_info(bbpd_solver *s, bbpd_info *info);

/* replaces calculatecontactforce.m:1 (dynamicsolverdisplacementcontrolled.m:107-112,
 * dynamicsolverdisplacementcontrolledADR.m:147-150): rigid cylinders (axis
 * along y) applied after every integration, in the given order. Each step a
 * cylinder's centre moves by `increment` in z; family nodes closer than the
 * radius in the x-z plane are put back on its surface, and their displacement
 * and velocity follow; the cylinder's z force is the momentum change of those
 * nodes (DENSITY x cellVolume), summed in family order. Families must be
 * disjoint; the solver needs DENSITY. With contact, bbpd_get_reaction returns
 * the sum of the forces of the cylinders flagged `reaction` (the reference's
 * reactionForce). n = 0 removes contact. At most 4 cylinders. */
typedef struct bbpd_penetrator {
    double centre_x, centre_z;   /* centre before step 1 */
    double radius;
    double increment;            /* centre z change per step (0 for a support) */
    const double *family;        /* 1-based node ids checked for contact, in order */
    int64_t n_family;
    int32_t reaction;            /* 1: its force is part of the reaction */
    int32_t reserved;
} bbpd_penetrator;
int bbpd_set_contact(bbpd_solver *s, int n, const bbpd_penetrator *penetrators);

/* Record the displacement of up to 8 DOFs (node ids 1-based; dof 0 x, 1 y,
 * 2 z) at every step of a launch; bbpd_get_probes returns them step-major,
 * out[it * n + k], for the first nsteps steps of the last launch (4096 kept).
 * The reference's CMOD (dynamicsolverdisplacementcontrolled.m:118) is the
 * difference of two x probes. n = 0 removes the probes. */
int bbpd_set_probes(bbpd_solver *s, int n, const double *node_ids, const int32_t *dofs);
int bbpd_get_probes(bbpd_solver *s, int64_t nsteps, double *host_out);

/* Reaction of each step of the last launch: with contact (bbpd_set_contact),
 * the reference's reactionForce (dynamicsolverdisplacementcontrolled.m:115),
 * either scheme; without contact (ADR only), the internal nodal force summed
 * over the prescribed DOFs in the fixed tree order of the damping sums, the
 * equivalent quantity under prescribed displacements (the applied load is its
 * negative). out[k] belongs to the k-th step of that launch (4096 kept). */
int bbpd_get_reaction(bbpd_solver *s, int64_t n, double *host_out);

/* ---- batches: many solver states stepped by one persistent launch ----
 * Serving and batching form. Members keep their own state, step number,
 * damping coefficient and reaction history, and compute exactly what a solo
 * launch computes (results are bit-identical alone and in a batch); the batch
 * only shares the SMs. Members are grouped in classes (law x kernel
 * variant); each class is one persistent launch of a kernel specialised for
 * it, whose warps take slices of all its members from one work counter.
 * Members: ADR solvers of the batch's precision form, 16-bit dictionary ids,
 * input or Morton node order. Membership may change between launches
 * (continuous batching); a launch is captured into a CUDA graph and replayed
 * while the membership and step count stay the same. */
typedef struct bbpd_batch bbpd_batch;
typedef struct bbpd_batch_info {
    int32_t n_members;
    int32_t blocks_per_sm;     /* schedule in use */
    int32_t grab;              /* slices taken per work-counter grab */
    int32_t graph;             /* 1 if the last launch replayed a CUDA graph */
    int32_t n_classes;         /* member classes: one launch each (one per kernel precision
                                  variant; with mixing off, per law and critical-stretch
                                  form too) */
    int32_t reserved;
    int64_t total_slices;
    int64_t device_bytes;      /* device memory held by the members */
} bbpd_batch_info;
int bbpd_batch_create(int device, int precision, bbpd_batch **out);
int bbpd_batch_destroy(bbpd_batch *b);          /* members stay valid */
int bbpd_batch_add(bbpd_batch *b, bbpd_solver *s);
int bbpd_batch_remove(bbpd_batch *b, bbpd_solver *s);
/* Advance every member by nsteps in one launch, then synchronize. */
int bbpd_batch_step(bbpd_batch *b, int64_t nsteps);
/* Autotuner: time candidate schedules (resident blocks per SM x slices per
 * grab and, unless bbpd_batch_set_mixing fixed it, one launch for all laws or
 * one per law), each on nsteps_per_trial real steps of the members, and keep
 * the fastest. */
int bbpd_batch_tune(bbpd_batch *b, int64_t nsteps_per_trial, int *blocks_per_sm, int *grab);
int bbpd_batch_set_schedule(bbpd_batch *b, int blocks_per_sm, int grab, int use_graph);
int bbpd_batch_get_info(bbpd_batch *b, bbpd_batch_info *info);
/* Mixing 1: members of every law, with or without a per-entry critical
 * stretch, step in one persistent launch per kernel precision variant, each
 * slice taking its member's law. 0 (the default until the autotuner or this
 * call chooses): one launch per law and critical-stretch form, each
 * specialised to it. The reference's batch is the sequential loop over
 * random-field realisations
 * (randomfield/dynamicsolverdisplacementcontrolledRF.m:20). */
int bbpd_batch_set_mixing(bbpd_batch *b, int mixed);
int bbpd_batch_last_kernel_ms(bbpd_batch *b, float *ms);

/* Elapsed device time of the last bbpd_step / bbpd_step_async launch (ms). */
int bbpd_last_kernel_ms(bbpd_solver *s, float *ms);

/* Diagnostic: runs the device-side bounded wait used by the solver's grid
 * barriers on a word that nothing writes. Returns BBPD_ERR_TIMEOUT when the
 * wait expires after timeout_s and the kernel returns (the expected outcome). */
int bbpd_selftest_wait_timeout(double timeout_s);

/* Diagnostic: compares the kernels' correctly rounded division by a shared
 * divisor (Markstein's reciprocal and quotient corrections) with IEEE double
 * division on n seeded samples on the device; reports the mismatches of the
 * reciprocal and of the quotients, the samples compared, and the largest
 * relative error of the hardware reciprocal approximation. */
int bbpd_selftest_division(int64_t n, uint64_t seed, int64_t *recip_mismatches,
                           int64_t *quot_mismatches, int64_t *samples,
                           double *rcp_approx_max_relerr);

/* Diagnostic: the device's correctly rounded exp (the exponential law's exp,
 * in place of CUDA's, so that the law rounds like the reference's libm call,
 * calculatebsfexponentialMex.c:43) on n samples uniform in [lo, hi) drawn
 * from `seed` (splitmix64 of the sample index): reports how many results of
 * the fast double-double step differ from the 128-bit accurate step, and the
 * sum modulo 2^64 of the results' bit patterns, which the host build of the
 * same code reproduces for the same samples. */
int bbpd_selftest_exp(double lo, double hi, int64_t n, uint64_t seed, int64_t *fast_vs_accurate,
                      uint64_t *bits_sum);

/* Measurement: the device's FP64 issue rate, from independent chains of
 * fused multiply-adds timed with CUDA events over about seconds_target
 * seconds; reports FP64 FMA lane-operations per second (each one FP64
 * instruction for one thread; FLOP/s is twice that). The denominator of the
 * bench line's FP64 roofline. */
int bbpd_selftest_fp64_peak(double seconds_target, double *fma_lanes_per_s);

/* ===================================================================== *
 *  Synthetic beam builder (the inputs of input/scripts/Gregoire_beam_    *
 *  tests.m and the functions it calls, for a regular lattice).          *
 * ===================================================================== */

typedef struct bbpd_beam_spec {
    int32_t nx, ny, nz;          /* nodes along length x, width y, depth z */
    double dx;                   /* lattice spacing (m) */
    double horizon_factor;       /* horizon = factor * dx */
    double E;                    /* Young's modulus (Pa) */
    double stiffness_factor;     /* c = factor * E / (pi * horizon^4) */
    double density;              /* kg/m^3 */
    double support_x[2];         /* pinned bottom-layer node lines (m) */
    int32_t n_supports;
    int32_t load_midspan_top;    /* 1: z of the midspan top nodes prescribed */
    int32_t notch;               /* 1: remove bonds crossing the notch plane */
    int32_t sc_lognormal;        /* 1: per-bond sc ~ lognormal(sc_mean, sc_cov) */
    double notch_x;              /* notch plane position (m) */
    double notch_depth;          /* notch height from the bottom face (m) */
    double sc_mean, sc_cov;
    uint64_t seed;
} bbpd_beam_spec;

typedef struct bbpd_beam_scalars {
    int64_t n_nodes, n_bonds;
    double horizon, cell_volume, bond_stiffness_concrete, dt;
    int64_t n_supported, n_prescribed;
} bbpd_beam_scalars;

/* Sizes and scalars of a beam (no arrays). */
int bbpd_beam_count(const bbpd_beam_spec *spec, bbpd_beam_scalars *out);
/* Fill caller-allocated arrays (reference layouts): X (nNodes x 3), bondlist
 * (nBonds x 2), L0, BS, VCF (nBonds), nfam, density, mass (nNodes), CF, PF
 * (nNodes x 3) and, if sc_lognormal, sc (nBonds; may be NULL otherwise). */
int bbpd_beam_build(const bbpd_beam_spec *spec, double *X, double *bondlist,
                    double *L0, double *BS, double *VCF, double *nfam,
                    double *density, double *mass, double *CF, double *PF,
                    double *sc);

#ifdef __cplusplus
}
#endif

#endif
