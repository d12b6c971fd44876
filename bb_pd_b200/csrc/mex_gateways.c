/*
 * mexFunction gateways: drop-in replacements for the reference's MEX files.
 * Compile once per routine with -DGW_<Name> (bb_pd_b200/build.py does this
 * against the stub mex.h; with MATLAB: `mex -DGW_<Name> mex_gateways.c
 * -I<repo>/include -L<repo>/bb_pd_b200/lib -lbbpd`). Each gateway keeps the reference's argument
 * list, argument count check, size source (mxGetM of the same argument) and
 * in-place semantics, and calls libbbpd's host-pointer entry point, which runs
 * the routine on the GPU. Library errors become mexErrMsgTxt calls.
 */
#include <stdio.h>

#include "mex.h"
#include "bbpd.h"

static int registered;

static void release(void) { bbpd_release_mirrors(); }

static int check(int rc)
{
    if (!registered) { mexAtExit(release); registered = 1; }
    if (rc != BBPD_OK) {
        static char msg[512];
        snprintf(msg, sizeof(msg), "libbbpd: %s: %s\n", bbpd_status_string(rc), bbpd_last_error());
        mexErrMsgTxt(msg);
        return 1;
    }
    return 0;
}

#if defined(GW_calculatedeformedlengthMex)
/* [] = calculatedeformedlengthMex(deformedCoordinates, BONDLIST, undeformedLength,
 *        deformedLength, deformedX, deformedY, deformedZ, stretch)
 * calculatedeformedlengthMex.c:50-79 */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 8) { mexErrMsgTxt("Eight input arguments required \n"); return; }
    int64_t nNodes = (int64_t)mxGetM(prhs[0]);
    int64_t nBonds = (int64_t)mxGetM(prhs[1]);
    check(bbpd_calculatedeformedlength(mxGetPr(prhs[0]), mxGetPr(prhs[1]), mxGetPr(prhs[2]),
          nBonds, nNodes, mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]),
          mxGetPr(prhs[6]), mxGetPr(prhs[7])));
}

#elif defined(GW_calculatebsfexponentialMex)
/* [] = calculatebsfexponentialMex(stretch, s0, sc, k, alpha, bsf,
 *        bondSofteningFactor, BONDTYPE, flagBondSoftening)
 * calculatebsfexponentialMex.c:69-95 */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 9) { mexErrMsgTxt("Nine input arguments required \n"); return; }
    int64_t nBonds = (int64_t)mxGetM(prhs[0]);
    check(bbpd_calculatebsfexponential(mxGetPr(prhs[0]), mxGetPr(prhs[1]), mxGetPr(prhs[2]),
          mxGetScalar(prhs[3]), mxGetScalar(prhs[4]), mxGetPr(prhs[5]), mxGetPr(prhs[6]),
          mxGetPr(prhs[7]), mxGetPr(prhs[8]), nBonds));
}

#elif defined(GW_calculatebondforcesMex)
/* [] = calculatebondforcesMex(bForceX, bForceY, bForceZ, fail, deformedX, deformedY,
 *        deformedZ, deformedLength, stretch, stretchPlastic, BONDSTIFFNESS,
 *        cellVolume, VOLUMECORRECTIONFACTORS, bondSofteningFactor)
 * calculatebondforcesMex.c:48-79 */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 14) { mexErrMsgTxt("Fourteen input arguments required \n"); return; }
    int64_t nBonds = (int64_t)mxGetM(prhs[0]);
    check(bbpd_calculatebondforces(mxGetPr(prhs[0]), mxGetPr(prhs[1]), mxGetPr(prhs[2]),
          mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]), mxGetPr(prhs[6]),
          mxGetPr(prhs[7]), mxGetPr(prhs[8]), mxGetPr(prhs[9]), mxGetPr(prhs[10]),
          mxGetScalar(prhs[11]), mxGetPr(prhs[12]), mxGetPr(prhs[13]), nBonds));
}

#elif defined(GW_calculatenodalforcesopenmpMex)
/* [] = calculatenodalforcesopenmpMex(BONDLIST, nodalForce, bForceX, bForceY, bForceZ,
 *        nodalForceX, nodalForceY, nodalForceZ)
 * calculatenodalforcesopenmpMex.c:88-116. The per-thread scratch arrays
 * (arguments 6-8) are not needed: nodes sum their bonds in the order the
 * reference's 8 threads produce. They are accepted and left untouched. */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 8) { mexErrMsgTxt("Eight input arguments required \n"); return; }
    int64_t nNodes = (int64_t)mxGetM(prhs[1]);
    int64_t nBonds = (int64_t)mxGetM(prhs[0]);
    check(bbpd_calculatenodalforces(mxGetPr(prhs[0]), nBonds, nNodes, mxGetPr(prhs[1]),
          mxGetPr(prhs[2]), mxGetPr(prhs[3]), mxGetPr(prhs[4]), 8));
}

#elif defined(GW_calculatenodalforcesMex)
/* [] = calculatenodalforcesMex(BONDLIST, nodalForce, bForceX, bForceY, bForceZ)
 * calculatenodalforcesMex.c:49-73 (serial bond order) */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 5) { mexErrMsgTxt("Five input arguments required \n"); return; }
    int64_t nNodes = (int64_t)mxGetM(prhs[1]);
    int64_t nBonds = (int64_t)mxGetM(prhs[0]);
    check(bbpd_calculatenodalforces(mxGetPr(prhs[0]), nBonds, nNodes, mxGetPr(prhs[1]),
          mxGetPr(prhs[2]), mxGetPr(prhs[3]), mxGetPr(prhs[4]), 1));
}

#elif defined(GW_timeintegrationeulercromerMex)
/* [] = timeintegrationeulercromerMex(nodalAcceleration, nodalForce, DAMPING,
 *        nodalVelocity, DENSITY, constraintFLAG, DT, nodalDisplacement,
 *        deformedCoordinates, undeformedCoordinates)
 * timeintegrationeulercromerMex.c:56-85 */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 10) { mexErrMsgTxt("Ten input arguments required \n"); return; }
    int64_t nNodes = (int64_t)mxGetM(prhs[0]);
    int NOD = (int)mxGetN(prhs[0]);
    check(bbpd_timeintegrationeulercromer(mxGetPr(prhs[0]), mxGetPr(prhs[1]),
          mxGetScalar(prhs[2]), mxGetPr(prhs[3]), mxGetPr(prhs[4]), mxGetPr(prhs[5]),
          mxGetScalar(prhs[6]), mxGetPr(prhs[7]), mxGetPr(prhs[8]), mxGetPr(prhs[9]),
          nNodes, NOD));
}

#elif defined(GW_calculatebondfailureMex)
/* [fail] = calculatebondfailureMex(fail, failureFunctionality, BONDTYPE, stretch,
 *        criticalStretchConcrete, criticalStretchSteel)
 * calculatebondfailureMex.c:47-71 (fail updated in place) */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 6) { mexErrMsgTxt("Six input arguments required \n"); return; }
    int64_t nBonds = (int64_t)mxGetM(prhs[0]);
    check(bbpd_calculatebondfailure(mxGetPr(prhs[0]), mxGetScalar(prhs[1]), mxGetPr(prhs[2]),
          mxGetPr(prhs[3]), mxGetScalar(prhs[4]), mxGetScalar(prhs[5]), nBonds));
}

#else
#error "define GW_<Name> for one of the gateways"
#endif

#ifdef BBPD_MEXSTUB_MEX_H
/* Stub builds only: errors recorded by the stub mex.h of this translation unit. */
int mexstub_error_count(void) { return mexstub_errcount; }
const char *mexstub_error_message(void) { return mexstub_errmsg; }
#endif
