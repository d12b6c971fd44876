/*
 * Minimal stand-in for MATLAB's mex.h / matrix.h, used to compile and test
 * mexFunction gateways on machines without MATLAB.
 *
 * Only the calls that the BB_PD MEX gateways use are provided:
 * mxGetM, mxGetN, mxGetPr, mxGetScalar, mexErrMsgTxt and mexAtExit
 * (e.g. solvers/functions/mex/calculatedeformedlengthMex.c:58-74 of the
 * reference). An mxArray here is a real double matrix in column-major
 * order: {rows, cols, data}. Production builds compile the same gateway
 * sources against MATLAB's own headers instead.
 *
 * mexErrMsgTxt in MATLAB long-jumps back to the prompt. This stub cannot,
 * so it records the message and returns; gateways written for this library
 * therefore `return` right after every mexErrMsgTxt call.
 */
#ifndef BBPD_MEXSTUB_MEX_H
#define BBPD_MEXSTUB_MEX_H

#include <stddef.h>
#include <stdio.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag {
    size_t m;    /* rows    */
    size_t n;    /* columns */
    double *pr;  /* column-major data, m * n doubles */
} mxArray;

typedef size_t mwSize;

static inline size_t mxGetM(const mxArray *a) { return a->m; }
static inline size_t mxGetN(const mxArray *a) { return a->n; }
static inline double *mxGetPr(const mxArray *a) { return a->pr; }
static inline double mxGetScalar(const mxArray *a) { return a->pr[0]; }

/* One error slot per translation unit (each MEX file is its own shared object). */
static char mexstub_errmsg[256];
static int mexstub_errcount;

static inline void mexErrMsgTxt(const char *msg)
{
    strncpy(mexstub_errmsg, msg, sizeof(mexstub_errmsg) - 1);
    mexstub_errmsg[sizeof(mexstub_errmsg) - 1] = '\0';
    mexstub_errcount++;
    fprintf(stderr, "mexErrMsgTxt: %s", msg);
}

static inline int mexAtExit(void (*fn)(void)) { (void)fn; return 0; }

#ifdef __cplusplus
}
#endif

#endif
