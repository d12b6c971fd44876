// Error reporting, status strings and defaults for libbbpd.
#include "bbpd_internal.h"

#include <cuda_runtime.h>

#include <cstring>

namespace bbpd {

static thread_local char g_err[1024];

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_err[0] = '\0'; }

int require_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(BBPD_ERR_NO_DEVICE, "no CUDA device visible (%s); libbbpd has no CPU path",
                    e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    }
    return BBPD_OK;
}

}  // namespace bbpd

extern "C" const char *bbpd_last_error(void) { return bbpd::g_err; }

extern "C" const char *bbpd_status_string(int s)
{
    switch (s) {
    case BBPD_OK: return "ok";
    case BBPD_ERR_ARG: return "invalid argument";
    case BBPD_ERR_CUDA: return "CUDA error";
    case BBPD_ERR_OOM: return "device out of memory";
    case BBPD_ERR_TIMEOUT: return "device wait timed out";
    case BBPD_ERR_NONFINITE: return "non-finite displacement or velocity";
    case BBPD_ERR_UNSUPPORTED: return "unsupported input";
    case BBPD_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
    }
}

extern "C" int bbpd_abi_version(void) { return BBPD_ABI_VERSION; }

extern "C" int bbpd_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" void bbpd_params_default(bbpd_params *p)
{
    std::memset(p, 0, sizeof(*p));
    p->law = BBPD_LAW_EXPONENTIAL;
    p->scheme = BBPD_SCHEME_EULERCROMER;
    p->precision = BBPD_PREC_FP64;
    p->n_chunks = 8;                 // calculatenodalforcesopenmpMex.c:39
    p->amplitude = BBPD_AMP_LINEAR;
    p->node_order = BBPD_ORDER_INPUT;
    p->cell_volume = 1.0;
    p->dt = 1.0;
    p->damping = 0.0;                // Gregoire_beam_tests.m:247
    p->s0 = 1.0e-4;
    p->s1 = 3.0e-4;
    p->sc = 2.0e-3;
    p->sc_steel = 1.0;               // Gregoire_beam_tests.m:213
    p->k_exp = 25.0;                 // dynamicsolverdisplacementcontrolled.m:87
    p->alpha_exp = 0.25;
    p->beta_tri = 0.25;              // calculatebsftrilinear.m:41
    p->failure_functionality = 0.0;  // dynamicsolverconfiguration.m:11-13 ('on')
    p->guard_band = 1.0e-5;
    p->barrier_timeout_s = 2.0;
}
