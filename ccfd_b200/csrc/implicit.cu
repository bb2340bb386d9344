// Implicit backward-Euler path (placeholder until the JFNK-GMRES kernels land).
#include "ccfd_ctx.cuh"

extern "C" int ccfd_run_implicit(ccfd_ctx* ctx, long nsteps, ccfd_report* report) {
    (void)ctx; (void)nsteps; (void)report;
    return CCFD_ERR_UNSUPPORTED;
}
