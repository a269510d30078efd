// ldp_output.cpp -- reference output files (pending).
#include "ldp_internal.h"

extern "C" ldp_status ldp_job_write_outputs(ldp_job* job, const char* dir) {
    (void)job; (void)dir;
    return LDP_ERR_UNSUPPORTED;
}

extern "C" ldp_status ldp_run_inp(ldp_ctx* ctx, const char* path, int model, const ldp_job_opts* o,
                                  const char* outdir) {
    (void)ctx; (void)path; (void)model; (void)o; (void)outdir;
    return LDP_ERR_UNSUPPORTED;
}
