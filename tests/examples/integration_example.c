/* Integration examples for C hosts, one after another as one function body
 * (each builds on the declarations of the ones before): creating a context
 * and a job from a .inp file, chaining runs through restart files, serving,
 * and the allocation-free entry point.  tests/test_integration_examples_cpu.py
 * compiles this file, so a renamed entry point, field or constant in
 * include/ldp.h makes it fail. */
#include "ldp.h"
#include <stddef.h>
void examples(void) {
ldp_ctx *ctx; ldp_params p; ldp_job_opts o; ldp_job *job; char err[512];
ldp_create(&ctx, 0);
ldp_params_from_inp("x.inp", LDP_MODEL_SINGLE, &p, err, sizeof err);
ldp_job_opts_default(&o); o.ranks = 4; o.lanes = 8;          /* 32 trajectories */
o.precision = LDP_PREC_FP32_BATCHED;                           /* or FP64_PLAIN  */
ldp_job_create(ctx, &p, &o, &job);
ldp_submit(ctx, job); ldp_wait(ctx, job);
ldp_job_write_outputs(job, ".");                               /* reference files */
ldp_job_destroy(job); ldp_destroy(ctx);
/* run 1: 3e9 steps, then checkpoint (event lists are what the files hold) */
o.event_cap = -1;                       /* automatic when WRITERESTART is true */
ldp_job_create(ctx, &p, &o, &job); ldp_submit(ctx, job); ldp_wait(ctx, job);
ldp_job_save_restart(job, "ck");        /* ck_00000_00000.restart, ...        */
/* run 2: NUMBEROFPREVIOUSSTEPS = 3e9, NUMBEROFSTEPS = what comes next */
ldp_job *job2;
p.number_of_previous_steps = 3000000000ull;
ldp_job_create(ctx, &p, &o, &job2);
ldp_job_restore(job2, "ck");            /* checks the files against p, as the reference */
ldp_submit(ctx, job2); ldp_wait(ctx, job2);   /* statistics and frames continue */
ldp_server *srv; ldp_server_opts so; uint64_t ticket; int state; double lat;
ldp_server_opts_default(&so); so.hbm_budget = 64LL << 30;      /* bytes      */
ldp_server_create(ctx, &so, &srv);
ldp_server_submit(srv, &p, &o, &ticket);        /* any time, any thread      */
for (;;) {                                      /* the thread owning ctx     */
    ldp_server_step(srv, NULL);
    ldp_server_poll(srv, ticket, &state, &lat);
    if (state == LDP_SRV_DONE) break;
}
ldp_server_job(srv, ticket, &job);              /* read results from job     */
ldp_server_release(srv, ticket);
ldp_server_destroy(srv);
}
