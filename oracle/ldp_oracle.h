/*
 * ldp_oracle.h -- CPU oracle for the trajectory hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the
 * checker.  The product (langevindynamicsforpcp_b200) never links it.
 *
 * It restates, in scalar FP64 C, the per-step semantics of the reference's
 * engines on the product's per-trajectory Philox4x32-10 streams, so that the
 * FP64 device path can be compared with it trajectory for trajectory.
 */
#ifndef LDP_ORACLE_H
#define LDP_ORACLE_H
#include <stdint.h>
#include "../include/ldp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ldpo_cfg {
    int64_t traj_begin, traj_end; /* global trajectory indices to simulate */
    int32_t lanes, ranks;         /* g = (rank*runs + trial)*lanes + lane  */
    int32_t table_slots;          /* ring slots (power of two)             */
    int64_t tick_cap;             /* waiting ticks kept per trajectory     */
    uint32_t seed;                /* Philox key word 0                     */
    uint32_t job_id;              /* Philox key word 1                     */
    int32_t mode;                 /* ldp_mode                              */
    uint64_t step_cap;            /* FIRST_PASSAGE cap                     */
    int64_t event_cap;            /* per-event lists kept (0: none)        */
} ldpo_cfg;

void     ldpo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double   ldpo_log(double u);
void     ldpo_sincos2pi(double t, double *s, double *c);
double   ldpo_expm1(double x);
uint64_t ldpo_prob_to_u64(double p);
uint64_t ldpo_flip_wait(uint32_t hi, uint32_t lo, double ln1m);
/* "Never" for a flip step: fits the cell table's (step << 1 | state). */
#define LDPO_NEVER ((int64_t)((1ull << 62) - 1))
int64_t  ldpo_schedule(uint64_t s, uint32_t hi, uint32_t lo, double ln1m);

/* Steps integrated per trajectory and frames recorded, as the reference's
 * Integrate loop does them (S.h:1403-1511). */
uint64_t ldpo_effective_steps(const ldp_params *p);
int64_t  ldpo_nframe(const ldp_params *p);
/* MOLUTILITY::GenerateLog10Scale as called by Run (S.h:3324-3326). */
int64_t  ldpo_lags(const ldp_params *p, int64_t *lags, int64_t cap);

/* Simulates trajectories [traj_begin, traj_end); arrays in out are laid out
 * for n = traj_end - traj_begin trajectories.  Returns 0 on success. */
int      ldpo_run(const ldp_params *p, const ldpo_cfg *c, ldp_traj_results *out);

/* Per-trajectory MSD (MeanSquareDisplacementBruteForce, S.h:24-45):
 * frames [nframe][ntraj], msd0 [nlag][ntraj].  Origins are summed as 32
 * interleaved partial sums combined by a fixed tree (see the definition). */
void     ldpo_msd_traj(const double *frames, int64_t nframe, int64_t ntraj,
                       const int64_t *lags, int64_t nlag, double *msd0);

#ifdef __cplusplus
}
#endif
#endif
