/*
 * ldp.h -- C ABI of the B200 trajectory engine for the single- and
 * double-barrier Langevin models of LangevinDynamicsForPCP.
 *
 * Plain C types only (no CUDA or torch types): a cgo / JNI / ctypes binding
 * can bind this header directly.  Every entry point returns an ldp_status;
 * none of them calls exit().  The library owns device memory and job
 * objects; the caller owns every host buffer and string it passes in.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   process entry  `mpirun ./langevinDynamics{Single,Double}Barrier -i x.inp`
 *                  src/langevinDynamicsSingleBarrier.cpp:6-252,
 *                  src/langevinDynamicsDoubleBarrier.cpp:6-270
 *   plugin seam    LangevinEquationSIMDMultiple (Initialize, Integrate,
 *                  Get*Average, GetStateCount, Write/ReadRestartFile)
 *                  src/langevinDynamicsSingleBarrier.h:823-2770,
 *                  src/langevinDynamicsDoubleBarrier.h:933-3410
 *   orchestration  LangevinEquationRunnerMPI::Setup/Run
 *                  src/langevinDynamicsSingleBarrier.h:3125-4039
 */
#ifndef LDP_H
#define LDP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LDP_ABI_VERSION 2
#define LDP_MAX_CG 16      /* FPTCG entries accepted per job              */
#define LDP_PATH_MAX 512   /* OUTPUTBASE / restart base name buffer sizes */

typedef enum ldp_status {
    LDP_OK = 0,
    LDP_ERR_INVALID = 1,     /* bad argument or inconsistent parameters      */
    LDP_ERR_NOMEM = 2,       /* device or host allocation failed / too large */
    LDP_ERR_DEVICE = 3,      /* CUDA error, or the CUDA library is missing   */
    LDP_ERR_TIMEOUT = 4,     /* a bounded wait ran out                       */
    LDP_ERR_IO = 5,          /* file could not be opened / written           */
    LDP_ERR_PARSE = 6,       /* .inp grammar or option error                 */
    LDP_ERR_UNSUPPORTED = 7, /* option combination not implemented           */
    LDP_ERR_NOT_READY = 8,   /* results asked for before the job finished    */
    LDP_ERR_RESTART = 9      /* restart file missing, corrupt or mismatched  */
} ldp_status;

typedef enum ldp_model { LDP_MODEL_SINGLE = 0, LDP_MODEL_DOUBLE = 1 } ldp_model;

typedef enum ldp_precision {
    LDP_PREC_FP64_PLAIN = 0,   /* FP64 state, one trajectory per thread      */
    LDP_PREC_FP32_BATCHED = 1  /* FP32 cell-local state, persistent kernel   */
} ldp_precision;

typedef enum ldp_mode {
    LDP_MODE_FIXED_STEPS = 0,   /* reference semantics: NUMBEROFSTEPS steps,
                                   renewal events recorded on the way        */
    LDP_MODE_FIRST_PASSAGE = 1  /* run each trajectory to its first
                                   bottom-to-different-bottom passage (FPT2
                                   event), capped at step_cap (censored)     */
} ldp_mode;

/*
 * One .inp file.  Field names follow the .inp keys; defaults are those of
 * the reference's AddOption calls (ldp_params_default).
 * Single model: barrier_heights[0][s] = BARRIERHEIGHTS s (state s),
 *               barrier_half_width[0] = BARRIERHALFWIDTH.
 * Double model: barrier_heights[b][s] = BARRIERHEIGHTSb s,
 *               barrier_half_width[b] = BARRIERHALFWIDTHb,
 *               barrier_position[b]   = BARRIERPOSITIONb.
 */
typedef struct ldp_params {
    int32_t model;                 /* ldp_model                              */
    int32_t overdamped;            /* OVERDAMPED                             */
    double x0, v0, gamma, kb, temperature, mass; /* X0 V0 GAMMA KB TEMPERATURE MASS */
    int32_t randomize_v;           /* RANDOMIZEV                             */
    double periodic_length;        /* PERIODICLENGTH                         */
    double barrier_heights[2][2];  /* see above                              */
    double barrier_half_width[2];
    double barrier_position[2];
    double timestep;               /* TIMESTEP                               */
    uint64_t number_of_steps;      /* NUMBEROFSTEPS                          */
    uint64_t number_of_previous_steps; /* NUMBEROFPREVIOUSSTEPS              */
    int32_t number_of_runs;        /* NUMBEROFRUNS (trials)                  */
    uint64_t freq_save;            /* FREQSAVE                               */
    uint64_t freq_stat;            /* FREQSTAT (accepted, ignored as in the reference) */
    int32_t distribution_v0;       /* DISTRIBUTIONV0                         */
    int32_t distribution_s0;       /* DISTRIBUTIONS0                         */
    double tau;                    /* TAU                                    */
    int32_t initial_state;         /* INITIALSTATE                           */
    int32_t randomize_states;      /* RANDOMIZESTATES                        */
    int32_t uniform_initial_states;/* UNIFORMINITALSTATES                    */
    int32_t eq;                    /* EQ (first value)                       */
    double eq_constant;            /* EQ (second value), K                   */
    int32_t waiting_time;          /* WAITINGTIME                            */
    int32_t fpt;                   /* FPT                                    */
    int32_t tpt;                   /* TPT                                    */
    int32_t fptcg;                 /* FPTCG flag (last entry's boolean)      */
    int32_t n_cg;                  /* number of FPTCG entries                */
    int32_t cg_sizes[LDP_MAX_CG];  /* FPTCG sizes                            */
    int32_t read_restart;          /* READRESTART                            */
    int32_t write_restart;         /* WRITERESTART                           */
    char input_restart[LDP_PATH_MAX];   /* INPUTRESTART                      */
    char output_restart[LDP_PATH_MAX];  /* OUTPUTRESTART                     */
    char output_base[LDP_PATH_MAX];     /* OUTPUTBASE                        */
    int32_t write_x;               /* WRITEX                                 */
    uint64_t number_of_log_samples;/* NUMBEROFLOGSAMPLES                     */
    int64_t random_seed;           /* RANDOMSEED (-1: time based)            */
    int32_t print_timer;           /* PRINTTIMER                             */
} ldp_params;

/* How a job is laid out and executed.  ntraj = ranks * runs * lanes. */
typedef struct ldp_job_opts {
    int32_t lanes;            /* trajectories per (rank, trial): the reference's
                                 SIMD width; default 8 (AVX-512 build)       */
    int32_t ranks;            /* virtual ranks (the reference's mpirun -n);
                                 default 1                                   */
    int32_t precision;        /* ldp_precision; default FP64_PLAIN           */
    int32_t mode;             /* ldp_mode; default FIXED_STEPS               */
    uint64_t step_cap;        /* FIRST_PASSAGE: max steps per trajectory     */
    int32_t table_slots;      /* per-trajectory cell-table ring slots (power
                                 of two, >= 16); default 256                 */
    int64_t tick_cap;         /* waiting-time ticks kept per trajectory;
                                 -1 = automatic, 0 = none                    */
    uint32_t job_id;          /* second Philox key word; default 0           */
    uint64_t steps_per_launch;/* 0 = automatic                               */
    int32_t block_size;       /* 0 = automatic                               */
    int32_t keep_frames;      /* keep x frames on the device after the MSD
                                 (needed for ldp_job_traj_results frames);
                                 default 1                                   */
    int32_t first_rank;       /* the job is virtual ranks first_rank ..
                                 first_rank + ranks - 1 of a larger run: its
                                 trajectory i draws the random streams of
                                 trajectory first_rank*runs*lanes + i, restart
                                 files and trajectory dumps carry the global
                                 rank, so ranks split over processes or GPUs
                                 give the whole run's trajectories; default 0 */
    int64_t event_cap;        /* per-event lists kept per trajectory and list
                                 (ldp_event_list; FP64 plain, fixed steps):
                                 the reference's per-lane event vectors that
                                 its .restart files hold.  0 = none (default);
                                 -1 = automatic when WRITERESTART is set     */
} ldp_job_opts;

/* Per-trajectory counters, laid out [field][ntraj]. */
enum ldp_count_field {
    LDP_C_FPT = 0,   /* bottom -> barrier top events                         */
    LDP_C_FPT2,      /* bottom -> different bottom events                    */
    LDP_C_TPT,       /* transition path (bottom -> top) events               */
    LDP_C_TPT2,      /* transition path (bottom -> other bottom) events      */
    LDP_C_INIT0,     /* FPT events whose initial barrier state was 0         */
    LDP_C_INIT1,     /* ... was 1                                            */
    LDP_C_INST0,     /* FPT events whose instantaneous barrier state was 0   */
    LDP_C_INST1,     /* ... was 1                                            */
    LDP_C_STATE0,    /* steps spent in state 0 (step 0 included)             */
    LDP_C_STATE1,    /* steps spent in state 1                               */
    LDP_C_WT,        /* waiting-time ticks recorded (may exceed tick_cap)    */
    LDP_C_EVICT,     /* cell-table ring evictions                            */
    LDP_C_FLAGS,     /* LDP_FLAG_* bits                                      */
    LDP_C_STEPS,     /* steps integrated by this trajectory                  */
    LDP_C_CG0,       /* FPTCG events, LDP_C_CG0 + j for FPTCG entry j        */
    LDP_NCOUNT = LDP_C_CG0 + LDP_MAX_CG
};

/* Per-trajectory event-time sums (FP64, event order), [field][ntraj]. */
enum ldp_sum_field {
    LDP_S_FPT = 0, LDP_S_FPT2, LDP_S_TPT, LDP_S_TPT2,
    LDP_S_FIRST_FPT,   /* duration of the trajectory's first FPT event  */
    LDP_S_FIRST_FPT2,  /* ... first FPT2 event                           */
    LDP_S_FIRST_TPT,   /* ... first TPT event                            */
    LDP_S_FIRST_TPT2,  /* ... first TPT2 event (0 while the count is 0)  */
    LDP_S_CG0,         /* LDP_S_CG0 + j */
    LDP_NSUM = LDP_S_CG0 + LDP_MAX_CG
};

#define LDP_FLAG_NONFINITE 1u   /* x became NaN/inf; trajectory frozen        */
#define LDP_FLAG_TICK_OVERFLOW 2u /* more waiting ticks than tick_cap          */
#define LDP_FLAG_CENSORED 4u    /* FIRST_PASSAGE: step_cap reached, no event  */
#define LDP_FLAG_EVENT_OVERFLOW 8u /* more events in a list than event_cap   */

/* Per-event lists (event durations in time units, event order), laid out
 * [list][ntraj][event_cap]: m_FirstPassageTime{,2}, m_TransitionPathTime{,2}
 * and m_FirstPassageTimeCG2 of each FPTCG entry
 * (src/langevinDynamicsSingleBarrier.h:2352-2590). */
enum ldp_event_list {
    LDP_E_FPT = 0, LDP_E_FPT2, LDP_E_TPT, LDP_E_TPT2,
    LDP_E_CG0          /* LDP_E_CG0 + j for FPTCG entry j; LDP_E_CG0 + n_cg lists */
};

typedef struct ldp_job_info {
    int64_t ntraj;        /* trajectories                                   */
    int64_t nframe;       /* frames per trajectory (NUMBEROFSTEPS/FREQSAVE+1) */
    int64_t nlag;         /* MSD lag points                                  */
    int64_t steps;        /* steps integrated per trajectory (fixed mode)    */
    int64_t tick_cap;     /* waiting ticks kept per trajectory               */
    int32_t n_cg;
    int32_t precision;
    int32_t mode;
    int32_t done;
    int64_t device_bytes; /* device memory the job holds while it runs      */
    int64_t event_cap;    /* events kept per trajectory and list            */
    int64_t steps_before; /* steps restored from a restart (0: fresh start) */
} ldp_job_info;

/*
 * Caller-allocated host buffers for per-trajectory results; any pointer may
 * be NULL to skip that array.  Frame arrays are [nframe][ntraj].
 */
typedef struct ldp_traj_results {
    int64_t *counts;        /* [LDP_NCOUNT][ntraj]                          */
    double  *sums;          /* [LDP_NSUM][ntraj]                            */
    int32_t *state0;        /* initial barrier state                        */
    double  *v0;            /* initial velocity instance                    */
    double  *x_final;       /* position after the last step                 */
    double  *v_final;
    int32_t *state_final;
    int64_t *ticks;         /* [ntraj][tick_cap] waiting-time ticks (steps) */
    double  *frames_x;      /* [nframe][ntraj]                              */
    double  *frames_v, *frames_f, *frames_barrier, *frames_pe, *frames_ke,
            *frames_state;  /* WRITEX series, [nframe][ntraj]               */
    double  *events;        /* [LDP_E_CG0 + n_cg][ntraj][event_cap]         */
    uint8_t *event_states;  /* [ntraj][event_cap]: per FPT event, bit 0 the
                               instantaneous and bit 1 the initial barrier
                               state (m_InstantBarrierList,
                               m_InitialBarrierList, S.h:2396-2404)         */
} ldp_traj_results;

typedef struct ldp_timing {
    double integrate_ms;    /* device time of the trajectory kernels         */
    double msd_ms;          /* device time of the MSD kernels                */
    double reduce_ms;       /* device time of the reduction kernels          */
    int64_t launches;       /* kernels launched                              */
    int64_t particle_steps; /* trajectory-steps integrated                   */
} ldp_timing;

typedef struct ldp_ctx ldp_ctx;
typedef struct ldp_job ldp_job;

/* Library / context.  Replaces MPIKERNEL::MPIKernel + runner construction
 * (src/mpiKernel.cpp:1-60, src/langevinDynamicsSingleBarrier.h:2890-3038). */
int         ldp_abi_version(void);
ldp_status  ldp_create(ldp_ctx **out, int device);
void        ldp_destroy(ldp_ctx *ctx);
const char *ldp_last_error(const ldp_ctx *ctx);
const char *ldp_status_string(ldp_status st);

/* Launch shape of the FP32 batched persistent kernel in this context:
 * threads per block, resident blocks per SM (0: as many as fit), step pairs
 * per slot and launch, and cell-table ring slots per resident slot (power of
 * two).  Zero keeps the default.  Must precede the context's first FP32
 * job.  No reference counterpart (the reference has no GPU launch). */
ldp_status  ldp_ctx_set_fp32_shape(ldp_ctx *ctx, int block, int blocks_per_sm, uint64_t pair_budget,
                                   int ring_slots);
/* Device-time markers on the context's stream (16 slots): record a marker,
 * then read the elapsed device time between two markers (waits for the
 * second).  They replace the reference's wall-clock timers around Integrate
 * (clsSystemTimeCPP, src/langevinDynamicsSingleBarrier.h:3416-3448). */
ldp_status  ldp_ctx_mark(ldp_ctx *ctx, int mark);
ldp_status  ldp_ctx_elapsed_ms(ldp_ctx *ctx, int mark_a, int mark_b, double *ms);
ldp_status  ldp_ctx_synchronize(ldp_ctx *ctx);
/* FP64 plain jobs in fixed-step mode with at most max_traj trajectories run
 * in latency mode: one CTA of two warps per trajectory, one warp drawing
 * the Gaussians and flip schedules of the next 32 steps while the other
 * integrates, for runs of few long trajectories (the reference's sample:
 * 16-32 trajectories x 3e9 steps), whose per-step dependency chain bounds
 * them.  Results are the same bit for bit either way.  0 disables it;
 * default 2048.  No reference counterpart. */
ldp_status  ldp_ctx_set_fp64_latency(ldp_ctx *ctx, int64_t max_traj);
/* FP64 plain fixed-step jobs above the latency-mode limit and of at most
 * max_traj trajectories run in group mode: a CTA of 32 trajectories, a
 * consumer warp stepping them (lane l one trajectory) while producer warps
 * draw their Gaussians and flip schedules ahead, for runs of a few thousand
 * trajectories.  Results are the same bit for bit.  0 disables it;
 * default 16384.  No reference counterpart. */
ldp_status  ldp_ctx_set_fp64_group(ldp_ctx *ctx, int64_t max_traj);
/* The shape in effect: the resolved values once the first FP32 job ran. */
ldp_status  ldp_ctx_get_fp32_shape(ldp_ctx *ctx, int *block, int *grid, uint64_t *pair_budget,
                                   int *ring_slots);

/* Parameters.  Replaces INPUTPARSER::InputParser::AddOption/Parse/
 * GetOptionValue (src/inputParser.cpp:45-330) as used by the two mains
 * (src/langevinDynamicsSingleBarrier.cpp:64-188). */
void        ldp_params_default(int model, ldp_params *p);
ldp_status  ldp_params_from_inp(const char *path, int model, ldp_params *p,
                                char *err, size_t errlen);
/* base_dir: the directory relative INCLUDE paths are opened from, at every
 * nesting level; NULL or "" opens them relative to the working directory,
 * as the reference does (src/inputParser.cpp:311) and ldp_params_from_inp
 * always does. */
ldp_status  ldp_params_from_inp_text(const char *text, const char *base_dir,
                                     int model, ldp_params *p,
                                     char *err, size_t errlen);
/* The reference's `-p` (InputParser::PrintAllValues, src/inputParser.cpp:
 * 188-196): every option of the parsed file in option-table order, one line
 * "%-20s %3d %s\n" per occurrence (key, occurrence index, its values joined
 * by single spaces), written to buf as a NUL-terminated string.  *needed
 * (if not NULL) receives the bytes required; LDP_ERR_NOMEM when buflen is
 * smaller.  On a parse error buf holds the message. */
ldp_status  ldp_inp_print_values(const char *path, int model, char *buf,
                                 size_t buflen, size_t *needed);
/* Writes the default .inp (the reference's `-o file.inp`,
 * src/inputParser.cpp:212-266). */
ldp_status  ldp_write_default_inp(const char *path, int model);

/* Jobs.  Replaces LangevinEquationSIMDMultiple::Initialize/Integrate and the
 * trial loop of LangevinEquationRunnerMPI::Run
 * (src/langevinDynamicsSingleBarrier.h:1276, 1386, 3429-3589). */
void        ldp_job_opts_default(ldp_job_opts *o);
ldp_status  ldp_job_create(ldp_ctx *ctx, const ldp_params *p,
                           const ldp_job_opts *o, ldp_job **out);
ldp_status  ldp_job_set_precision(ldp_job *job, int precision);
ldp_status  ldp_submit(ldp_ctx *ctx, ldp_job *job);   /* asynchronous      */
/* Submits several jobs at once: all FP32 batched jobs are registered in the
 * work queue before any launch, so their trajectories share every persistent
 * launch (the reference runs one .inp per mpirun; no counterpart). */
ldp_status  ldp_submit_batch(ldp_ctx *ctx, ldp_job **jobs, int njobs);
/* As ldp_submit_batch for FP32 batched jobs only, with every persistent
 * launch and every job's post-processing captured in one CUDA graph (launch
 * count: an upper bound that drains the queues), so the host is not involved
 * until the results.  The batch's device time is in the first job's timing.
 * A parameter scan runs as one graph launch (no counterpart in the
 * reference, which runs one .inp per process). */
ldp_status  ldp_submit_batch_graph(ldp_ctx *ctx, ldp_job **jobs, int njobs);
ldp_status  ldp_poll(ldp_ctx *ctx, ldp_job *job, int *done);
ldp_status  ldp_wait(ldp_ctx *ctx, ldp_job *job);
ldp_status  ldp_job_info_get(const ldp_job *job, ldp_job_info *info);
ldp_status  ldp_job_timing_get(const ldp_job *job, ldp_timing *t);
void        ldp_job_destroy(ldp_job *job);

/* Serving loop (continuous batching of FP32 batched jobs).  No counterpart
 * in the reference, which runs one .inp per MPI process (src/mpiKernel.cpp).
 * Requests are submitted at any time (ldp_server_submit is thread-safe);
 * each ldp_server_step admits queued jobs, oldest first, while their device
 * footprint fits hbm_budget (later jobs that fit may pass a waiting one for
 * at most 0.25 s), publishes their trajectories shortest-remaining-job
 * first in chunks, keeps short persistent launches in
 * flight for every model type with work, and finishes jobs whose
 * trajectories all retired.  Jobs joining mid-run share the launches with
 * those already running; every result equals that of the job run alone.
 * Drive it with ldp_server_step from one thread (the one that owns ctx). */
typedef struct ldp_server ldp_server;
typedef enum {
    LDP_SRV_QUEUED = 0, LDP_SRV_RUNNING = 1, LDP_SRV_FINISHING = 2, LDP_SRV_DONE = 3, LDP_SRV_FAILED = 4
} ldp_server_state;
typedef struct ldp_server_opts {
    int64_t hbm_budget;     /* bytes of job arenas resident at once (0: 80% of free memory,
                               counting what the device's memory pool holds unused)        */
    int64_t pair_budget;    /* step pairs per slot per persistent launch (0: 1024)           */
    int32_t max_inflight;   /* persistent launches in flight (1..16; each covers every
                               model type's queue)                                          */
    int32_t region;         /* 1 (default): allocate the budget once, at creation, as one
                               device region that admitted jobs' arenas are placed in (no
                               device allocation per job); 0: each arena from the device's
                               stream-ordered pool                                          */
} ldp_server_opts;
typedef struct ldp_server_info {
    int64_t queued, running, finishing, done;
    int64_t hbm_in_use, hbm_budget;
    int64_t launches;
    int64_t steps;            /* ldp_server_step calls                                      */
    /* Host seconds spent in each phase of ldp_server_step (admission
     * bookkeeping and arena allocation, registration, publication, launches,
     * completion, finished jobs): total and longest single call.          */
    double phase_s[6], phase_max_s[6];
} ldp_server_info;
void        ldp_server_opts_default(ldp_server_opts *o);
ldp_status  ldp_server_create(ldp_ctx *ctx, const ldp_server_opts *o, ldp_server **out);
ldp_status  ldp_server_submit(ldp_server *s, const ldp_params *p, const ldp_job_opts *o, uint64_t *ticket);
ldp_status  ldp_server_step(ldp_server *s, int *ndone);
/* state: ldp_server_state; latency_s: submission to done (0 until done). */
ldp_status  ldp_server_poll(ldp_server *s, uint64_t ticket, int *state, double *latency_s);
/* Tickets of jobs that ended (done or failed) since the last call, oldest
 * first: up to cap of them into tickets, *n = how many; with cap 0, *n = how
 * many are waiting (none taken).  A host loop driving many jobs polls only
 * these instead of every ticket. */
ldp_status  ldp_server_take_ended(ldp_server *s, uint64_t *tickets, int64_t cap, int64_t *n);
/* Seconds from submission to admission, to all trajectories retired, and to
 * done (-1 for a stage not reached yet): where a job's latency went. */
ldp_status  ldp_server_job_times(ldp_server *s, uint64_t ticket, double times[3]);
/* The finished job (owned by the server until ldp_server_release). */
ldp_status  ldp_server_job(ldp_server *s, uint64_t ticket, ldp_job **job);
ldp_status  ldp_server_release(ldp_server *s, uint64_t ticket);
ldp_status  ldp_server_info_get(ldp_server *s, ldp_server_info *info);
void        ldp_server_destroy(ldp_server *s);

/* Results.  Replaces the getters GetFirstPassageTimeAverage{,2},
 * GetTransitionPathTimeAverage{,2}, GetFirstPassageTimeCGAverage2,
 * GetStateCount, GetBarrierTick, GetX
 * (src/langevinDynamicsSingleBarrier.h:2632-2769). */
ldp_status  ldp_job_traj_results(ldp_job *job, ldp_traj_results *out);
/* MSD over all trajectories (MeanSquareDisplacementBruteForce summed and
 * divided by nrun, src/langevinDynamicsSingleBarrier.h:24-45, 3452-3461,
 * 3893-3912); lags in frames. */
ldp_status  ldp_job_msd(ldp_job *job, int64_t *lags, double *msd, int64_t nlag);
/* Per-trajectory mean event times (time units) of each event list, the
 * reference's getters GetFirstPassageTimeAverage{,2},
 * GetTransitionPathTimeAverage{,2} and GetFirstPassageTimeCGAverage2
 * (src/langevinDynamicsSingleBarrier.h:2722-2763): sum / count of the
 * list, 0 for a list without events (STATISTICS::AVERAGE,
 * src/STATISTICS.cpp:100-106); laid out [LDP_E_CG0 + n_cg][ntraj] in
 * ldp_event_list order.  Computed on the device: only the means are
 * copied. */
ldp_status  ldp_job_traj_means(ldp_job *job, double *means);
/* Per-trajectory MSD before the sum over trajectories (the reference's msd0
 * of one lane, S.h:3454-3455), [nlag][ntraj]. */
ldp_status  ldp_job_msd_traj(ldp_job *job, double *msd0);
/* Writes the reference's output files under dir (NULL: current directory):
 * src/langevinDynamicsSingleBarrier.h:3594-4036. */
ldp_status  ldp_job_write_outputs(ldp_job *job, const char *dir);

/*
 * FP64 plain integration that allocates nothing.  No counterpart in the
 * reference.  For callers that cannot allocate device memory -- a host
 * application or framework that owns the whole device-memory budget, a
 * real-time loop that cannot pay for an allocation (or the synchronization
 * that freeing implies), a plugin that may only use the buffers it is given.
 * The caller passes the parameters and its own device buffers for the
 * outputs: d_counts [LDP_NCOUNT][ntraj], d_sums [LDP_NSUM][ntraj],
 * d_x_final [ntraj], and optionally d_frames_x [nframe][ntraj] with
 * nframe = NUMBEROFSTEPS / FREQSAVE + 1 (NULL: no frames);
 * ntraj = ranks * NUMBEROFRUNS * lanes, at most LDP_NOALLOC_MAX_TRAJ.
 * o->table_slots (cell-table ring slots per trajectory, a power of two from
 * 16 to LDP_NOALLOC_MAX_SLOTS; ldp_job_opts_default gives 256) is honoured;
 * larger values are rejected with LDP_ERR_UNSUPPORTED.  o->block_size,
 * tick_cap and keep_frames are ignored (the FP64 kernels run 128-thread
 * blocks, as in a job); o->steps_per_launch is honoured as in a job.  The
 * working state lives in one fixed device array of the library (about
 * 18.5 MB, held by every GPU that loads the library's module until the
 * process exits); every call overwrites it, so calls whose device work
 * overlaps (other streams, other host threads) race on it -- serialize them.
 * The first call on a device (and the first after a cudaDeviceReset) looks
 * up that array's address in the current context; make it before any stream
 * capture.  The work is enqueued on `stream` (NULL: the current device's
 * default stream) on the current device; the call returns without waiting.
 * Results equal ldp_job_create/ldp_submit with LDP_PREC_FP64_PLAIN for the
 * same params, layout and table_slots; RANDOMSEED < 0 means seed 0 here;
 * WAITINGTIME, WRITEX series and event lists are not produced (event_cap
 * > 0 is rejected; 0 and -1, automatic, mean none here), and FP32 precision or first-passage mode is rejected.  Errors
 * come back as a status and a message in err.
 */
#define LDP_NOALLOC_MAX_TRAJ 4096
#define LDP_NOALLOC_MAX_SLOTS 256
ldp_status  ldp_integrate_fp64_noalloc(const ldp_params *p, const ldp_job_opts *o, int64_t *d_counts,
                                       double *d_sums, double *d_x_final, double *d_frames_x,
                                       void *stream, char *err, size_t errlen);

/*
 * Restart files (READRESTART / WRITERESTART / INPUTRESTART / OUTPUTRESTART):
 * one file per virtual rank and trial, <base>_%05d_%05d.restart, in the
 * layout of LangevinEquationSIMDMultiple::Write/ReadRestartFile
 * (src/langevinDynamicsSingleBarrier.h:385-820, 1048-1275;
 * src/langevinDynamicsDoubleBarrier.h:414-932, 1202-1447), FP64 plain jobs
 * in fixed-step mode.  ldp_job_restore loads the files into a created job
 * before ldp_submit (the job's NUMBEROFPREVIOUSSTEPS must equal the steps
 * the files hold; NUMBEROFSTEPS more steps follow, frames and statistics
 * continue the file's); ldp_job_save_restart writes them after the run
 * (the job needs event_cap > 0: the files hold every event).  Files written
 * here carry, after the reference's trailer, a block that makes a resumed
 * run equal the uninterrupted one bit for bit; files the reference wrote
 * resume with the same statistics (the barrier flips' pending steps are
 * drawn from the job's streams).
 */
typedef struct ldp_restart_summary {
    int32_t lanes;            /* SIMDWIDTH of the writer (lanes per file)    */
    int32_t rank;             /* the writer's rank                           */
    uint64_t steps;           /* steps done                                  */
    int64_t frames;           /* frames of the x series                      */
    int32_t has_exact_resume; /* written by this library                     */
    int32_t pad;
    int64_t ncell[2];         /* barrier-table cells (double model: two)     */
    int32_t min_id[2];        /* first cell index of each table              */
} ldp_restart_summary;
ldp_status  ldp_job_restore(ldp_job *job, const char *input_base);
/*
 * Continuation of FP32 batched runs (the chaining the reference does with
 * WRITERESTART / READRESTART, src/langevinDynamicsSingleBarrier.h:1048-1275,
 * whose .restart files hold per-event lists this path does not keep).
 * ldp_job_keep_state, before ldp_submit: the job keeps every trajectory's
 * state at its last step (~(40 + 16 x ring slots) device bytes per
 * trajectory).  ldp_job_save_state, after the run: writes that state, the
 * counts, duration sums, frames and waiting-time ticks to a file of this
 * library.  ldp_job_load_state, before ldp_submit: loads such a file into a
 * job of the same parameters, layout, RANDOMSEED and job id whose
 * NUMBEROFPREVIOUSSTEPS equals the steps the file holds (a multiple of 4);
 * NUMBEROFSTEPS more steps follow and the job can be saved again.  The
 * random streams are keyed by absolute step, so a chained run equals the
 * uninterrupted one bit for bit.  Fixed-step mode only.  No reference
 * counterpart for the file itself.
 */
ldp_status  ldp_job_keep_state(ldp_job *job);
ldp_status  ldp_job_save_state(ldp_job *job, const char *path);
ldp_status  ldp_job_load_state(ldp_job *job, const char *path);
ldp_status  ldp_job_save_restart(ldp_job *job, const char *output_base);
/* One file: its summary and, optionally, the per-lane counts and sums a
 * job restored from it starts with ([LDP_NCOUNT][lanes], [LDP_NSUM][lanes]).
 * p selects the layout (model, OVERDAMPED, TPT, FPTCG). */
ldp_status  ldp_restart_inspect(const ldp_params *p, const char *path, ldp_restart_summary *s,
                                int64_t *counts, double *sums, char *err, size_t errlen);
/* Reads a file and writes it again (a byte-identical copy for a file of
 * the same layout): validates a file against the layout. */
ldp_status  ldp_restart_rewrite(const ldp_params *p, const char *in, const char *out, char *err,
                                size_t errlen);

/* One-shot drop-in for `mpirun -n ranks ./exe -i path`. */
ldp_status  ldp_run_inp(ldp_ctx *ctx, const char *path, int model,
                        const ldp_job_opts *o, const char *outdir);

#ifdef __cplusplus
}
#endif
#endif /* LDP_H */
