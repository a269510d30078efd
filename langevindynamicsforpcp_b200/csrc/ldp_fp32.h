// ldp_fp32.h -- FP32 batched persistent runtime: job table, work queue and
// slot state shared by the host scheduler and the persistent kernel.
//
// A "job" is one parameter set (one .inp) with its own output arrays; its
// trajectories are the work items.  Jobs of one model type (single/double x
// overdamped/underdamped) share one persistent kernel instance and one work
// queue.  Each resident thread ("slot") owns one trajectory at a time, holds
// its hot state in registers, and pulls the next trajectory from the queue
// when its trajectory retires (warp-aggregated claim).  Results never depend
// on which slot ran a trajectory: every random draw is keyed by
// (seed, job id, trajectory, step).
#pragma once
#include <cstdint>
#include <vector_types.h>
#include "ldp_engine.h"

namespace ldp {

constexpr int kFp32MaxJobs = 16384;     // resident jobs per queue
constexpr int kFp32MaxRanges = 1 << 20; // published item ranges per queue (one per job)

// Statistics switches of a job, folded for the kernel's event path.
enum : int32_t {
    EV_WT = 1,     // waiting times (single barrier, fixed steps)
    EV_FPT = 2,    // bottom-to-top first passages (single barrier, fixed steps)
    EV_FPT2 = 4,   // bottom-to-bottom first passages (FPT on, or FIRST_PASSAGE mode)
    EV_TPT = 8,    // transition paths (single barrier, fixed steps)
    EV_CG = 16,    // coarse-grained first passages (fixed steps)
    EV_FP = 32     // FIRST_PASSAGE mode: the first FPT2 event ends the trajectory
};

// Per-job constants and output pointers (device resident, one per job).
struct JobF {
    // model switches (jobs of one queue share dbl/over)
    int32_t eta, eq, rs, rv, us, init_state, wt, fpt, tpt, cg, n_cg, write_x, at_bottom, fp_mode;
    int32_t lanes, nruns, slots_log2;
    int32_t evm;         // EV_* statistics switches of the event path
    int32_t cg_size[LDP_MAX_CG];
    uint32_t key0, key1;
    uint32_t g0;         // stream index of the job's trajectory 0 (first_rank * runs * lanes)
    // FP32 step constants
    float L, halfL, w, slope[2], xb[2], lo0, hi1, xc, sN[2][2], sP[2][2];
    float c_drift, sig_r, hdt_invM, hdt, expg, sig_v;
    float bm_k;          // Box-Muller radius scale: -2 ln2 sigma^2 (sigma of the step noise)
    float a_lapf, c_lapf[2];  // catch-up flip probability c (1 - e^{a lap}) in FP32
    float invLf;         // 1 / L
    float bp[8];         // force breakpoints in [-L/2, L/2], ascending (cell edges included)
    int32_t nbp, pad1;
    // The bands next to the cell edges, (-L/2, edge_lo) and (edge_hi, L/2),
    // and whether the force is zero in both (no barrier flank reaches the
    // cell edge): then a crossing of the cell edge lands in a known flat
    // band (the hot loop's light step).
    float edge_lo, edge_hi;
    int32_t edge_flat, pad2;
    // FP64 constants (step 0, events, frames)
    double x0, v0, dt, Ld, invL, sig_v0, sig_r_d, a_lap, c_lap[2], p_first, p_cell0, mhalf;
    double Hs[2], Hd[2][2], iN[2][2], iP[2][2], sNd[2][2], sPd[2][2], wd, xbd[2], lo0d, hi1d, xcd;
    uint64_t T_eq, T_as[2];
    double ln1m[2];      // log(1 - per-step flip probability) by state; 0: never flips
    uint64_t nsteps, freq_save;
    int64_t nframe, tick_cap, ntraj;
    // per-trajectory outputs [field][ntraj] (job local)
    int64_t* counts;     // [LDP_NCOUNT][ntraj]
    int64_t* ssum;       // [LDP_NSUM][ntraj] event durations in steps
    int32_t* state0;
    double *v0s, *x_final, *v_final;
    int32_t* state_final;
    int64_t* ticks;      // [ntraj][tick_cap]
    double *fx, *fv, *ff, *fb, *fpe, *fke, *fst;  // frames [nframe][ntraj]
    // per-trajectory cold statistics state (touched only on events)
    int32_t* bits;
    int64_t *fpt_last, *fpt2_last, *tpt_last, *tpt2_last, *wt_tick;
    int32_t *init_idx0, *init_idx1, *idx2_0, *idx2_1, *tpt2_well;
    int64_t* cg_last;    // [LDP_MAX_CG][ntraj]
    int32_t* cg_well;    // [LDP_MAX_CG][ntraj]
    unsigned long long* remaining;   // trajectories of this job not yet retired
    // Continuation state at a trajectory's last step (kept when ck_xp is set:
    // ldp_job_keep_state), and the resume of a job continuing from it
    // (resume: ldp_job_load_state): position, velocity (underdamped) or the
    // previous random force (overdamped), cell, slot word (local barrier,
    // cache, eviction), the cached cell and its pending flip, the current
    // barrier's pending flip, the cell-table ring [ring slots][ntraj].
    float *ck_xp, *ck_rv;
    int32_t *ck_cell, *ck_sw, *ck_ckey;
    int64_t *ck_cflip, *ck_nflip;
    longlong2* ck_ring;
    uint64_t step0;      // the job's first step (1; S + 1 after S previous steps)
    int32_t resume, pad3;
};

// A work queue: published item ranges (job index, trajectory count) with
// inclusive prefix ends; head is claimed by the kernel, tail by the host.
struct QueueDev {
    int64_t* range_end;     // [kFp32MaxRanges] prefix sums of published items
    int32_t* range_job;     // [kFp32MaxRanges]
    int64_t* range_first;   // [kFp32MaxRanges] first trajectory of the range
    unsigned long long* head;  // claimed items
    unsigned long long* tail;  // published items (written by the host)
    int32_t* nranges;       // published ranges (written by the host)
    JobF* jobs;             // [kFp32MaxJobs]
};

// Per-slot state saved between launches, [nslots].
struct SlotsDev {
    int64_t nslots;
    int32_t* job;           // -1: no trajectory
    int64_t* traj;
    int64_t* step;          // next step to integrate (odd: launches end on step pairs)
    float *xp, *rv;         // rv: R_prev (overdamped) or v (underdamped)
    int32_t *cell, *st;     // st: state | slot flags << 1 (local barrier, cache, eviction)
    int32_t* ckey;          // key of the cell left last (cached state)
    int64_t* cflip;         // its pending flip step when it was left
    int64_t *sc1, *since;   // completed state-1 steps; start of the current state-1 run
    int32_t *cgw, *fidx;    // well of the last FPTCG evaluation; index of the next frame
    int64_t* nxf;           // step of the next frame
    int64_t* nflip;         // step of the current barrier's next flip
    longlong2* ring;        // [R][nslots] cell table: {key, stamp << 1 | state}
    unsigned long long* retired;   // total retired trajectories (all jobs)
    int32_t ring_slots;
};

// The four model types' queues and one set of slots shared by them, for the
// mixed persistent kernel (the serving loop's launches); wtype[w] is the
// type warp w serves (-1: none); sm_type[smid & (kMixedSmTypes - 1)] the type
// the warps of an SM take first when they pick one (-1: none), so that an SM
// runs one type's code at a time.
constexpr int kMixedSmTypes = 1024;
struct MixedDev {
    QueueDev q[4];
    SlotsDev S;
    int32_t* wtype;
    int32_t* sm_type;
    int64_t nwarps;
};

// Appends published work: clamps head to the old tail, sets tail and nranges.
int launch_fp32_publish(const QueueDev& q, unsigned long long new_tail, int32_t new_nranges, void* stream);
// Resident blocks per SM of the persistent kernel (0 on error).
int fp32_blocks_per_sm(bool dbl, bool over, int block);
int launch_fp32_persistent(bool dbl, bool over, const QueueDev& q, const SlotsDev& s, uint32_t pair_budget,
                           int grid, int block, void* stream);
// Resident 256-thread blocks per SM of the mixed kernel, and its launch.
int fp32_mixed_blocks_per_sm(int block);
int launch_fp32_mixed(const MixedDev& m, uint32_t pair_budget, int grid, int block, void* stream);

}  // namespace ldp
