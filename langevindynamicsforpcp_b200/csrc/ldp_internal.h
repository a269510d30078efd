// ldp_internal.h -- library-private definitions of the opaque C ABI handles.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <mutex>
#include <string>
#include <vector>

#include "ldp_engine.h"

namespace ldp {
struct Fp32Runtime;
}

constexpr int kCtxMarks = 16;
constexpr int kCtxF64Streams = 2;   // streams FP64 plain jobs of a batch share
// FP64 plain fixed-step jobs of at most this many trajectories run in
// latency mode (a CTA per trajectory) by default, jobs above that and up to
// kFp64GroupMaxTraj in group mode (32 trajectories per CTA with producer
// warps), larger ones one trajectory per thread.  On the reference's sample
// shape (particle-steps/s): 1024 trajectories 6.2e9 / 2.8e9 / 1.1e9
// (latency / group / thread), 4096: 7.2e9 / 1.12e10 / 4.4e9, 8192: 7.3e9 /
// 2.05e10 / 8.8e9, 16384: - / 2.75e10 / 1.72e10, 32768: - / 2.81e10 / 3.07e10.
constexpr int64_t kFp64LatencyMaxTraj = 2048;
constexpr int64_t kFp64GroupMaxTraj = 16384;

struct ldp_ctx {
    cudaEvent_t marks[kCtxMarks] = {};   // ldp_ctx_mark / ldp_ctx_elapsed_ms
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    std::mutex mu;
    std::string err;
    // FP32 batched path: runtime (queues, slots) and its launch shape.
    ldp::Fp32Runtime* fp32 = nullptr;
    int fp32_block = 0;            // threads per block (0: default 256)
    int fp32_blocks_per_sm = 0;    // resident blocks per SM (0: default 4)
    uint64_t fp32_pair_budget = 0; // step pairs per slot per launch (0: default)
    int fp32_ring_slots = 0;       // cell-table ring slots per slot (0: default 64)
    int64_t fp64_latency_max = kFp64LatencyMaxTraj;   // latency mode up to this many trajectories
    int64_t fp64_group_max = kFp64GroupMaxTraj;       // then group mode up to this many
    cudaStream_t side = nullptr;   // post-processing beside running batches (high priority)
    cudaStream_t rd = nullptr;     // result reads of finished jobs, beside running work
    // pinned staging for result reads (two halves, copied to the caller's
    // buffer while the next half lands), allocated at the first read
    char* hstage = nullptr;
    cudaEvent_t hstage_ev[2] = {nullptr, nullptr};
    cudaStream_t gside = nullptr;  // side branch captured into batch graphs
    cudaEvent_t gjoin = nullptr;   // joins that branch back before the capture ends
    // FP64 plain jobs of a batch: forked from `stream`, joined back to it.
    cudaStream_t f64s[kCtxF64Streams] = {};
    cudaEvent_t f64j[kCtxF64Streams] = {};
    cudaEvent_t f64fork = nullptr;
};

struct ldp_job {
    ldp_ctx* ctx = nullptr;
    ldp_params p{};
    ldp_job_opts o{};
    ldp::KConst k{};
    int64_t ntraj = 0;
    int64_t nframe = 0;
    uint64_t nsteps = 0;
    uint32_t seed = 0;
    std::vector<int64_t> lags;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    bool arena_owned = false;    // allocated by the job (else placed by its owner)
    ldp::TrajState st{};
    double* d_msd0 = nullptr;
    double* d_msd = nullptr;
    int64_t* d_lags = nullptr;
    void* d_aux = nullptr;   // 4 KiB of job-private device scratch
    double* d_means = nullptr;   // per-trajectory mean event times [list][ntraj]
    int64_t* d_ssum = nullptr;   // FP32 batched: event durations in steps [LDP_NSUM][ntraj]
    int32_t* d_i32b = nullptr;   // FP32 batched: 32-bit statistics state
    int fp32_type = -1;          // FP32 batched: queue (dbl*2 + over) the job is in
    int fp32_slot = -1;          // FP32 batched: index in that queue's job table
    int64_t fp32_published = 0;  // FP32 batched: trajectories published to the queue
    bool finalized = false;      // results post-processed after completion
    int fp32_phase = 0;          // 0 idle, 1 integrating, 2 finalizing, 3 in a batch graph
    cudaGraphExec_t gexec = nullptr;   // batch graph this job owns (first job of the batch)
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool submitted = false;
    bool rem_snapshot = false;   // FP32 batched: counter copied to d_aux before post-processing
    bool done = false;
    int64_t launches = 0;
    int64_t steps_total = 0;
    double wall_start = 0.0;
    bool restored = false;       // state loaded by ldp_job_restore
    uint64_t steps_before = 0;   // steps the restart files held
    // FP32 batched continuation (ldp_job_keep_state / ldp_job_load_state)
    bool keep_state = false;     // keep each trajectory's state at its last step
    bool fp32_resume = false;    // continue from a loaded state
    int ck_ring_slots = 0;       // ring slots of the kept state
    float *ck_xp = nullptr, *ck_rv = nullptr;
    int32_t *ck_cell = nullptr, *ck_sw = nullptr, *ck_ckey = nullptr;
    int64_t *ck_cflip = nullptr, *ck_nflip = nullptr;
    void* ck_ring = nullptr;
    bool ev_auto = false;        // event_cap / tick_cap chosen by the library
    bool tick_auto = false;
    int64_t particle_steps_done() const;
};

void ldp_set_error(ldp_ctx* ctx, const char* fmt, ...);

namespace ldp {
int fp32_register(ldp_job* job, cudaStream_t stream = nullptr, bool publish = true);
int fp32_publish_range(ldp_job* job, int64_t count, cudaStream_t stream = nullptr);
int fp32_pump(ldp_job* job, int nlaunch);
int fp32_estimate_launches(const ldp_job* job);
int fp32_launch_bound(ldp_ctx* ctx, int type, double total_pairs, double max_pairs);
int fp32_remaining(ldp_job* job, unsigned long long* rem);
int fp32_type_of(const ldp_job* job);
int fp32_launch_type(ldp_ctx* ctx, int type, uint32_t pair_budget, cudaStream_t st);
// One launch of the mixed kernel over all four types' queues (serving).
int fp32_launch_mixed(ldp_ctx* ctx, uint32_t pair_budget, cudaStream_t st);
int64_t fp32_mixed_slots(ldp_ctx* ctx);
int fp32_copy_remaining(ldp_ctx* ctx, int type, unsigned long long* host, unsigned long long* head,
                        cudaStream_t st);
int64_t fp32_nslots(ldp_ctx* ctx, int type);
unsigned long long fp32_published(ldp_ctx* ctx, int type);
int fp32_finalize(ldp_job* job, cudaStream_t stream = nullptr, bool lean = false);
// Whether every job in the type's queue has finished (or it has none): the
// queue's items are then exactly those published after this call.
bool fp32_queue_quiet(ldp_ctx* ctx, int type);
// Stream-ordered copy of the job's "not yet retired" counter to dst.
int fp32_snapshot_remaining(ldp_job* job, unsigned long long* dst, cudaStream_t stream);
void fp32_release(ldp_job* job);
void fp32_destroy_runtime(ldp_ctx* ctx);
}  // namespace ldp
std::vector<int64_t> ldp_lag_grid(const ldp_params& p);
// Job creation without the free-memory check, and the job's device arena
// (size, or allocation): the serving loop admits jobs by footprint itself.
ldp_status ldp_job_create_unchecked(ldp_ctx* ctx, const ldp_params* p, const ldp_job_opts* o, ldp_job** out);
size_t ldp_job_arena(ldp_job* job, bool alloc);
// Lays the job's arena out at `base` (ldp_job_arena(job, false) bytes owned
// by the caller, who keeps them until the job is destroyed) and zeroes it.
size_t ldp_job_arena_at(ldp_job* job, void* base);
