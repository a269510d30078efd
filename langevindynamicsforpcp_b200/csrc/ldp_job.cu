// ldp_job.cu -- contexts, jobs and the C ABI entry points of include/ldp.h.
//
// A job is one .inp run: ranks x runs x lanes trajectories (the reference's
// nrun, src/langevinDynamicsSingleBarrier.h:3226-3227).  ldp_submit enqueues
// the whole run on the context's stream -- init kernel, the chunked step
// kernels, then the MSD kernels -- and returns; ldp_poll / ldp_wait observe a
// completion event.  Device memory is one arena per job.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <string>
#include <vector>

#include "ldp_engine.h"
#include "ldp_internal.h"
#include "ldp_msd.h"

using namespace ldp;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void ldp_set_error(ldp_ctx* ctx, const char* fmt, ...) {
    if (!ctx) return;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->err = buf;
}

#define CUDA_OR_FAIL(ctx, call)                                                                  \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            ldp_set_error((ctx), "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                          __LINE__);                                                             \
            return LDP_ERR_DEVICE;                                                               \
        }                                                                                        \
    } while (0)

extern "C" int ldp_abi_version(void) { return LDP_ABI_VERSION; }

extern "C" const char* ldp_status_string(ldp_status st) {
    switch (st) {
        case LDP_OK: return "ok";
        case LDP_ERR_INVALID: return "invalid argument";
        case LDP_ERR_NOMEM: return "out of memory";
        case LDP_ERR_DEVICE: return "device error";
        case LDP_ERR_TIMEOUT: return "timeout";
        case LDP_ERR_IO: return "i/o error";
        case LDP_ERR_PARSE: return "parse error";
        case LDP_ERR_UNSUPPORTED: return "unsupported";
        case LDP_ERR_NOT_READY: return "not ready";
        case LDP_ERR_RESTART: return "restart error";
    }
    return "unknown";
}

extern "C" ldp_status ldp_create(ldp_ctx** out, int device) {
    if (!out) return LDP_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return LDP_ERR_DEVICE;
    if (device < 0 || device >= ndev) return LDP_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return LDP_ERR_DEVICE;
    ldp_ctx* ctx = new ldp_ctx();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return LDP_ERR_DEVICE;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    ctx->sm_count = prop.multiProcessorCount;
    // Keep freed job arenas in the stream-ordered pool.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    for (int i = 0; i < kCtxMarks; ++i) cudaEventCreate(&ctx->marks[i]);
    *out = ctx;
    return LDP_OK;
}

extern "C" void ldp_destroy(ldp_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (cudaStream_t* x : {&ctx->side, &ctx->rd, &ctx->gside})
        if (*x) {
            cudaStreamSynchronize(*x);
            cudaStreamDestroy(*x);
        }
    for (int k = 0; k < kCtxF64Streams; ++k) {
        if (ctx->f64s[k]) {
            cudaStreamSynchronize(ctx->f64s[k]);
            cudaStreamDestroy(ctx->f64s[k]);
        }
        if (ctx->f64j[k]) cudaEventDestroy(ctx->f64j[k]);
    }
    if (ctx->f64fork) cudaEventDestroy(ctx->f64fork);
    if (ctx->hstage) cudaFreeHost(ctx->hstage);
    for (cudaEvent_t e : ctx->hstage_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->gjoin) cudaEventDestroy(ctx->gjoin);
    fp32_destroy_runtime(ctx);
    for (int i = 0; i < kCtxMarks; ++i)
        if (ctx->marks[i]) cudaEventDestroy(ctx->marks[i]);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" const char* ldp_last_error(const ldp_ctx* ctx) {
    if (!ctx) return "no context";
    return ctx->err.c_str();
}

// ---------------------------------------------------------------------------
// defaults
// ---------------------------------------------------------------------------
extern "C" void ldp_params_default(int model, ldp_params* p) {
    // AddOption defaults, src/langevinDynamicsSingleBarrier.cpp:65-108 and
    // src/langevinDynamicsDoubleBarrier.cpp:65-125.
    std::memset(p, 0, sizeof(*p));
    p->model = model;
    p->overdamped = 0;
    p->x0 = 0.0;
    p->v0 = 1.0;
    p->gamma = 1.0;
    p->kb = 1.0;
    p->temperature = 1.0;
    p->mass = 1.0;
    p->randomize_v = 1;
    p->periodic_length = 10.0;
    p->barrier_heights[0][0] = 2.0;
    p->barrier_heights[0][1] = 6.0;
    p->barrier_heights[1][0] = 2.0;
    p->barrier_heights[1][1] = 6.0;
    p->barrier_half_width[0] = 1.0;
    p->barrier_half_width[1] = 1.0;
    p->barrier_position[0] = 1.0;
    p->barrier_position[1] = 2.0;
    p->timestep = 0.1;
    p->number_of_steps = 10000;
    p->number_of_previous_steps = 0;
    p->number_of_runs = 1;
    p->freq_save = 1;
    p->freq_stat = 1;
    p->distribution_v0 = 0;
    p->distribution_s0 = 0;
    p->tau = 0.1;
    p->initial_state = 0;
    p->randomize_states = 1;
    p->uniform_initial_states = 0;
    p->eq = 1;
    p->eq_constant = 1.0;
    p->waiting_time = 0;
    p->fpt = 0;
    p->tpt = 0;
    p->fptcg = 0;          // default FPTCG entry "false 10"
    p->n_cg = 1;
    p->cg_sizes[0] = 10;
    p->read_restart = 0;
    p->write_restart = 0;
    std::snprintf(p->input_restart, LDP_PATH_MAX, "%s", "inputRestart");
    std::snprintf(p->output_restart, LDP_PATH_MAX, "%s", "outputRestart");
    // Both mains default OUTPUTBASE to the single-barrier name.
    std::snprintf(p->output_base, LDP_PATH_MAX, "%s", "langevinDynamicsSingleBarrier");
    p->write_x = 0;
    p->number_of_log_samples = 20;
    p->random_seed = -1;
    p->print_timer = 0;
}

extern "C" void ldp_job_opts_default(ldp_job_opts* o) {
    std::memset(o, 0, sizeof(*o));
    o->lanes = 8;
    o->ranks = 1;
    o->precision = LDP_PREC_FP64_PLAIN;
    o->mode = LDP_MODE_FIXED_STEPS;
    o->step_cap = 100000000ull;
    o->table_slots = 256;
    o->tick_cap = -1;
    o->job_id = 0;
    o->steps_per_launch = 0;
    o->block_size = 0;
    o->keep_frames = 1;
    o->first_rank = 0;
    o->event_cap = -1;
}

// ---------------------------------------------------------------------------
// lag grid: GenerateLog10Scale (src/MOLUTILITY.cpp:59-73) with the frame
// count of Run (S.h:3220, includes NUMBEROFPREVIOUSSTEPS).
// ---------------------------------------------------------------------------
std::vector<int64_t> ldp_lag_grid(const ldp_params& p) {
    std::vector<int64_t> out;
    const uint64_t nf = (p.number_of_steps + p.number_of_previous_steps) / p.freq_save + 1;
    const double ts = p.timestep * (double)p.freq_save;
    const double step = 1.0 / (double)p.number_of_log_samples;
    const double maxTime = ts * (double)(nf - 1000);
    const double t0 = std::log10(ts), t1 = std::log10(maxTime);
    out.push_back(0);
    for (double t = t0; t <= t1; t += step) {
        const int64_t iv = (int64_t)(uint64_t)std::round(std::pow(10.0, t) / ts);
        if (out.back() != iv) out.push_back(iv);
    }
    return out;
}

// ---------------------------------------------------------------------------
// jobs
// ---------------------------------------------------------------------------
static ldp_status validate(ldp_ctx* ctx, const ldp_params& p, const ldp_job_opts& o, bool fixed) {
    if (p.model != LDP_MODEL_SINGLE && p.model != LDP_MODEL_DOUBLE) {
        ldp_set_error(ctx, "unknown model %d", p.model);
        return LDP_ERR_INVALID;
    }
    if (o.lanes < 1 || o.ranks < 1 || p.number_of_runs < 1) {
        ldp_set_error(ctx, "lanes, ranks and NUMBEROFRUNS must be >= 1");
        return LDP_ERR_INVALID;
    }
    if (o.first_rank < 0 ||
        ((int64_t)o.first_rank + o.ranks) * (int64_t)p.number_of_runs * o.lanes > ((int64_t)1 << 32)) {
        ldp_set_error(ctx, "first_rank must be >= 0 and (first_rank + ranks) x runs x lanes at most 2^32");
        return LDP_ERR_INVALID;
    }
    if (o.table_slots < 16 || (o.table_slots & (o.table_slots - 1))) {
        ldp_set_error(ctx, "table_slots must be a power of two >= 16 (got %d)", o.table_slots);
        return LDP_ERR_INVALID;
    }
    if (!(p.timestep > 0.0) || !(p.periodic_length > 0.0) || !(p.mass > 0.0) || !(p.gamma > 0.0)) {
        ldp_set_error(ctx, "TIMESTEP, PERIODICLENGTH, MASS and GAMMA must be positive");
        return LDP_ERR_INVALID;
    }
    if (p.freq_save < 1) {
        ldp_set_error(ctx, "FREQSAVE must be >= 1");
        return LDP_ERR_INVALID;
    }
    if (p.n_cg < 0 || p.n_cg > LDP_MAX_CG) {
        ldp_set_error(ctx, "at most %d FPTCG entries are supported", LDP_MAX_CG);
        return LDP_ERR_UNSUPPORTED;
    }
    for (int j = 0; j < p.n_cg; ++j)
        if (p.cg_sizes[j] == 0) {
            ldp_set_error(ctx, "FPTCG size must be non-zero");
            return LDP_ERR_INVALID;
        }
    if (p.tau < 0.0) {
        ldp_set_error(ctx, "TAU must be >= 0");
        return LDP_ERR_INVALID;
    }
    if (!p.eq && !(p.eq_constant > 0.0)) {
        ldp_set_error(ctx, "EQ constant must be positive");
        return LDP_ERR_INVALID;
    }
    if (p.model == LDP_MODEL_SINGLE && !(p.barrier_half_width[0] > 0.0)) {
        ldp_set_error(ctx, "BARRIERHALFWIDTH must be positive");
        return LDP_ERR_INVALID;
    }
    const bool plain = o.precision == LDP_PREC_FP64_PLAIN;
    if (p.number_of_previous_steps && !fixed) {
        ldp_set_error(ctx, "NUMBEROFPREVIOUSSTEPS (a continued run) needs fixed-step mode");
        return LDP_ERR_UNSUPPORTED;
    }
    if (o.event_cap > 0 && !(plain && fixed)) {
        ldp_set_error(ctx, "per-event lists (event_cap) need the FP64 plain path in fixed-step mode");
        return LDP_ERR_UNSUPPORTED;
    }
    if (fixed) {
        const uint64_t nf = (p.number_of_steps + p.number_of_previous_steps) / p.freq_save + 1;
        if (nf < 1000) {
            // S.h:3221-3224
            ldp_set_error(ctx, "numberOfFrame < 1000");
            return LDP_ERR_INVALID;
        }
    } else if (o.step_cap < 1) {
        ldp_set_error(ctx, "step_cap must be >= 1");
        return LDP_ERR_INVALID;
    }
    return LDP_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device arena of a job.  With alloc == false only the size is computed.
// FP64 plain jobs hold their whole trajectory state and cell-table rings;
// FP32 batched jobs hold outputs and the per-trajectory statistics state
// touched on events (their hot state lives in the persistent slots).
static size_t job_arena(ldp_job* job, bool alloc, void* at = nullptr) {
    const ldp_params* p = &job->p;
    const bool fixed = job->o.mode == LDP_MODE_FIXED_STEPS;
    const bool f32 = job->o.precision == LDP_PREC_FP32_BATCHED;
    const int64_t n = job->ntraj;
    const int ncg_rows = std::max(1, p->n_cg);
    const int nser = (fixed ? 1 : 0) + ((fixed && p->write_x) ? 6 : 0);
    const int64_t nlag = (int64_t)job->lags.size();
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o0 = off; off += align256(bytes); return o0; };
    const size_t o_d = take(sizeof(double) * 9 * n);
    const size_t o_i64 = take(sizeof(int64_t) * 9 * n);
    const size_t o_i32 = take(sizeof(int32_t) * 4 * n);
    const size_t o_cg = take(sizeof(double) * ncg_rows * n);
    const size_t o_cgw = take(sizeof(int64_t) * ncg_rows * n);
    const size_t o_cnt = take(sizeof(int64_t) * LDP_NCOUNT * n);
    const size_t o_sum = take(sizeof(double) * LDP_NSUM * n);
    const size_t o_ring = take(f32 ? 0 : sizeof(int64_t) * 2 * (size_t)job->o.table_slots * n);
    const size_t o_tick = take(sizeof(int64_t) * (size_t)std::max<int64_t>(job->o.tick_cap, 1) * n);
    const size_t ev_elems = (size_t)std::max<int64_t>(job->o.event_cap, 0) * n;
    const size_t o_ev = take(sizeof(double) * (LDP_E_CG0 + p->n_cg) * ev_elems);
    const size_t o_evst = take(ev_elems);
    const size_t o_fr = take(sizeof(double) * (size_t)std::max<int64_t>(job->nframe, 1) * n * std::max(nser, 1));
    const size_t o_msd0 = take(sizeof(double) * (size_t)std::max<int64_t>(nlag, 1) * n);
    const size_t o_msd = take(sizeof(double) * (size_t)std::max<int64_t>(nlag, 1));
    const size_t o_lag = take(sizeof(int64_t) * (size_t)std::max<int64_t>(nlag, 1));
    const size_t o_aux = take(4096);
    const size_t o_mean = take(sizeof(double) * (LDP_E_CG0 + p->n_cg) * n);
    // FP32 batched extras: integer event-duration sums and 32-bit cell indices.
    const size_t o_ssum = take(f32 ? sizeof(int64_t) * LDP_NSUM * n : 0);
    const size_t o_i32b = take(f32 ? sizeof(int32_t) * (5 + ncg_rows) * n : 0);
    // FP32 continuation state (ldp_job_keep_state)
    const bool ck = f32 && job->keep_state;
    const int ckR = ck ? job->ck_ring_slots : 0;
    const size_t o_ck32 = take(ck ? sizeof(int32_t) * 5 * n : 0);       // xp, rv, cell, sw, ckey
    const size_t o_ck64 = take(ck ? sizeof(int64_t) * 2 * n : 0);       // cflip, nflip
    const size_t o_ckr = take(ck ? sizeof(int64_t) * 2 * (size_t)ckR * n : 0);
    if (!alloc) return off;
    job->arena_bytes = off;
    // Stream-ordered allocation from the device pool: jobs created and freed
    // in a loop reuse the same memory without a device synchronization.
    cudaStream_t st = job->ctx->stream;
    if (at) {
        job->arena = at;
        job->arena_owned = false;
    } else if (cudaMallocAsync(&job->arena, off, st) != cudaSuccess) {
        job->arena = nullptr;
        return 0;
    } else {
        job->arena_owned = true;
    }
    if (cudaMemsetAsync(job->arena, 0, off, st) != cudaSuccess) {
        if (job->arena_owned) cudaFreeAsync(job->arena, st);
        job->arena = nullptr;
        return 0;
    }
    char* a = (char*)job->arena;
    TrajState& S = job->st;
    S.n = n;
    double* dd = (double*)(a + o_d);
    S.x = dd; S.v = dd + n; S.F = dd + 2 * n; S.rprev = dd + 3 * n; S.fpt_last = dd + 4 * n;
    S.fpt2_last = dd + 5 * n; S.tpt_last = dd + 6 * n; S.tpt2_last = dd + 7 * n; S.v0 = dd + 8 * n;
    int64_t* ii = (int64_t*)(a + o_i64);
    S.cell = ii; S.well = ii + n; S.init_idx0 = ii + 2 * n; S.init_idx1 = ii + 3 * n; S.idx2_0 = ii + 4 * n;
    S.idx2_1 = ii + 5 * n; S.tpt2_well = ii + 6 * n; S.wt_tick = ii + 7 * n; S.nflip = ii + 8 * n;
    int32_t* i32 = (int32_t*)(a + o_i32);
    S.state = i32; S.lb = i32 + n; S.bits = i32 + 2 * n; S.state0 = i32 + 3 * n;
    S.cg_last = (double*)(a + o_cg);
    S.cg_well = (int64_t*)(a + o_cgw);
    S.counts = (int64_t*)(a + o_cnt);
    S.sums = (double*)(a + o_sum);
    S.ring_tag = f32 ? nullptr : (int64_t*)(a + o_ring);
    S.ring_data = f32 ? nullptr : S.ring_tag + (size_t)job->o.table_slots * n;
    S.ticks = (int64_t*)(a + o_tick);
    S.ev = ev_elems ? (double*)(a + o_ev) : nullptr;
    S.ev_st = ev_elems ? (uint8_t*)(a + o_evst) : nullptr;
    double* fr = (double*)(a + o_fr);
    const size_t fstride = (size_t)std::max<int64_t>(job->nframe, 1) * n;
    S.fx = fixed ? fr : nullptr;
    S.fv = S.ff = S.fb = S.fpe = S.fke = S.fst = nullptr;
    if (fixed && p->write_x) {
        S.fv = fr + 1 * fstride; S.ff = fr + 2 * fstride; S.fb = fr + 3 * fstride;
        S.fpe = fr + 4 * fstride; S.fke = fr + 5 * fstride; S.fst = fr + 6 * fstride;
    }
    job->d_msd0 = (double*)(a + o_msd0);
    job->d_msd = (double*)(a + o_msd);
    job->d_lags = (int64_t*)(a + o_lag);
    job->d_aux = (void*)(a + o_aux);
    job->d_means = (double*)(a + o_mean);
    job->d_ssum = f32 ? (int64_t*)(a + o_ssum) : nullptr;
    job->d_i32b = f32 ? (int32_t*)(a + o_i32b) : nullptr;
    if (ck) {
        int32_t* c32 = (int32_t*)(a + o_ck32);
        job->ck_xp = (float*)c32; job->ck_rv = (float*)(c32 + n); job->ck_cell = c32 + 2 * n;
        job->ck_sw = c32 + 3 * n; job->ck_ckey = c32 + 4 * n;
        int64_t* c64 = (int64_t*)(a + o_ck64);
        job->ck_cflip = c64; job->ck_nflip = c64 + n;
        job->ck_ring = (void*)(a + o_ckr);
    }
    if (nlag > 0 &&
        cudaMemcpyAsync(job->d_lags, job->lags.data(), sizeof(int64_t) * nlag, cudaMemcpyHostToDevice, st) !=
            cudaSuccess) {
        if (job->arena_owned) cudaFreeAsync(job->arena, st);
        job->arena = nullptr;
        return 0;
    }
    return off;
}

size_t ldp_job_arena(ldp_job* job, bool alloc) { return job_arena(job, alloc); }
size_t ldp_job_arena_at(ldp_job* job, void* base) { return job_arena(job, true, base); }

static ldp_status job_create(ldp_ctx* ctx, const ldp_params* p, const ldp_job_opts* o, ldp_job** out, bool check_mem);

extern "C" ldp_status ldp_job_create(ldp_ctx* ctx, const ldp_params* p, const ldp_job_opts* o, ldp_job** out) {
    return job_create(ctx, p, o, out, true);
}

ldp_status ldp_job_create_unchecked(ldp_ctx* ctx, const ldp_params* p, const ldp_job_opts* o, ldp_job** out) {
    return job_create(ctx, p, o, out, false);
}

static ldp_status job_create(ldp_ctx* ctx, const ldp_params* p, const ldp_job_opts* o, ldp_job** out, bool check_mem) {
    if (!ctx || !p || !out) return LDP_ERR_INVALID;
    *out = nullptr;
    ldp_job_opts opts;
    if (o) opts = *o; else ldp_job_opts_default(&opts);
    const bool fixed = opts.mode == LDP_MODE_FIXED_STEPS;
    ldp_status st = validate(ctx, *p, opts, fixed);
    if (st != LDP_OK) return st;

    ldp_job* job = new ldp_job();
    job->ctx = ctx;
    job->p = *p;
    job->o = opts;
    job->ntraj = (int64_t)opts.ranks * p->number_of_runs * opts.lanes;
    if (job->ntraj > (int64_t)0xffffffffll) {
        delete job;
        ldp_set_error(ctx, "at most 2^32 trajectories per job");
        return LDP_ERR_INVALID;
    }
    if (p->random_seed < 0) job->seed = (uint32_t)time(nullptr);
    else job->seed = (uint32_t)p->random_seed;
    job->nsteps = fixed ? effective_steps(*p) : opts.step_cap;
    job->nframe = fixed ? frame_count(*p) : 0;
    if (fixed) {
        job->lags = ldp_lag_grid(*p);
        if (job->lags.size() < 20) {
            // S.h:3327-3332
            ldp_set_error(ctx, "interval is less than 20 (%zu)", job->lags.size());
            delete job;
            return LDP_ERR_INVALID;
        }
    }
    int64_t n = job->ntraj;
    job->ev_auto = job->o.event_cap < 0;
    job->tick_auto = job->o.tick_cap < 0;
    const bool wt = p->waiting_time && p->model == LDP_MODEL_SINGLE && fixed;
    if (!wt) job->o.tick_cap = 0;
    else if (job->o.tick_cap < 0) {
        int64_t a = (int64_t)std::max<uint64_t>(64, job->nsteps / 2000);
        int64_t b = std::max<int64_t>(64, ((int64_t)1 << 27) / n);
        job->o.tick_cap = std::min(a, b);
    }
    if (job->o.event_cap < 0) {
        // Enough for about one event per 10^4 steps (the quick_test model
        // records one FPT event per ~4*10^5 steps), within 2^28 list entries.
        const int64_t lists = LDP_E_CG0 + p->n_cg;
        const int64_t a = std::max<int64_t>(64, (int64_t)(job->nsteps / 10000));
        const int64_t b = std::max<int64_t>(64, ((int64_t)1 << 28) / (n * lists));
        job->o.event_cap = (p->write_restart && fixed && opts.precision == LDP_PREC_FP64_PLAIN) ? std::min(a, b) : 0;
    }
    prepare_kconst(job->p, job->o, job->seed, &job->k);
    job->k.tick_cap = job->o.tick_cap;
    job->k.ev_cap = job->o.event_cap;

    const size_t need = job_arena(job, false);
    cudaSetDevice(ctx->device);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if (check_mem && need + ((size_t)256 << 20) > free_b) {
        ldp_set_error(ctx, "job needs %.2f GB of device memory, %.2f GB free", need / 1e9, free_b / 1e9);
        delete job;
        return LDP_ERR_NOMEM;
    }
    for (int i = 0; i < 4; ++i) cudaEventCreate(&job->ev[i]);
    *out = job;
    return LDP_OK;
}

extern "C" ldp_status ldp_job_set_precision(ldp_job* job, int precision) {
    if (!job) return LDP_ERR_INVALID;
    if (precision != LDP_PREC_FP64_PLAIN && precision != LDP_PREC_FP32_BATCHED) return LDP_ERR_INVALID;
    if (job->submitted || job->arena) return LDP_ERR_INVALID;
    if (precision == LDP_PREC_FP32_BATCHED && job->o.event_cap > 0) {
        ldp_set_error(job->ctx, "per-event lists need the FP64 plain path");
        return LDP_ERR_UNSUPPORTED;
    }
    job->o.precision = precision;
    return LDP_OK;
}

static uint64_t auto_steps_per_launch(const ldp_job* job) {
    if (job->o.steps_per_launch) return job->o.steps_per_launch;
    // Aim at ~2^31 trajectory-steps per launch: short enough for progress and
    // bounded kernels, long enough that the per-launch state traffic
    // (~200 B per trajectory) is negligible.
    uint64_t s = (uint64_t)(((int64_t)1 << 31) / std::max<int64_t>(job->ntraj, 1));
    s = std::max<uint64_t>(s, 4096);
    s = std::min<uint64_t>(s, (uint64_t)1 << 24);
    return s;
}

// Enqueues a job's work on stream s (the context's stream, or for FP64
// plain jobs of a batch one of the context's FP64 batch streams).
static ldp_status submit_on(ldp_ctx* ctx, ldp_job* job, cudaStream_t s) {
    if (!ctx || !job) return LDP_ERR_INVALID;
    if (job->submitted) {
        ldp_set_error(ctx, "job already submitted");
        return LDP_ERR_INVALID;
    }
    CUDA_OR_FAIL(ctx, cudaSetDevice(ctx->device));
    if (!job->arena && job_arena(job, true) == 0) {
        ldp_set_error(ctx, "cudaMalloc of %zu bytes failed", job_arena(job, false));
        return LDP_ERR_NOMEM;
    }
    if (job->p.number_of_previous_steps && !job->restored) {
        ldp_set_error(ctx, "NUMBEROFPREVIOUSSTEPS > 0 continues a run: call ldp_job_restore (FP64 plain) or "
                           "ldp_job_load_state (FP32 batched) first");
        return LDP_ERR_INVALID;
    }
    job->submitted = true;
    job->launches = 0;
    if (job->o.precision == LDP_PREC_FP32_BATCHED) {
        int e = fp32_register(job);
        if (!e) e = (int)cudaEventRecord(job->ev[0], s);
        if (!e) e = fp32_pump(job, fp32_estimate_launches(job));
        if (!e) e = (int)cudaEventRecord(job->ev[1], s);
        if (!e) e = (int)cudaEventRecord(job->ev[2], s);
        if (e) {
            ldp_set_error(ctx, "FP32 batched launch failed: %s", cudaGetErrorString((cudaError_t)e));
            return LDP_ERR_DEVICE;
        }
        job->fp32_phase = 1;
        return LDP_OK;
    } else {
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[0], s));
        int e = 0;
        if (!job->restored) {
            e = launch_fp64_init(job->k, job->st, job->k.g0, job->o.block_size, s);
            if (e) {
                ldp_set_error(ctx, "init launch failed: %s", cudaGetErrorString((cudaError_t)e));
                return LDP_ERR_DEVICE;
            }
            ++job->launches;
        }
        // Steps continue the restart's numbering (S.h:1420: iStep =
        // m_NumberOfStepDonePreviously + ...): the streams are keyed by it.
        const uint64_t spl = auto_steps_per_launch(job);
        const uint64_t first = job->steps_before + 1, last = job->steps_before + job->nsteps;
        // Few trajectories: latency mode (same results bit for bit).
        const bool fixed = job->o.mode == LDP_MODE_FIXED_STEPS;
        const bool latency = fixed && job->ntraj <= ctx->fp64_latency_max;
        const bool group = fixed && !latency && job->ntraj <= ctx->fp64_group_max;
        for (uint64_t s0 = first; s0 <= last; s0 += spl) {
            const uint64_t s1 = std::min<uint64_t>(s0 + spl, last + 1);
            e = latency ? launch_fp64_latency(job->k, job->st, job->k.g0, s0, s1, s)
                : group ? launch_fp64_group(job->k, job->st, job->k.g0, s0, s1, s)
                        : launch_fp64_steps(job->k, job->st, job->k.g0, s0, s1, job->o.block_size, s);
            if (e) {
                ldp_set_error(ctx, "step launch failed: %s", cudaGetErrorString((cudaError_t)e));
                return LDP_ERR_DEVICE;
            }
            ++job->launches;
        }
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[1], s));
    }
    if (job->o.mode == LDP_MODE_FIXED_STEPS && !job->lags.empty()) {
        int e = launch_msd(job->st.fx, job->nframe, job->ntraj, job->d_lags, (int64_t)job->lags.size(), job->d_msd0,
                           job->d_msd, s, LDP_MSD_FP64);
        if (e) {
            ldp_set_error(ctx, "MSD launch failed: %s", cudaGetErrorString((cudaError_t)e));
            return LDP_ERR_DEVICE;
        }
        job->launches += 2;
    }
    CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[2], s));
    return LDP_OK;
}

extern "C" ldp_status ldp_ctx_set_fp64_latency(ldp_ctx* ctx, int64_t max_traj) {
    if (!ctx || max_traj < 0) return LDP_ERR_INVALID;
    ctx->fp64_latency_max = max_traj;
    return LDP_OK;
}

extern "C" ldp_status ldp_ctx_set_fp64_group(ldp_ctx* ctx, int64_t max_traj) {
    if (!ctx || max_traj < 0) return LDP_ERR_INVALID;
    ctx->fp64_group_max = max_traj;
    return LDP_OK;
}

extern "C" ldp_status ldp_submit(ldp_ctx* ctx, ldp_job* job) {
    if (!ctx) return LDP_ERR_INVALID;
    return submit_on(ctx, job, ctx->stream);
}

// FP32 batched jobs advance in rounds: when the launches enqueued so far
// have drained, either more are enqueued (trajectories remain) or the
// post-processing is (all retired).
static ldp_status fp32_advance(ldp_ctx* ctx, ldp_job* job, int* done) {
    *done = 0;
    if (job->fp32_phase == 1) {
        unsigned long long rem = 0;
        CUDA_OR_FAIL(ctx, (cudaError_t)fp32_remaining(job, &rem));
        if (rem > 0) {
            const double frac = (double)rem / (double)std::max<int64_t>(job->ntraj, 1);
            const int n = std::max(1, (int)(fp32_estimate_launches(job) * frac) + 1);
            CUDA_OR_FAIL(ctx, (cudaError_t)fp32_pump(job, n));
            CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[1], ctx->stream));
            CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[2], ctx->stream));
            return LDP_OK;
        }
        CUDA_OR_FAIL(ctx, (cudaError_t)fp32_finalize(job));
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[2], ctx->stream));
        job->fp32_phase = 2;
        return LDP_OK;
    }
    if (job->fp32_phase == 3) {
        // The batch ran every launch its bound allows before the job's
        // post-processing; all trajectories must have retired by then (the
        // counter as copied just before the post-processing, when taken).
        unsigned long long rem = 0;
        if (job->rem_snapshot) {
            CUDA_OR_FAIL(ctx, cudaMemcpy(&rem, job->d_aux, sizeof(rem), cudaMemcpyDeviceToHost));
        } else {
            CUDA_OR_FAIL(ctx, (cudaError_t)fp32_remaining(job, &rem));
        }
        if (rem > 0) {
            ldp_set_error(ctx, "%llu trajectories not retired after the batch's launch bound", rem);
            return LDP_ERR_DEVICE;
        }
    }
    job->fp32_phase = 0;
    fp32_release(job);
    *done = 1;
    return LDP_OK;
}

extern "C" ldp_status ldp_poll(ldp_ctx* ctx, ldp_job* job, int* done) {
    if (!ctx || !job || !done) return LDP_ERR_INVALID;
    *done = 0;
    if (!job->submitted) return LDP_ERR_NOT_READY;
    if (job->done) {
        *done = 1;
        return LDP_OK;
    }
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaEventQuery(job->ev[2]);
    if (e == cudaErrorNotReady) return LDP_OK;
    if (e != cudaSuccess) {
        ldp_set_error(ctx, "device error: %s", cudaGetErrorString(e));
        return LDP_ERR_DEVICE;
    }
    if (job->fp32_phase) {
        ldp_status st = fp32_advance(ctx, job, done);
        if (st != LDP_OK || !*done) return st;
    }
    *done = 1;
    job->done = true;
    return LDP_OK;
}

extern "C" ldp_status ldp_wait(ldp_ctx* ctx, ldp_job* job) {
    if (!ctx || !job) return LDP_ERR_INVALID;
    if (!job->submitted) return LDP_ERR_NOT_READY;
    cudaSetDevice(ctx->device);
    for (;;) {
        CUDA_OR_FAIL(ctx, cudaEventSynchronize(job->ev[2]));
        int done = 0;
        ldp_status st = ldp_poll(ctx, job, &done);
        if (st != LDP_OK) return st;
        if (done) return LDP_OK;
    }
}

extern "C" ldp_status ldp_job_info_get(const ldp_job* job, ldp_job_info* info) {
    if (!job || !info) return LDP_ERR_INVALID;
    info->ntraj = job->ntraj;
    info->nframe = job->nframe;
    info->nlag = (int64_t)job->lags.size();
    info->steps = (int64_t)job->nsteps;
    info->tick_cap = job->o.tick_cap;
    info->n_cg = job->p.n_cg;
    info->precision = job->o.precision;
    info->mode = job->o.mode;
    info->done = job->done ? 1 : 0;
    info->device_bytes = (int64_t)job_arena(const_cast<ldp_job*>(job), false);
    info->event_cap = job->o.event_cap;
    info->steps_before = (int64_t)job->steps_before;
    return LDP_OK;
}

extern "C" ldp_status ldp_job_timing_get(const ldp_job* job, ldp_timing* t) {
    if (!job || !t) return LDP_ERR_INVALID;
    if (!job->done) return LDP_ERR_NOT_READY;
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, job->ev[0], job->ev[1]);
    cudaEventElapsedTime(&b, job->ev[1], job->ev[2]);
    t->integrate_ms = a;
    t->msd_ms = b;
    t->reduce_ms = 0.0;
    t->launches = job->launches;
    t->particle_steps = job->particle_steps_done();
    return LDP_OK;
}

int64_t ldp_job::particle_steps_done() const {
    if (o.mode == LDP_MODE_FIXED_STEPS) return ntraj * (int64_t)nsteps;
    return steps_total;
}

extern "C" void ldp_job_destroy(ldp_job* job) {
    if (!job) return;
    cudaSetDevice(job->ctx->device);
    if (job->submitted && !job->done) ldp_wait(job->ctx, job);
    fp32_release(job);
    if (job->gexec) cudaGraphExecDestroy(job->gexec);
    for (int i = 0; i < 4; ++i)
        if (job->ev[i]) cudaEventDestroy(job->ev[i]);
    if (job->arena && job->arena_owned) cudaFreeAsync(job->arena, job->ctx->stream);
    delete job;
}

// The stream result reads of finished jobs go on: its own, so that a read
// does not queue behind later jobs' launches on the context's stream.
static cudaError_t read_stream(ldp_ctx* ctx, cudaStream_t* s) {
    if (!ctx->rd) {
        int lo_prio = 0, hi_prio = 0;
        cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
        const cudaError_t e = cudaStreamCreateWithPriority(&ctx->rd, cudaStreamNonBlocking, hi_prio);
        if (e != cudaSuccess) return e;
    }
    *s = ctx->rd;
    return cudaSuccess;
}

// Device-to-host copy of a finished job's results into the caller's
// (pageable) buffer through the context's pinned staging halves: the DMA of
// one half overlaps the host copy of the other, and the DMA runs at pinned
// speed whatever the caller's memory.  Without staging (pinned allocation
// refused) a plain copy.
static constexpr size_t kStageHalf = (size_t)8 << 20;
static ldp_status copy_d2h_on(ldp_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (!dst || !src || !bytes) return LDP_OK;
    cudaError_t e = cudaSuccess;
    if (!ctx->hstage) {
        if (cudaHostAlloc((void**)&ctx->hstage, 2 * kStageHalf, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            ctx->hstage = nullptr;
        }
        for (int k = 0; k < 2 && ctx->hstage; ++k)
            if (!ctx->hstage_ev[k]) e = cudaEventCreateWithFlags(&ctx->hstage_ev[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess && !ctx->hstage) {
        e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    } else if (e == cudaSuccess) {
        const char* from = (const char*)src;
        char* to = (char*)dst;
        size_t off = 0, prev_off = 0, prev_n = 0;
        int k = 0, prev_k = -1;
        while (e == cudaSuccess && (off < bytes || prev_k >= 0)) {
            size_t n = 0;
            if (off < bytes) {
                n = std::min(kStageHalf, bytes - off);
                e = cudaMemcpyAsync(ctx->hstage + k * kStageHalf, from + off, n, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaEventRecord(ctx->hstage_ev[k], s);
            }
            if (e == cudaSuccess && prev_k >= 0) {
                e = cudaEventSynchronize(ctx->hstage_ev[prev_k]);
                if (e == cudaSuccess) std::memcpy(to + prev_off, ctx->hstage + prev_k * kStageHalf, prev_n);
            }
            if (off < bytes) {
                prev_k = k;
                prev_off = off;
                prev_n = n;
                off += n;
                k ^= 1;
            } else {
                prev_k = -1;
            }
        }
    }
    if (e != cudaSuccess) {
        ldp_set_error(ctx, "device-to-host copy failed: %s", cudaGetErrorString(e));
        return LDP_ERR_DEVICE;
    }
    return LDP_OK;
}

static ldp_status copy_d2h(ldp_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!dst || !src || !bytes) return LDP_OK;
    cudaStream_t s;
    const cudaError_t e = read_stream(ctx, &s);
    if (e != cudaSuccess) {
        ldp_set_error(ctx, "read stream: %s", cudaGetErrorString(e));
        return LDP_ERR_DEVICE;
    }
    return copy_d2h_on(ctx, dst, src, bytes, s);
}

extern "C" ldp_status ldp_job_traj_results(ldp_job* job, ldp_traj_results* r) {
    if (!job || !r) return LDP_ERR_INVALID;
    if (!job->done) {
        ldp_status st = ldp_wait(job->ctx, job);
        if (st != LDP_OK) return st;
    }
    ldp_ctx* ctx = job->ctx;
    cudaSetDevice(ctx->device);
    const int64_t n = job->ntraj;
    const TrajState& S = job->st;
    ldp_status st;
#define CP(dst, src, bytes) \
    if ((st = copy_d2h(ctx, dst, src, bytes)) != LDP_OK) return st
    // Rows past the job's FPTCG entries are zero by construction: cleared
    // on the host instead of copied.
    const int ncr = LDP_C_CG0 + job->p.n_cg, nsr = LDP_S_CG0 + job->p.n_cg;
    CP(r->counts, S.counts, sizeof(int64_t) * ncr * n);
    CP(r->sums, S.sums, sizeof(double) * nsr * n);
    if (r->counts) std::memset(r->counts + (size_t)ncr * n, 0, sizeof(int64_t) * (LDP_NCOUNT - ncr) * n);
    if (r->sums) std::memset(r->sums + (size_t)nsr * n, 0, sizeof(double) * (LDP_NSUM - nsr) * n);
    CP(r->state0, S.state0, sizeof(int32_t) * n);
    CP(r->v0, S.v0, sizeof(double) * n);
    CP(r->x_final, S.x, sizeof(double) * n);
    CP(r->v_final, S.v, sizeof(double) * n);
    CP(r->state_final, S.state, sizeof(int32_t) * n);
    if (job->o.tick_cap > 0) CP(r->ticks, S.ticks, sizeof(int64_t) * job->o.tick_cap * n);
    if (job->o.event_cap > 0) {
        CP(r->events, S.ev, sizeof(double) * (LDP_E_CG0 + job->p.n_cg) * job->o.event_cap * n);
        CP(r->event_states, S.ev_st, (size_t)job->o.event_cap * n);
    }
    const size_t fb = sizeof(double) * (size_t)job->nframe * n;
    if (S.fx) CP(r->frames_x, S.fx, fb);
    if (S.fv) {
        CP(r->frames_v, S.fv, fb);
        CP(r->frames_f, S.ff, fb);
        CP(r->frames_barrier, S.fb, fb);
        CP(r->frames_pe, S.fpe, fb);
        CP(r->frames_ke, S.fke, fb);
        CP(r->frames_state, S.fst, fb);
    }
#undef CP
    return LDP_OK;
}

extern "C" ldp_status ldp_job_msd(ldp_job* job, int64_t* lags, double* msd, int64_t nlag) {
    if (!job) return LDP_ERR_INVALID;
    if (job->o.mode != LDP_MODE_FIXED_STEPS) return LDP_ERR_UNSUPPORTED;
    if (nlag < (int64_t)job->lags.size()) {
        ldp_set_error(job->ctx, "nlag %lld < %zu", (long long)nlag, job->lags.size());
        return LDP_ERR_INVALID;
    }
    if (!job->done) {
        ldp_status st = ldp_wait(job->ctx, job);
        if (st != LDP_OK) return st;
    }
    const int64_t nl = (int64_t)job->lags.size();
    if (lags) std::memcpy(lags, job->lags.data(), sizeof(int64_t) * nl);
    if (msd) {
        std::vector<double> sum(nl);
        ldp_status st = copy_d2h(job->ctx, sum.data(), job->d_msd, sizeof(double) * nl);
        if (st != LDP_OK) return st;
        const double nrun = (double)job->ntraj;
        for (int64_t i = 0; i < nl; ++i) msd[i] = sum[i] / nrun;
    }
    return LDP_OK;
}

// Per-trajectory mean event times, computed on the device so that only
// the means cross to the host: [LDP_E_CG0 + n_cg][ntraj].
extern "C" ldp_status ldp_job_traj_means(ldp_job* job, double* means) {
    if (!job || !means) return LDP_ERR_INVALID;
    if (!job->done) {
        ldp_status st = ldp_wait(job->ctx, job);
        if (st != LDP_OK) return st;
    }
    ldp_ctx* ctx = job->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t s;
    CUDA_OR_FAIL(ctx, read_stream(ctx, &s));
    const int e = launch_traj_means(job->st.counts, job->st.sums, job->d_means, job->ntraj, job->p.n_cg, s);
    if (e) {
        ldp_set_error(ctx, "means launch failed: %s", cudaGetErrorString((cudaError_t)e));
        return LDP_ERR_DEVICE;
    }
    const size_t bytes = sizeof(double) * (LDP_E_CG0 + job->p.n_cg) * (size_t)job->ntraj;
    return copy_d2h_on(ctx, means, job->d_means, bytes, s);
}

// Per-trajectory MSD (debug / parity): [nlag][ntraj].
extern "C" ldp_status ldp_job_msd_traj(ldp_job* job, double* msd0) {
    if (!job || !msd0) return LDP_ERR_INVALID;
    if (!job->done) {
        ldp_status st = ldp_wait(job->ctx, job);
        if (st != LDP_OK) return st;
    }
    return copy_d2h(job->ctx, msd0, job->d_msd0, sizeof(double) * job->lags.size() * job->ntraj);
}

// Registers every FP32 batched job of the list before enqueueing any launch,
// so that all of them share each persistent launch; FP64 plain jobs run
// side by side on two streams forked from the context's stream.
extern "C" ldp_status ldp_submit_batch(ldp_ctx* ctx, ldp_job** jobs, int njobs) {
    if (!ctx || (!jobs && njobs) || njobs < 0) return LDP_ERR_INVALID;
    CUDA_OR_FAIL(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    for (int i = 0; i < njobs; ++i) {
        ldp_job* job = jobs[i];
        if (!job || job->submitted || job->ctx != ctx) {
            ldp_set_error(ctx, "job %d is null, submitted already or of another context", i);
            return LDP_ERR_INVALID;
        }
    }
    // FP64 plain jobs: one alone runs on the context's stream.  Several run
    // side by side on the context's FP64 batch streams, forked from and
    // joined back to the context's stream: a job smaller than a wave of
    // resident blocks (65536 trajectories are 512 blocks of 128 threads,
    // 86 % of the 592 slots of 148 SMs) leaves the rest of the GPU to the
    // next job instead of idling until it drains.
    int n64 = 0;
    for (int i = 0; i < njobs; ++i) n64 += jobs[i]->o.precision != LDP_PREC_FP32_BATCHED;
    if (n64 == 1) {
        for (int i = 0; i < njobs; ++i)
            if (jobs[i]->o.precision != LDP_PREC_FP32_BATCHED) {
                ldp_status st = submit_on(ctx, jobs[i], s);
                if (st != LDP_OK) return st;
            }
    } else if (n64 > 1) {
        if (!ctx->f64s[0]) {
            for (int k = 0; k < kCtxF64Streams; ++k) {
                CUDA_OR_FAIL(ctx, cudaStreamCreateWithFlags(&ctx->f64s[k], cudaStreamNonBlocking));
                CUDA_OR_FAIL(ctx, cudaEventCreateWithFlags(&ctx->f64j[k], cudaEventDisableTiming));
            }
            CUDA_OR_FAIL(ctx, cudaEventCreateWithFlags(&ctx->f64fork, cudaEventDisableTiming));
        }
        CUDA_OR_FAIL(ctx, cudaEventRecord(ctx->f64fork, s));
        for (int k = 0; k < kCtxF64Streams; ++k) CUDA_OR_FAIL(ctx, cudaStreamWaitEvent(ctx->f64s[k], ctx->f64fork, 0));
        int k = 0;
        for (int i = 0; i < njobs; ++i)
            if (jobs[i]->o.precision != LDP_PREC_FP32_BATCHED) {
                ldp_status st = submit_on(ctx, jobs[i], ctx->f64s[k]);
                if (st != LDP_OK) return st;
                k = (k + 1) % kCtxF64Streams;
            }
        for (int k2 = 0; k2 < kCtxF64Streams; ++k2) {
            CUDA_OR_FAIL(ctx, cudaEventRecord(ctx->f64j[k2], ctx->f64s[k2]));
            CUDA_OR_FAIL(ctx, cudaStreamWaitEvent(s, ctx->f64j[k2], 0));
        }
    }
    int launches[4] = {0, 0, 0, 0};
    ldp_job* first[4] = {nullptr, nullptr, nullptr, nullptr};
    // A type whose queue holds no unfinished job gets each job's
    // post-processing as soon as that job has surely retired: items are
    // claimed in publication order by slots that never idle while items
    // remain, so a list-scheduling bound on the launches that drain the
    // jobs published so far (fp32_launch_bound of the prefix) holds per
    // job.  The post-processing then runs on a side stream beside the
    // later jobs' launches, in the registers and shared memory three
    // persistent blocks leave on an SM.
    bool early[4];
    for (int t = 0; t < 4; ++t) early[t] = fp32_queue_quiet(ctx, t);
    for (int i = 0; i < njobs; ++i)   // first-passage jobs: no tight bound
        if (jobs[i]->o.precision == LDP_PREC_FP32_BATCHED && jobs[i]->o.mode != LDP_MODE_FIXED_STEPS)
            early[fp32_type_of(jobs[i])] = false;
    std::vector<int> bound(njobs, 0);
    int top[4] = {0, 0, 0, 0};
    double prefix[4] = {0, 0, 0, 0}, longest[4] = {0, 0, 0, 0};
    for (int i = 0; i < njobs; ++i) {
        ldp_job* job = jobs[i];
        if (job->o.precision != LDP_PREC_FP32_BATCHED) continue;
        if (!job->arena && job_arena(job, true) == 0) {
            ldp_set_error(ctx, "cudaMalloc of %zu bytes failed", job_arena(job, false));
            return LDP_ERR_NOMEM;
        }
        job->launches = 0;
        int e = fp32_register(job);
        if (e) {
            ldp_set_error(ctx, "FP32 registration failed: %s", cudaGetErrorString((cudaError_t)e));
            return LDP_ERR_DEVICE;
        }
        job->submitted = true;
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[0], s));
        const int t = job->fp32_type;
        launches[t] += fp32_estimate_launches(job);
        if (!first[t]) first[t] = job;
        if (early[t]) {
            const double pairs = (double)((job->nsteps + 1) / 2);
            prefix[t] += pairs * (double)job->ntraj;
            longest[t] = std::max(longest[t], pairs);
            bound[i] = fp32_launch_bound(ctx, t, prefix[t], longest[t]);
            top[t] = std::max(top[t], bound[i]);
        }
    }
    for (int t = 0; t < 4; ++t) launches[t] = std::max(launches[t], top[t]);
    if (!ctx->side && (early[0] || early[1] || early[2] || early[3])) {
        int lo_prio = 0, hi_prio = 0;
        cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
        CUDA_OR_FAIL(ctx, cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, hi_prio));
    }
    for (int t = 0; t < 4; ++t) {
        if (!first[t]) continue;
        for (int k = 1; k <= launches[t]; ++k) {
            int e = fp32_pump(first[t], 1);
            if (e) {
                ldp_set_error(ctx, "FP32 launch failed: %s", cudaGetErrorString((cudaError_t)e));
                return LDP_ERR_DEVICE;
            }
            if (!early[t]) continue;
            for (int i = 0; i < njobs; ++i) {
                ldp_job* job = jobs[i];
                if (job->o.precision != LDP_PREC_FP32_BATCHED || job->fp32_type != t || bound[i] != k) continue;
                CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[1], s));
                CUDA_OR_FAIL(ctx, cudaStreamWaitEvent(ctx->side, job->ev[1], 0));
                CUDA_OR_FAIL(ctx, (cudaError_t)fp32_snapshot_remaining(job, (unsigned long long*)job->d_aux,
                                                                       ctx->side));
                job->rem_snapshot = true;
                CUDA_OR_FAIL(ctx, (cudaError_t)fp32_finalize(job, ctx->side, true));
                CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[2], ctx->side));
                job->fp32_phase = 3;   // checked when waited on: every trajectory retired
            }
        }
    }
    for (int i = 0; i < njobs; ++i) {
        ldp_job* job = jobs[i];
        if (job->o.precision != LDP_PREC_FP32_BATCHED || early[job->fp32_type]) continue;
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[1], s));
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[2], s));
        job->fp32_phase = 1;
    }
    return LDP_OK;
}

// Registers every job, then runs all their persistent launches and their
// post-processing as one CUDA graph: the launch count is an upper bound for
// draining the queues, so no host round trip happens until the results.
extern "C" ldp_status ldp_submit_batch_graph(ldp_ctx* ctx, ldp_job** jobs, int njobs) {
    if (!ctx || !jobs || njobs < 1) return LDP_ERR_INVALID;
    CUDA_OR_FAIL(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    for (int i = 0; i < njobs; ++i) {
        ldp_job* job = jobs[i];
        if (!job || job->submitted || job->ctx != ctx || job->o.precision != LDP_PREC_FP32_BATCHED) {
            ldp_set_error(ctx, "job %d is null, submitted already, of another context or not FP32 batched", i);
            return LDP_ERR_INVALID;
        }
    }
    // Per-job post-processing at prefix launch bounds, as in
    // ldp_submit_batch, captured as a side branch of the graph.
    bool early[4];
    for (int t = 0; t < 4; ++t) early[t] = fp32_queue_quiet(ctx, t);
    for (int i = 0; i < njobs; ++i)
        if (jobs[i]->o.mode != LDP_MODE_FIXED_STEPS) early[fp32_type_of(jobs[i])] = false;
    std::vector<int> bound(njobs, 0);
    double total[4] = {0, 0, 0, 0}, longest[4] = {0, 0, 0, 0};
    for (int i = 0; i < njobs; ++i) {
        ldp_job* job = jobs[i];
        if (!job->arena && job_arena(job, true) == 0) {
            ldp_set_error(ctx, "cudaMalloc of %zu bytes failed", job_arena(job, false));
            return LDP_ERR_NOMEM;
        }
        job->launches = 0;
        int e = fp32_register(job);
        if (e) {
            ldp_set_error(ctx, "FP32 registration failed: %s", cudaGetErrorString((cudaError_t)e));
            return LDP_ERR_DEVICE;
        }
        job->submitted = true;
        const int t = job->fp32_type;
        const double pairs = (double)((job->nsteps + 1) / 2);
        total[t] += pairs * (double)job->ntraj;
        longest[t] = std::max(longest[t], pairs);
        bound[i] = fp32_launch_bound(ctx, t, total[t], longest[t]);
    }
    const bool any_early = early[0] || early[1] || early[2] || early[3];
    if (any_early && !ctx->gside) {
        int lo_prio = 0, hi_prio = 0;
        cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
        CUDA_OR_FAIL(ctx, cudaStreamCreateWithPriority(&ctx->gside, cudaStreamNonBlocking, hi_prio));
        CUDA_OR_FAIL(ctx, cudaEventCreateWithFlags(&ctx->gjoin, cudaEventDisableTiming));
    }
    CUDA_OR_FAIL(ctx, cudaEventRecord(jobs[0]->ev[0], s));
    CUDA_OR_FAIL(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    // Inside the capture errors accumulate: the capture must end either way.
    int e = 0;
    bool forked = false;
    for (int t = 0; t < 4 && !e; ++t) {
        if (total[t] <= 0.0) continue;
        ldp_job* first = nullptr;
        for (int i = 0; i < njobs; ++i)
            if (jobs[i]->fp32_type == t) { first = jobs[i]; break; }
        const int nl = fp32_launch_bound(ctx, t, total[t], longest[t]);
        for (int k = 1; k <= nl && !e; ++k) {
            e = fp32_pump(first, 1);
            if (!early[t]) continue;
            for (int i = 0; i < njobs && !e; ++i) {
                ldp_job* job = jobs[i];
                if (job->fp32_type != t || bound[i] != k) continue;
                e = (int)cudaEventRecord(job->ev[3], s);
                if (!e) e = (int)cudaStreamWaitEvent(ctx->gside, job->ev[3], 0);
                if (!e) e = fp32_snapshot_remaining(job, (unsigned long long*)job->d_aux, ctx->gside);
                if (!e) e = fp32_finalize(job, ctx->gside, true);
                job->rem_snapshot = true;
                forked = true;
            }
        }
    }
    for (int i = 0; i < njobs && !e; ++i)
        if (!early[jobs[i]->fp32_type]) e = fp32_finalize(jobs[i]);
    if (forked) {
        const cudaError_t ej = cudaEventRecord(ctx->gjoin, ctx->gside);
        const cudaError_t ew = ej == cudaSuccess ? cudaStreamWaitEvent(s, ctx->gjoin, 0) : ej;
        if (!e && ew != cudaSuccess) e = (int)ew;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (e || ec != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        ldp_set_error(ctx, "batch graph capture failed: %s", cudaGetErrorString(e ? (cudaError_t)e : ec));
        return LDP_ERR_DEVICE;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        ldp_set_error(ctx, "batch graph instantiation failed: %s", cudaGetErrorString(ei));
        return LDP_ERR_DEVICE;
    }
    jobs[0]->gexec = exec;
    CUDA_OR_FAIL(ctx, cudaGraphLaunch(exec, s));
    for (int i = 0; i < njobs; ++i) {
        ldp_job* job = jobs[i];
        if (i) CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[0], s));
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[1], s));
        CUDA_OR_FAIL(ctx, cudaEventRecord(job->ev[2], s));
        job->fp32_phase = 3;
    }
    return LDP_OK;
}

extern "C" ldp_status ldp_ctx_mark(ldp_ctx* ctx, int mark) {
    if (!ctx || mark < 0 || mark >= kCtxMarks) return LDP_ERR_INVALID;
    CUDA_OR_FAIL(ctx, cudaEventRecord(ctx->marks[mark], ctx->stream));
    return LDP_OK;
}

extern "C" ldp_status ldp_ctx_elapsed_ms(ldp_ctx* ctx, int mark_a, int mark_b, double* ms) {
    if (!ctx || !ms || mark_a < 0 || mark_b < 0 || mark_a >= kCtxMarks || mark_b >= kCtxMarks) return LDP_ERR_INVALID;
    CUDA_OR_FAIL(ctx, cudaEventSynchronize(ctx->marks[mark_b]));
    float f = 0.f;
    CUDA_OR_FAIL(ctx, cudaEventElapsedTime(&f, ctx->marks[mark_a], ctx->marks[mark_b]));
    *ms = f;
    return LDP_OK;
}

extern "C" ldp_status ldp_ctx_synchronize(ldp_ctx* ctx) {
    if (!ctx) return LDP_ERR_INVALID;
    CUDA_OR_FAIL(ctx, cudaStreamSynchronize(ctx->stream));
    return LDP_OK;
}
