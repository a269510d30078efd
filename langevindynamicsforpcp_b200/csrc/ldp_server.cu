// ldp_server.cu -- serving loop: continuous batching of FP32 batched jobs.
//
// Requests (.inp parameter sets with job options) are submitted at any time
// and from any thread; each step of the loop
//  1. admits queued jobs while their device footprint fits the memory
//     budget, oldest first, letting later jobs that fit pass one that does
//     not for at most kBypassWindow (a job larger than the whole budget is
//     admitted alone), placing their arena in the server's device region
//     (allocated once: no device allocation per job, which can stall the
//     loop for seconds while the pool grows) and registering them with the
//     work queue of their model type;
//  2. publishes admitted jobs' trajectories to their type's queue in chunks,
//     keeping about as much unclaimed work queued as the launches in flight
//     and the next one will claim, and always publishing next for the job
//     with the fewest unpublished trajectories of any type (shortest
//     remaining first): a small job that arrives while large ones run
//     starts within about one launch, instead of after every earlier job;
//  3. keeps up to `max_inflight` short persistent launches (pair budget
//     `pair_budget`) in flight while any job is active, each over all four
//     model types' queues (a warp serves one type at a time and moves to
//     another type with work when its lanes are idle), so the types share
//     every launch and newly published work is reached within one launch;
//  4. reads every queue's per-job "trajectories not yet retired" counters
//     (and its claimed-items count) with one asynchronous copy, and for each
//     job whose counter reached zero enqueues its post-processing (event
//     sums, MSD) on a separate stream;
//  5. marks jobs done when their post-processing has run.
// A context that runs a server should not also run FP32 batched jobs
// through ldp_submit: the server's streams order the queues' work.
// Job state (RNG counters, partial statistics) stays in HBM from admission
// to release; results are identical alone and in any mix, since every draw
// is keyed by (seed, job id, trajectory, step).
//
// The reference runs one .inp per MPI process (src/mpiKernel.cpp); the
// serving loop has no counterpart there.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "ldp_fp32.h"
#include "ldp_internal.h"
#include "ldp_region.h"

namespace {

constexpr double kBypassWindow = 0.25;   // seconds the oldest pending job may be passed

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Entry {
    uint64_t ticket = 0;
    ldp_job* job = nullptr;
    size_t bytes = 0;
    size_t offset = ldp::Region::kNone;   // arena's place in the server's region
    int state = LDP_SRV_QUEUED;
    int type = -1;
    uint64_t gen_admit = 0;          // remaining-counter copies issued before admission
    double t_submit = 0, t_admit = 0, t_ready = 0, t_done = 0;
    cudaEvent_t fin = nullptr;       // post-processing done
};

}  // namespace

struct ldp_server {
    ldp_ctx* ctx = nullptr;
    size_t budget = 0, in_use = 0;
    char* region = nullptr;              // device memory of the job arenas (budget bytes)
    ldp::Region placer;
    uint32_t pair_budget = 0;
    int max_inflight = 2;
    cudaStream_t side = nullptr;         // post-processing
    cudaStream_t q = nullptr;            // the queues' work: registration, publication, launches, counter copies
    cudaStream_t qs[4] = {};             // per model type: all q (one stream orders every queue's work)
    unsigned long long head_seen[4] = {};
    std::mutex mu;                       // guards pending and all
    std::deque<Entry*> pending;
    std::vector<Entry*> running;         // integrating
    std::vector<Entry*> finishing;       // post-processing enqueued
    std::unordered_map<uint64_t, Entry*> all;
    std::deque<uint64_t> ended;          // tickets done or failed, not yet taken
    uint64_t next_ticket = 1;
    unsigned long long* h_rem[4] = {};   // pinned copies of the queues' counters
    cudaEvent_t rem_ev[4] = {};
    bool rem_pending[4] = {};
    uint64_t rem_gen[4] = {};            // copies issued per type
    std::deque<cudaEvent_t> inflight[4];
    std::vector<cudaEvent_t> pool;       // idle events
    int64_t launches = 0;
    int64_t steps = 0;
    double phase_s[6] = {}, phase_max_s[6] = {};   // host time per phase of a step
    double phase_cur[6] = {};                       // of the current step

    // Adds the time since t0 to phase i of the current step; t0 = now.
    void phase(int i, double& t0) {
        const double t = now_s();
        phase_cur[i] += t - t0;
        t0 = t;
    }
    void close_step() {
        for (int i = 0; i < 6; ++i) {
            phase_s[i] += phase_cur[i];
            phase_max_s[i] = std::max(phase_max_s[i], phase_cur[i]);
            phase_cur[i] = 0;
        }
    }

    cudaEvent_t get_event() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) e = nullptr;
        return e;
    }
};

static ldp_status fail(ldp_server* s, const char* what, cudaError_t e) {
    ldp_set_error(s->ctx, "%s: %s", what, cudaGetErrorString(e));
    return LDP_ERR_DEVICE;
}

extern "C" void ldp_server_opts_default(ldp_server_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->hbm_budget = 0;        // 80% of the free device memory at creation
    o->pair_budget = 1024;    // step pairs per slot per launch
    o->max_inflight = 2;
    o->region = 1;
}

extern "C" ldp_status ldp_server_create(ldp_ctx* ctx, const ldp_server_opts* o, ldp_server** out) {
    if (!ctx || !out) return LDP_ERR_INVALID;
    ldp_server_opts opts;
    if (o) opts = *o; else ldp_server_opts_default(&opts);
    if (opts.max_inflight < 1 || opts.max_inflight > 16) {
        ldp_set_error(ctx, "max_inflight must be 1..16 (got %d)", opts.max_inflight);
        return LDP_ERR_INVALID;
    }
    cudaSetDevice(ctx->device);
    ldp_server* s = new ldp_server();
    s->ctx = ctx;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    // Job arenas come from the device's stream-ordered pool (ldp_create keeps
    // freed memory in it): memory the pool holds unused counts as free.
    cudaMemPool_t pool = nullptr;
    uint64_t held = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &held);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    }
    const size_t avail = free_b + (size_t)(held > used ? held - used : 0);
    s->budget = opts.hbm_budget ? (size_t)opts.hbm_budget : (size_t)(0.8 * (double)avail);
    s->pair_budget = opts.pair_budget ? (uint32_t)opts.pair_budget : 1024u;
    s->max_inflight = opts.max_inflight;
    // Post-processing runs at the highest stream priority: the persistent
    // launches fill every SM, and a finished job's MSD blocks should take
    // the SMs the next launch boundary frees before new persistent blocks.
    int lo_prio = 0, hi_prio = 0;
    cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    cudaError_t e = cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, hi_prio);
    for (int t = 0; t < 4 && e == cudaSuccess; ++t) {
        // the queue's counters, then its claimed-items count
        e = cudaMallocHost((void**)&s->h_rem[t], sizeof(unsigned long long) * (ldp::kFp32MaxJobs + 1));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->rem_ev[t], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->q, cudaStreamNonBlocking, lo_prio);
    for (int t = 0; t < 4; ++t) s->qs[t] = s->q;
    if (e != cudaSuccess) {
        ldp_server_destroy(s);
        ldp_set_error(ctx, "server set-up failed: %s", cudaGetErrorString(e));
        return LDP_ERR_DEVICE;
    }
    if (opts.region) {
        // Memory the pool holds unused goes back to the device first.
        if (pool && held > used) {
            cudaDeviceSynchronize();
            cudaMemPoolTrimTo(pool, 0);
        }
        s->budget &= ~(size_t)255;
        if (cudaMalloc((void**)&s->region, s->budget) != cudaSuccess) {
            cudaGetLastError();
            ldp_server_destroy(s);
            ldp_set_error(ctx, "server region of %zu bytes: device allocation failed", s->budget);
            return LDP_ERR_NOMEM;
        }
        s->placer.reset(s->budget);
    }
    *out = s;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_submit(ldp_server* s, const ldp_params* p, const ldp_job_opts* o,
                                        uint64_t* ticket) {
    if (!s || !p || !ticket) return LDP_ERR_INVALID;
    ldp_job_opts opts;
    if (o) opts = *o; else ldp_job_opts_default(&opts);
    if (opts.precision != LDP_PREC_FP32_BATCHED) {
        ldp_set_error(s->ctx, "the serving loop runs FP32 batched jobs");
        return LDP_ERR_UNSUPPORTED;
    }
    ldp_job* job = nullptr;
    ldp_status st = ldp_job_create_unchecked(s->ctx, p, &opts, &job);
    if (st != LDP_OK) return st;
    Entry* en = new Entry();
    en->job = job;
    en->bytes = ldp_job_arena(job, false);
    en->type = (job->k.dbl ? 2 : 0) + (job->k.over ? 1 : 0);
    en->t_submit = now_s();
    std::lock_guard<std::mutex> lk(s->mu);
    en->ticket = s->next_ticket++;
    s->pending.push_back(en);
    s->all[en->ticket] = en;
    *ticket = en->ticket;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_step(ldp_server* s, int* ndone) {
    if (!s) return LDP_ERR_INVALID;
    ldp_ctx* ctx = s->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    int done = 0;
    ++s->steps;

    // 1. admission by footprint, oldest first; a later job that fits may
    //    pass one that does not, unless the oldest pending job has waited
    //    longer than the bypass window (then it is admitted next).
    const double t_now = now_s();
    double tp = t_now;
    for (size_t i = 0;;) {
        Entry* en = nullptr;
        size_t pos = 0;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (i >= s->pending.size()) break;
            Entry* c = s->pending[i];
            const bool idle = s->running.empty() && s->finishing.empty();
            if (idle || s->in_use + c->bytes <= s->budget) {
                en = c;
                pos = i;
                s->pending.erase(s->pending.begin() + (std::ptrdiff_t)i);
            } else {
                if (i == 0 && t_now - c->t_submit > kBypassWindow) break;
                ++i;
                continue;
            }
        }
        ldp_job* job = en->job;
        bool got = false;
        if (s->region && en->bytes <= s->budget) {
            {
                std::lock_guard<std::mutex> lk(s->mu);
                en->offset = s->placer.take(en->bytes);
            }
            got = en->offset != ldp::Region::kNone;
            if (got) ldp_job_arena_at(job, s->region + en->offset);
        } else {
            // no region, or a job larger than the whole budget (admitted
            // alone): its own allocation
            got = ldp_job_arena(job, true) != 0;
        }
        s->phase(0, tp);
        if (!got && s->region && en->bytes <= s->budget) {
            // the region is fragmented or held by finished jobs not yet
            // released: wait for releases
            std::lock_guard<std::mutex> lk(s->mu);
            s->pending.insert(s->pending.begin() + (std::ptrdiff_t)pos, en);
            break;
        }
        if (!got) {
            const bool idle = s->running.empty() && s->finishing.empty();
            if (idle) {
                en->state = LDP_SRV_FAILED;
                en->t_done = now_s();
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->ended.push_back(en->ticket);
                }
                ldp_set_error(ctx, "job %llu: device allocation of %zu bytes failed",
                              (unsigned long long)en->ticket, en->bytes);
                continue;
            }
            std::lock_guard<std::mutex> lk(s->mu);
            s->pending.insert(s->pending.begin() + (std::ptrdiff_t)pos, en);
            break;
        }
        job->launches = 0;
        // the arena was allocated on the context's stream
        cudaEvent_t ready = s->get_event();
        if (!ready) return fail(s, "event creation", cudaErrorMemoryAllocation);
        s->pool.push_back(ready);
        cudaError_t ce = cudaEventRecord(ready, st);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s->qs[en->type], ready, 0);
        if (ce != cudaSuccess) return fail(s, "admission ordering", ce);
        const int e = ldp::fp32_register(job, s->qs[en->type], false);
        s->phase(1, tp);
        if (e) return fail(s, "job registration", (cudaError_t)e);
        job->submitted = true;
        job->fp32_phase = 1;
        en->state = LDP_SRV_RUNNING;
        en->gen_admit = s->rem_gen[en->type];
        en->t_admit = now_s();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->in_use += en->bytes;
        }
        s->running.push_back(en);
    }

    s->phase(0, tp);

    // 2. publication: unclaimed work kept at about what the launches in
    //    flight and the next one will claim (slots x steps per launch x the
    //    running jobs' mean 1 / trajectory length, per launch), shortest
    //    remaining job first over all model types, so a job that arrives
    //    waits behind little queued work
    bool active[4] = {false, false, false, false};
    double inv_len = 0.0;
    for (Entry* en : s->running) {
        active[en->type] = true;
        inv_len += 1.0 / (double)std::max<uint64_t>(en->job->nsteps, 1);
    }
    if (!s->running.empty()) {
        int64_t total = 0;
        int64_t nslots = ldp::fp32_mixed_slots(ctx);
        for (int t = 0; t < 4; ++t) {
            if (!active[t]) continue;
            const unsigned long long pub = ldp::fp32_published(ctx, t);
            total += (int64_t)(pub - std::min(pub, s->head_seen[t]));
            if (!nslots) nslots = ldp::fp32_nslots(ctx, t);
        }
        const double per_launch = (double)nslots * 2.0 * (double)s->pair_budget * inv_len /
                                  (double)s->running.size();
        const int64_t target = std::min<int64_t>(
            std::max<int64_t>((int64_t)(per_launch * (s->max_inflight + 1)), 4096), 2 * nslots);
        while (total < target) {
            Entry* best = nullptr;
            int64_t best_left = 0;
            for (Entry* en : s->running) {
                const int64_t left = en->job->ntraj - en->job->fp32_published;
                if (left > 0 && (!best || left < best_left)) { best = en; best_left = left; }
            }
            if (!best) break;
            const int64_t chunk = std::min<int64_t>(best_left, std::max<int64_t>(target - total, 1024));
            const int e = ldp::fp32_publish_range(best->job, chunk, s->qs[best->type]);
            if (e) return fail(s, "publication", (cudaError_t)e);
            total += chunk;
        }
    }

    s->phase(2, tp);

    // 3. persistent launches: each covers every model type's queue (a warp
    //    serves one type at a time and moves to another with work when its
    //    lanes are idle), so no type waits behind another type's launch
    {
        auto& q = s->inflight[0];
        while (!q.empty() && cudaEventQuery(q.front()) == cudaSuccess) {
            s->pool.push_back(q.front());
            q.pop_front();
        }
        const bool any = active[0] || active[1] || active[2] || active[3];
        while (any && (int)q.size() < s->max_inflight) {
            const int e = ldp::fp32_launch_mixed(ctx, s->pair_budget, s->q);
            if (e) return fail(s, "persistent launch", (cudaError_t)e);
            ++s->launches;
            cudaEvent_t ev = s->get_event();
            if (!ev) return fail(s, "event creation", cudaErrorMemoryAllocation);
            q.push_back(ev);
            const cudaError_t ce = cudaEventRecord(ev, s->q);
            if (ce != cudaSuccess) return fail(s, "launch event", ce);
        }
    }

    s->phase(3, tp);

    // 4. completion: one counter copy per type, read when it has landed
    for (int t = 0; t < 4; ++t) {
        if (s->rem_pending[t]) {
            const cudaError_t q = cudaEventQuery(s->rem_ev[t]);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) return fail(s, "counter copy", q);
            s->rem_pending[t] = false;
            s->head_seen[t] = s->h_rem[t][ldp::kFp32MaxJobs];
            const uint64_t gen = s->rem_gen[t];
            for (size_t i = 0; i < s->running.size();) {
                Entry* en = s->running[i];
                // a copy issued before the job was registered holds the
                // counter of the slot's previous job
                if (en->type != t || en->gen_admit >= gen || s->h_rem[t][en->job->fp32_slot] != 0) {
                    ++i;
                    continue;
                }
                cudaStreamWaitEvent(s->side, s->rem_ev[t], 0);
                const int e = ldp::fp32_finalize(en->job, s->side, true);   // lean MSD: runs beside the launches
                if (e) return fail(s, "post-processing", (cudaError_t)e);
                en->fin = s->get_event();
                if (!en->fin) return fail(s, "event creation", cudaErrorMemoryAllocation);
                const cudaError_t ce = cudaEventRecord(en->fin, s->side);
                if (ce != cudaSuccess) return fail(s, "post-processing event", ce);
                en->state = LDP_SRV_FINISHING;
                en->t_ready = now_s();
                en->job->fp32_phase = 2;
                s->finishing.push_back(en);
                s->running[i] = s->running.back();
                s->running.pop_back();
            }
        }
        if (!s->rem_pending[t]) {
            bool any = false;
            for (Entry* en : s->running) any = any || en->type == t;
            if (!any) continue;
            const int e = ldp::fp32_copy_remaining(ctx, t, s->h_rem[t], s->h_rem[t] + ldp::kFp32MaxJobs, s->qs[t]);
            if (e) return fail(s, "counter copy", (cudaError_t)e);
            cudaEventRecord(s->rem_ev[t], s->qs[t]);
            s->rem_pending[t] = true;
            ++s->rem_gen[t];
        }
    }

    s->phase(4, tp);

    // 5. jobs whose post-processing ran
    for (size_t i = 0; i < s->finishing.size();) {
        Entry* en = s->finishing[i];
        const cudaError_t q = cudaEventQuery(en->fin);
        if (q == cudaErrorNotReady) { ++i; continue; }
        if (q != cudaSuccess) return fail(s, "post-processing", q);
        s->pool.push_back(en->fin);
        en->fin = nullptr;
        ldp_job* job = en->job;
        job->fp32_phase = 0;
        ldp::fp32_release(job);
        job->done = true;
        en->state = LDP_SRV_DONE;
        en->t_done = now_s();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->ended.push_back(en->ticket);
        }
        ++done;
        s->finishing[i] = s->finishing.back();
        s->finishing.pop_back();
    }
    s->phase(5, tp);
    s->close_step();
    if (ndone) *ndone = done;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_poll(ldp_server* s, uint64_t ticket, int* state, double* latency_s) {
    if (!s || !state) return LDP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return LDP_ERR_INVALID;
    const Entry* en = it->second;
    *state = en->state;
    if (latency_s) *latency_s = (en->state == LDP_SRV_DONE || en->state == LDP_SRV_FAILED) ? en->t_done - en->t_submit
                                                                                          : 0.0;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_take_ended(ldp_server* s, uint64_t* tickets, int64_t cap, int64_t* n) {
    if (!s || !n || cap < 0 || (cap > 0 && !tickets)) return LDP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (cap == 0) {
        *n = (int64_t)s->ended.size();
        return LDP_OK;
    }
    int64_t k = 0;
    while (k < cap && !s->ended.empty()) {
        tickets[k++] = s->ended.front();
        s->ended.pop_front();
    }
    *n = k;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_job_times(ldp_server* s, uint64_t ticket, double* times) {
    if (!s || !times) return LDP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end()) return LDP_ERR_INVALID;
    const Entry* en = it->second;
    auto rel = [&](double t) { return t > 0.0 ? t - en->t_submit : -1.0; };
    times[0] = rel(en->t_admit);
    times[1] = rel(en->t_ready);
    times[2] = rel(en->t_done);
    return LDP_OK;
}

extern "C" ldp_status ldp_server_job(ldp_server* s, uint64_t ticket, ldp_job** job) {
    if (!s || !job) return LDP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(ticket);
    if (it == s->all.end() || it->second->state != LDP_SRV_DONE) return LDP_ERR_NOT_READY;
    *job = it->second->job;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_release(ldp_server* s, uint64_t ticket) {
    if (!s) return LDP_ERR_INVALID;
    Entry* en = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->all.find(ticket);
        if (it == s->all.end()) return LDP_ERR_INVALID;
        en = it->second;
        if (en->state != LDP_SRV_DONE && en->state != LDP_SRV_FAILED) return LDP_ERR_NOT_READY;
        s->all.erase(it);
    }
    ldp_job_destroy(en->job);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (en->state == LDP_SRV_DONE) s->in_use -= en->bytes;
        if (en->offset != ldp::Region::kNone) s->placer.give(en->offset, en->bytes);
    }
    delete en;
    return LDP_OK;
}

extern "C" ldp_status ldp_server_info_get(ldp_server* s, ldp_server_info* info) {
    if (!s || !info) return LDP_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(info, 0, sizeof(*info));
    info->queued = (int64_t)s->pending.size();
    info->running = (int64_t)s->running.size();
    info->finishing = (int64_t)s->finishing.size();
    int64_t d = 0;
    for (auto& kv : s->all) d += kv.second->state == LDP_SRV_DONE;
    info->done = d;
    info->hbm_in_use = (int64_t)s->in_use;
    info->hbm_budget = (int64_t)s->budget;
    info->launches = s->launches;
    info->steps = s->steps;
    for (int i = 0; i < 6; ++i) {
        info->phase_s[i] = s->phase_s[i];
        info->phase_max_s[i] = s->phase_max_s[i];
    }
    return LDP_OK;
}

extern "C" void ldp_server_destroy(ldp_server* s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    if (s->side) cudaStreamSynchronize(s->side);
    if (s->q) cudaStreamSynchronize(s->q);
    {
        // Jobs never admitted are dropped; jobs still integrating hold queue
        // slots until their trajectories retired, so the loop runs on until
        // nothing is active.
        std::lock_guard<std::mutex> lk(s->mu);
        s->pending.clear();
    }
    for (int guard = 0; guard < 100000 && (!s->running.empty() || !s->finishing.empty()); ++guard) {
        if (ldp_server_step(s, nullptr) != LDP_OK) break;
        cudaStreamSynchronize(s->side);
        if (s->q) cudaStreamSynchronize(s->q);
    }
    for (auto& kv : s->all) {
        if (kv.second->fin) cudaEventDestroy(kv.second->fin);
        ldp_job_destroy(kv.second->job);
        delete kv.second;
    }
    for (int t = 0; t < 4; ++t) {
        for (cudaEvent_t e : s->inflight[t]) cudaEventDestroy(e);
        if (s->rem_ev[t]) cudaEventDestroy(s->rem_ev[t]);
        if (s->h_rem[t]) cudaFreeHost(s->h_rem[t]);
    }
    for (cudaEvent_t e : s->pool) cudaEventDestroy(e);
    if (s->region) cudaFree(s->region);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->q) cudaStreamDestroy(s->q);
    delete s;
}
