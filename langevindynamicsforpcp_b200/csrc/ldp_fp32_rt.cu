// ldp_fp32_rt.cu -- host side of the FP32 batched persistent path.
//
// One work queue and one set of persistent slots per model type
// (single/double x overdamped/underdamped), created on first use in a
// context.  Submitting an FP32 job writes its JobF into the queue's device
// job table, publishes its trajectories as one item range, and enqueues
// persistent-kernel launches; completion is the job's device "remaining"
// counter reaching zero.  The job scheduler (mpiKernel's role in the
// reference, src/mpiKernel.cpp) is this queue: trajectories of many jobs
// share every launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ldp_fp32.h"
#include "ldp_internal.h"
#include "ldp_msd.h"

namespace ldp {

struct Fp32Queue {
    bool ready = false;
    QueueDev q{};
    SlotsDev s{};
    void* qmem = nullptr;
    void* smem = nullptr;
    int grid = 0, block = 256;
    uint64_t pair_budget = 1 << 15;
    int64_t nranges = 0;
    unsigned long long tail = 0;
    unsigned long long* rem = nullptr;   // [kFp32MaxJobs] trajectories not yet retired, by job slot
    // Pinned staging for job uploads: a ring of 4 KiB blocks, each reused
    // only after the copies that read it have run (its event), so that
    // registering a job never waits for the launches in flight.
    static constexpr int kStageSlots = 64;
    int64_t* h_stage = nullptr;
    cudaEvent_t stage_ev[kStageSlots] = {};
    int stage_next = 0, stage_last = 0;
    std::vector<ldp_job*> table;  // job table slot -> job
    std::vector<int> free_slots;
};

struct Fp32Runtime {
    Fp32Queue q[4];
    // mixed launches (serving): one set of slots for all four queues, the
    // type each warp serves
    SlotsDev mixed{};
    void* mixed_mem = nullptr;
    int32_t* wtype = nullptr;
    int mixed_grid = 0;
};

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Next pinned staging block of the queue, once the copies that read it last
// have run; the caller records stage_ev[stage_last] after its copies.
static int64_t* stage(Fp32Queue& Q) {
    const int si = Q.stage_next;
    Q.stage_next = (Q.stage_next + 1) % Fp32Queue::kStageSlots;
    cudaEventSynchronize(Q.stage_ev[si]);
    Q.stage_last = si;
    return Q.h_stage + (size_t)si * (4096 / sizeof(int64_t));
}

// One set of persistent slots (their state between launches): nslots
// slots with R cell-table ring entries each, every slot empty.
static int slots_init(int64_t nslots, int R, SlotsDev* Sp, void** mem) {
    size_t sb = al256(sizeof(int32_t) * nslots) * 6 + al256(sizeof(int64_t) * nslots) * 7 +
                al256(sizeof(float) * nslots) * 2 + al256(sizeof(longlong2) * (size_t)R * nslots) +
                al256(sizeof(unsigned long long));
    cudaError_t e = cudaMalloc(mem, sb);
    if (e != cudaSuccess) return (int)e;
    e = cudaMemset(*mem, 0, sb);
    if (e != cudaSuccess) return (int)e;
    char* a = (char*)*mem;
    size_t o = 0;
    SlotsDev& S = *Sp;
    S.nslots = nslots;
    S.ring_slots = R;
    S.job = (int32_t*)(a + o); o += al256(sizeof(int32_t) * nslots);
    S.cell = (int32_t*)(a + o); o += al256(sizeof(int32_t) * nslots);
    S.st = (int32_t*)(a + o); o += al256(sizeof(int32_t) * nslots);
    S.ckey = (int32_t*)(a + o); o += al256(sizeof(int32_t) * nslots);
    S.cgw = (int32_t*)(a + o); o += al256(sizeof(int32_t) * nslots);
    S.fidx = (int32_t*)(a + o); o += al256(sizeof(int32_t) * nslots);
    S.nxf = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.nflip = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.traj = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.step = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.cflip = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.sc1 = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.since = (int64_t*)(a + o); o += al256(sizeof(int64_t) * nslots);
    S.xp = (float*)(a + o); o += al256(sizeof(float) * nslots);
    S.rv = (float*)(a + o); o += al256(sizeof(float) * nslots);
    S.ring = (longlong2*)(a + o); o += al256(sizeof(longlong2) * (size_t)R * nslots);
    S.retired = (unsigned long long*)(a + o);
    // every slot starts empty
    std::vector<int32_t> neg((size_t)nslots, -1);
    e = cudaMemcpy(S.job, neg.data(), sizeof(int32_t) * nslots, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return (int)e;
    return 0;
}

static int queue_init(ldp_ctx* ctx, Fp32Queue& Q, int type, int ring_slots) {
    if (Q.ready) return 0;
    Q.block = ctx->fp32_block ? ctx->fp32_block : 256;
    // A persistent grid never exceeds what is resident at once.
    const int resident = fp32_blocks_per_sm(type >= 2, (type & 1) != 0, Q.block);
    int bps = ctx->fp32_blocks_per_sm ? ctx->fp32_blocks_per_sm : resident;
    if (resident > 0) bps = std::min(bps, resident);
    bps = std::max(bps, 1);
    Q.grid = ctx->sm_count * bps;
    Q.pair_budget = ctx->fp32_pair_budget ? ctx->fp32_pair_budget : (1u << 15);
    const int64_t nslots = (int64_t)Q.grid * Q.block;
    // queue + job table
    size_t qb = al256(sizeof(int64_t) * kFp32MaxRanges) * 2 + al256(sizeof(int32_t) * kFp32MaxRanges) +
                al256(sizeof(unsigned long long) * 2) + al256(sizeof(int32_t)) + al256(sizeof(JobF) * kFp32MaxJobs) +
                al256(sizeof(unsigned long long) * kFp32MaxJobs);
    cudaError_t e = cudaMalloc(&Q.qmem, qb);
    if (e != cudaSuccess) return (int)e;
    e = cudaMemset(Q.qmem, 0, qb);
    if (e != cudaSuccess) return (int)e;
    char* a = (char*)Q.qmem;
    size_t o = 0;
    Q.q.range_end = (int64_t*)(a + o); o += al256(sizeof(int64_t) * kFp32MaxRanges);
    Q.q.range_first = (int64_t*)(a + o); o += al256(sizeof(int64_t) * kFp32MaxRanges);
    Q.q.range_job = (int32_t*)(a + o); o += al256(sizeof(int32_t) * kFp32MaxRanges);
    Q.q.head = (unsigned long long*)(a + o);
    Q.q.tail = Q.q.head + 1;
    o += al256(sizeof(unsigned long long) * 2);
    Q.q.nranges = (int32_t*)(a + o); o += al256(sizeof(int32_t));
    Q.q.jobs = (JobF*)(a + o); o += al256(sizeof(JobF) * kFp32MaxJobs);
    Q.rem = (unsigned long long*)(a + o);
    e = (cudaError_t)slots_init(nslots, ring_slots, &Q.s, &Q.smem);
    if (e != cudaSuccess) return (int)e;
    e = cudaMallocHost((void**)&Q.h_stage, 4096 * Fp32Queue::kStageSlots);
    if (e != cudaSuccess) return (int)e;
    for (int i = 0; i < Fp32Queue::kStageSlots; ++i) {
        e = cudaEventCreateWithFlags(&Q.stage_ev[i], cudaEventDisableTiming);
        if (e != cudaSuccess) return (int)e;
    }
    Q.table.assign(kFp32MaxJobs, nullptr);
    Q.free_slots.clear();
    for (int i = kFp32MaxJobs - 1; i >= 0; --i) Q.free_slots.push_back(i);
    Q.ready = true;
    return 0;
}

static void fill_jobf(const ldp_job* job, JobF* J) {
    std::memset(J, 0, sizeof(*J));
    const KConst& k = job->k;
    const TrajState& S = job->st;
    const int64_t n = job->ntraj;
    J->eta = k.eta; J->eq = k.eq; J->rs = k.rs; J->rv = k.rv; J->us = k.us; J->init_state = k.init_state;
    J->wt = k.wt; J->fpt = k.fpt; J->tpt = k.tpt; J->cg = k.cg; J->n_cg = k.n_cg; J->write_x = k.write_x;
    J->at_bottom = k.at_bottom; J->fp_mode = k.fp_mode; J->lanes = k.lanes; J->nruns = k.nruns;
    {
        const bool fp = k.fp_mode != 0, single = !k.dbl;
        J->evm = ((single && k.wt && !fp) ? EV_WT : 0) | ((single && k.fpt && !fp) ? EV_FPT : 0) |
                 ((k.fpt || fp) ? EV_FPT2 : 0) | ((single && k.tpt && !fp) ? EV_TPT : 0) |
                 ((k.cg && !fp) ? EV_CG : 0) | (fp ? EV_FP : 0);
    }
    for (int j = 0; j < LDP_MAX_CG; ++j) J->cg_size[j] = k.cg_size[j] ? k.cg_size[j] : 1;
    J->key0 = k.key0; J->key1 = k.key1;
    J->g0 = k.g0;
    J->L = k.fL; J->halfL = k.fhalfL; J->w = k.fw;
    J->slope[0] = k.fslope[0]; J->slope[1] = k.fslope[1];
    J->xb[0] = k.fxb[0]; J->xb[1] = k.fxb[1]; J->lo0 = k.flo0; J->hi1 = k.fhi1; J->xc = k.fxc;
    for (int b = 0; b < 2; ++b)
        for (int s = 0; s < 2; ++s) {
            J->sN[b][s] = k.fsN[b][s]; J->sP[b][s] = k.fsP[b][s];
            J->sNd[b][s] = k.sN[b][s]; J->sPd[b][s] = k.sP[b][s];
            J->Hd[b][s] = k.Hd[b][s]; J->iN[b][s] = k.iN[b][s]; J->iP[b][s] = k.iP[b][s];
        }
    J->c_drift = k.fc_drift; J->sig_r = k.fsig_r; J->hdt_invM = k.fhdt_invM; J->hdt = k.fhdt;
    J->expg = k.fexpg; J->sig_v = k.fsig_v;
    {
        const double sg = k.over ? (double)k.fsig_r : (double)k.fsig_v;
        J->bm_k = (float)(-2.0 * 0.69314718055994530942 * sg * sg);
        J->invLf = (float)(1.0 / (double)k.fL);
        J->a_lapf = (float)k.a_lap;
        J->c_lapf[0] = (float)k.c_lap[0];
        J->c_lapf[1] = (float)k.c_lap[1];
        // Breakpoints of the FP32 force (the comparisons of the kernel's
        // force_of use exactly these floats), the barrier top 0 (well
        // boundary) and the cell edges.
        float c[8];
        int nc = 0;
        c[nc++] = -k.fhalfL;
        c[nc++] = k.fhalfL;
        c[nc++] = 0.0f;
        if (!k.dbl) { c[nc++] = -k.fw; c[nc++] = k.fw; }
        else { c[nc++] = k.flo0; c[nc++] = k.fxb[0]; c[nc++] = k.fxc; c[nc++] = k.fxb[1]; c[nc++] = k.fhi1; }
        std::sort(c, c + nc);
        int nb = 0;
        for (int i = 0; i < nc; ++i)
            if (c[i] >= -k.fhalfL && c[i] <= k.fhalfL && (nb == 0 || c[i] != J->bp[nb - 1])) J->bp[nb++] = c[i];
        J->nbp = nb;
        J->edge_lo = nb >= 3 ? J->bp[1] : k.fhalfL;
        J->edge_hi = nb >= 3 ? J->bp[nb - 2] : -k.fhalfL;
        const bool flat = k.dbl ? (k.flo0 > -k.fhalfL && k.fhi1 < k.fhalfL) : (k.fw < k.fhalfL);
        J->edge_flat = (nb >= 3 && flat) ? 1 : 0;
    }
    J->x0 = k.x0; J->v0 = k.v0; J->dt = k.dt; J->Ld = k.L; J->invL = k.invL; J->sig_v0 = k.sig_v0;
    J->sig_r_d = k.sig_r; J->a_lap = k.a_lap; J->c_lap[0] = k.c_lap[0]; J->c_lap[1] = k.c_lap[1];
    J->p_first = k.p_first; J->p_cell0 = k.p_cell0; J->mhalf = k.mhalf;
    J->Hs[0] = k.Hs[0]; J->Hs[1] = k.Hs[1]; J->wd = k.w;
    J->xbd[0] = k.xb[0]; J->xbd[1] = k.xb[1]; J->lo0d = k.lo0; J->hi1d = k.hi1; J->xcd = k.xc;
    J->T_eq = k.T_eq; J->T_as[0] = k.T_as[0]; J->T_as[1] = k.T_as[1];
    J->ln1m[0] = k.ln1m[0]; J->ln1m[1] = k.ln1m[1];
    // steps are numbered after the previous ones of a continued run
    J->nsteps = job->steps_before + job->nsteps;
    J->step0 = job->steps_before + 1;
    J->resume = job->fp32_resume ? 1 : 0;
    J->freq_save = k.freq_save;
    J->nframe = k.nframe;
    J->tick_cap = job->o.tick_cap;
    J->ntraj = n;
    J->counts = S.counts;
    J->ssum = job->d_ssum;
    J->state0 = S.state0;
    J->v0s = S.v0;
    J->x_final = S.x;
    J->v_final = S.v;
    J->state_final = S.state;
    J->ticks = S.ticks;
    J->fx = S.fx; J->fv = S.fv; J->ff = S.ff; J->fb = S.fb; J->fpe = S.fpe; J->fke = S.fke; J->fst = S.fst;
    J->bits = S.bits;
    // 64-bit step clocks reuse the FP64 arrays of the arena.
    J->fpt_last = (int64_t*)S.fpt_last;
    J->fpt2_last = (int64_t*)S.fpt2_last;
    J->tpt_last = (int64_t*)S.tpt_last;
    J->tpt2_last = (int64_t*)S.tpt2_last;
    J->wt_tick = S.wt_tick;
    int32_t* b = job->d_i32b;
    J->init_idx0 = b; J->init_idx1 = b + n; J->idx2_0 = b + 2 * n; J->idx2_1 = b + 3 * n; J->tpt2_well = b + 4 * n;
    J->cg_well = b + 5 * n;
    J->cg_last = S.cg_well;   // int64 [ncg][n]
    J->remaining = nullptr;   // the queue's counter of the job's slot, set at registration
    J->ck_xp = job->ck_xp; J->ck_rv = job->ck_rv; J->ck_cell = job->ck_cell; J->ck_sw = job->ck_sw;
    J->ck_ckey = job->ck_ckey; J->ck_cflip = job->ck_cflip; J->ck_nflip = job->ck_nflip;
    J->ck_ring = (longlong2*)job->ck_ring;
}

int fp32_type_of(const ldp_job* job) { return (job->k.dbl ? 2 : 0) + (job->k.over ? 1 : 0); }

bool fp32_queue_quiet(ldp_ctx* ctx, int type) {
    if (!ctx->fp32) return true;
    const Fp32Queue& Q = ctx->fp32->q[type];
    if (!Q.ready) return true;
    for (const ldp_job* j : Q.table)
        if (j && !j->done) return false;
    return true;
}

// One persistent launch of a queue with a given pair budget (serving).
int fp32_launch_type(ldp_ctx* ctx, int type, uint32_t pair_budget, cudaStream_t st) {
    Fp32Queue& Q = ctx->fp32->q[type];
    if (!Q.ready) return 0;
    return launch_fp32_persistent(type >= 2, (type & 1) != 0, Q.q, Q.s, pair_budget, Q.grid, Q.block, st);
}

// One persistent launch over all four model types' queues (serving): the
// queues are created if they were not, and the mixed kernel's slots on
// first use.
int fp32_launch_mixed(ldp_ctx* ctx, uint32_t pair_budget, cudaStream_t st) {
    if (!ctx->fp32) ctx->fp32 = new Fp32Runtime();
    Fp32Runtime& R = *ctx->fp32;
    const int ring = ctx->fp32_ring_slots ? ctx->fp32_ring_slots : 64;
    for (int t = 0; t < 4; ++t) {
        const int e = queue_init(ctx, R.q[t], t, ring);
        if (e) return e;
    }
    if (!R.mixed_mem) {
        const int block = 256;
        int bps = fp32_mixed_blocks_per_sm(block);
        if (ctx->fp32_blocks_per_sm) bps = std::min(bps, ctx->fp32_blocks_per_sm);
        bps = std::max(bps, 1);
        R.mixed_grid = ctx->sm_count * bps;
        const int64_t nslots = (int64_t)R.mixed_grid * block;
        int e = slots_init(nslots, ring, &R.mixed, &R.mixed_mem);
        if (e) return e;
        const size_t n = (size_t)(nslots / 32) + kMixedSmTypes;   // wtype, then sm_type
        cudaError_t ce = cudaMalloc((void**)&R.wtype, sizeof(int32_t) * n);
        if (ce == cudaSuccess) ce = cudaMemset(R.wtype, 0xff, sizeof(int32_t) * n);   // -1
        if (ce != cudaSuccess) return (int)ce;
    }
    MixedDev m;
    for (int t = 0; t < 4; ++t) m.q[t] = R.q[t].q;
    m.S = R.mixed;
    m.wtype = R.wtype;
    m.sm_type = R.wtype + R.mixed.nslots / 32;
    m.nwarps = R.mixed.nslots / 32;
    return launch_fp32_mixed(m, pair_budget, R.mixed_grid, 256, st);
}

// Slots of the mixed launches (0 before the first).
int64_t fp32_mixed_slots(ldp_ctx* ctx) { return ctx->fp32 ? ctx->fp32->mixed.nslots : 0; }

// Asynchronous copy of a queue's per-slot remaining counters and of its
// claimed-items count (serving).
int fp32_copy_remaining(ldp_ctx* ctx, int type, unsigned long long* host, unsigned long long* head,
                        cudaStream_t st) {
    Fp32Queue& Q = ctx->fp32->q[type];
    if (!Q.ready) return 0;
    cudaError_t e = cudaMemcpyAsync(host, Q.rem, sizeof(unsigned long long) * kFp32MaxJobs,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(head, Q.q.head, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    return (int)e;
}

// Slots of a queue's persistent grid and items published so far (serving).
int64_t fp32_nslots(ldp_ctx* ctx, int type) {
    const Fp32Queue& Q = ctx->fp32->q[type];
    return Q.ready ? Q.s.nslots : 0;
}
unsigned long long fp32_published(ldp_ctx* ctx, int type) {
    const Fp32Queue& Q = ctx->fp32->q[type];
    return Q.ready ? Q.tail : 0;
}

static Fp32Runtime* runtime(ldp_ctx* ctx) {
    if (!ctx->fp32) ctx->fp32 = new Fp32Runtime();
    return ctx->fp32;
}

// Registers the job (job table entry, remaining counter) and, unless
// publish is false, publishes all its trajectories as one item range.
int fp32_register(ldp_job* job, cudaStream_t stream, bool publish) {
    ldp_ctx* ctx = job->ctx;
    cudaStream_t st = stream ? stream : ctx->stream;
    Fp32Runtime* rt = runtime(ctx);
    const int type = fp32_type_of(job);
    Fp32Queue& Q = rt->q[type];
    int e = queue_init(ctx, Q, type, ctx->fp32_ring_slots ? ctx->fp32_ring_slots : 64);
    if (e) return e;
    if (Q.free_slots.empty()) return (int)cudaErrorMemoryAllocation;
    const int slot = Q.free_slots.back();
    Q.free_slots.pop_back();
    Q.table[slot] = job;
    job->fp32_type = type;
    job->fp32_slot = slot;
    job->fp32_published = 0;
    JobF J;
    fill_jobf(job, &J);
    J.remaining = &Q.rem[slot];
    int64_t* h = stage(Q);
    static_assert(sizeof(JobF) <= 4096 - 64, "JobF must fit the staging buffer");
    std::memcpy(h + 8, &J, sizeof(J));
    h[0] = (int64_t)job->ntraj;
    cudaMemcpyAsync(J.remaining, &h[0], sizeof(unsigned long long), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(&Q.q.jobs[slot], h + 8, sizeof(J), cudaMemcpyHostToDevice, st);
    cudaEventRecord(Q.stage_ev[Q.stage_last], st);
    ++job->launches;
    if (publish) return fp32_publish_range(job, job->ntraj, st);
    return (int)cudaGetLastError();
}

// Publishes the job's next `count` trajectories (after those published
// already) as one item range.
int fp32_publish_range(ldp_job* job, int64_t count, cudaStream_t stream) {
    ldp_ctx* ctx = job->ctx;
    cudaStream_t st = stream ? stream : ctx->stream;
    Fp32Queue& Q = ctx->fp32->q[job->fp32_type];
    count = std::min<int64_t>(count, job->ntraj - job->fp32_published);
    if (count <= 0) return 0;
    if (Q.nranges >= kFp32MaxRanges) return (int)cudaErrorMemoryAllocation;
    int64_t* h = stage(Q);
    const int64_t r = Q.nranges;
    Q.tail += (unsigned long long)count;
    h[1] = (int64_t)Q.tail;               // range_end
    h[2] = job->fp32_published;           // range_first
    h[3] = job->fp32_slot;                // range_job (low 32 bits)
    cudaMemcpyAsync(&Q.q.range_end[r], &h[1], sizeof(int64_t), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(&Q.q.range_first[r], &h[2], sizeof(int64_t), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(&Q.q.range_job[r], &h[3], sizeof(int32_t), cudaMemcpyHostToDevice, st);
    cudaEventRecord(Q.stage_ev[Q.stage_last], st);
    Q.nranges = r + 1;
    job->fp32_published += count;
    const int e = launch_fp32_publish(Q.q, Q.tail, (int32_t)Q.nranges, st);
    if (e) return e;
    ++job->launches;
    return (int)cudaGetLastError();
}

// Enqueues nlaunch persistent-kernel launches of the job's queue.
int fp32_pump(ldp_job* job, int nlaunch) {
    ldp_ctx* ctx = job->ctx;
    Fp32Queue& Q = ctx->fp32->q[job->fp32_type];
    const bool dbl = job->k.dbl, over = job->k.over;
    for (int i = 0; i < nlaunch; ++i) {
        const uint32_t pb = (uint32_t)std::min<uint64_t>(Q.pair_budget, 0xffffffffull);
        int e = launch_fp32_persistent(dbl, over, Q.q, Q.s, pb, Q.grid, Q.block, ctx->stream);
        if (e) return e;
        ++job->launches;
    }
    return 0;
}

// Launches needed for the job's queue to drain, assuming it runs alone.
int fp32_estimate_launches(const ldp_job* job) {
    const Fp32Queue& Q = job->ctx->fp32->q[job->fp32_type];
    const double pairs = (double)job->ntraj * (double)((job->nsteps + 1) / 2);
    const double cap = (double)Q.s.nslots * (double)Q.pair_budget;
    // A trajectory's steps run in order in one slot: at least its own length
    // in launches, however many slots are free.
    const double serial = (double)((job->nsteps + 1) / 2) / (double)Q.pair_budget;
    int n = (int)std::max(pairs / cap, serial) + 1;
    if (job->o.mode == LDP_MODE_FIRST_PASSAGE) n = std::max(1, n / 8);
    return std::min(n, 4096);
}

// Persistent launches that drain the type's queue for certain: a work-
// conserving list schedule of independent trajectories on m slots ends
// within total/m + longest (Graham's bound), in pairs of the launch budget.
int fp32_launch_bound(ldp_ctx* ctx, int type, double total_pairs, double max_pairs) {
    const Fp32Queue& Q = ctx->fp32->q[type];
    const double pb = (double)std::min<uint64_t>(Q.pair_budget, 0xffffffffull);
    const double n = std::ceil(total_pairs / ((double)Q.s.nslots * pb)) + std::ceil(max_pairs / pb) + 1.0;
    return (int)std::min(n, 1.0e6);
}

int fp32_snapshot_remaining(ldp_job* job, unsigned long long* dst, cudaStream_t stream) {
    const Fp32Queue& Q = job->ctx->fp32->q[job->fp32_type];
    return (int)cudaMemcpyAsync(dst, &Q.rem[job->fp32_slot], sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                stream);
}

int fp32_remaining(ldp_job* job, unsigned long long* rem) {
    const Fp32Queue& Q = job->ctx->fp32->q[job->fp32_type];
    return (int)cudaMemcpy(rem, &Q.rem[job->fp32_slot], sizeof(unsigned long long), cudaMemcpyDeviceToHost);
}

__global__ void ssum_to_time_kernel(const int64_t* ssum, double* sums, double dt, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sums[i] = dt * (double)ssum[i];
}

// Post-processing after all trajectories retired: event-duration sums in
// time units, then the MSD of the saved frames (lean: the MSD instance that
// fits beside running persistent blocks; same results).
int fp32_finalize(ldp_job* job, cudaStream_t stream, bool lean) {
    cudaStream_t st = stream ? stream : job->ctx->stream;
    const int64_t n = (int64_t)LDP_NSUM * job->ntraj;
    ssum_to_time_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(job->d_ssum, job->st.sums, job->k.dt, n);
    int e = (int)cudaGetLastError();
    if (e) return e;
    ++job->launches;
    if (job->o.mode == LDP_MODE_FIXED_STEPS && !job->lags.empty()) {
        e = launch_msd(job->st.fx, job->nframe, job->ntraj, job->d_lags, (int64_t)job->lags.size(), job->d_msd0,
                       job->d_msd, st, lean ? LDP_MSD_FP32_LEAN : LDP_MSD_FP32);
        if (e) return e;
        job->launches += 2;
    }
    return 0;
}

void fp32_release(ldp_job* job) {
    if (job->fp32_slot < 0 || !job->ctx->fp32) return;
    Fp32Queue& Q = job->ctx->fp32->q[job->fp32_type];
    Q.table[job->fp32_slot] = nullptr;
    Q.free_slots.push_back(job->fp32_slot);
    job->fp32_slot = -1;
}

void fp32_destroy_runtime(ldp_ctx* ctx) {
    if (!ctx->fp32) return;
    if (ctx->fp32->mixed_mem) cudaFree(ctx->fp32->mixed_mem);
    if (ctx->fp32->wtype) cudaFree(ctx->fp32->wtype);
    for (auto& Q : ctx->fp32->q) {
        if (Q.qmem) cudaFree(Q.qmem);
        if (Q.smem) cudaFree(Q.smem);
        if (Q.h_stage) cudaFreeHost(Q.h_stage);
        for (auto& ev : Q.stage_ev)
            if (ev) cudaEventDestroy(ev);
    }
    delete ctx->fp32;
    ctx->fp32 = nullptr;
}

}  // namespace ldp

extern "C" ldp_status ldp_ctx_set_fp32_shape(ldp_ctx* ctx, int block, int blocks_per_sm, uint64_t pair_budget,
                                             int ring_slots) {
    if (!ctx) return LDP_ERR_INVALID;
    if (ctx->fp32) {
        ldp_set_error(ctx, "the FP32 launch shape is fixed once the context ran an FP32 job");
        return LDP_ERR_INVALID;
    }
    if (block < 0 || (block && (block % 32 || block > 256)) || blocks_per_sm < 0 ||
        (ring_slots && (ring_slots < 16 || (ring_slots & (ring_slots - 1))))) {
        ldp_set_error(ctx, "invalid FP32 shape: block %d (multiple of 32, <= 256), ring %d (power of two >= 16)",
                      block, ring_slots);
        return LDP_ERR_INVALID;
    }
    ctx->fp32_block = block;
    ctx->fp32_blocks_per_sm = blocks_per_sm;
    ctx->fp32_pair_budget = pair_budget;
    ctx->fp32_ring_slots = ring_slots;
    return LDP_OK;
}

extern "C" ldp_status ldp_ctx_get_fp32_shape(ldp_ctx* ctx, int* block, int* grid, uint64_t* pair_budget,
                                             int* ring_slots) {
    if (!ctx) return LDP_ERR_INVALID;
    int b = ctx->fp32_block ? ctx->fp32_block : 256, g = 0;
    uint64_t pb = ctx->fp32_pair_budget ? ctx->fp32_pair_budget : (1u << 15);
    int r = ctx->fp32_ring_slots ? ctx->fp32_ring_slots : 64;
    if (ctx->fp32)
        for (auto& Q : ctx->fp32->q)
            if (Q.ready) { b = Q.block; g = Q.grid; pb = Q.pair_budget; r = Q.s.ring_slots; break; }
    if (block) *block = b;
    if (grid) *grid = g;
    if (pair_budget) *pair_budget = pb;
    if (ring_slots) *ring_slots = r;
    return LDP_OK;
}
