// ldp_fp32_state.cpp -- continuation of FP32 batched runs.
//
// The reference chains long runs through .restart files
// (src/langevinDynamicsSingleBarrier.h:1048-1275: WRITERESTART at the end of
// a run, READRESTART with NUMBEROFPREVIOUSSTEPS in the next).  The FP32
// batched path keeps no per-event lists, which those files hold, so it has a
// file of its own: ldp_job_keep_state makes a job keep every trajectory's
// state at its last step (cell-local position, velocity or previous random
// force, cell, barrier cache and pending flips, the cell-table ring,
// statistics clocks), ldp_job_save_state writes that state with the counts,
// duration sums and frames, and ldp_job_load_state loads it into a job whose
// NUMBEROFPREVIOUSSTEPS equals the steps it holds.  The random streams are
// keyed by (seed, job id, trajectory, absolute step), so the continued run
// equals the uninterrupted one bit for bit.
//
// File: "LDPF32ST", version, a header (layout and the parameters the
// streams and the step depend on), then the arrays, each preceded by its
// byte count; little-endian, as the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ldp_internal.h"

namespace {

constexpr char kMagic[8] = {'L', 'D', 'P', 'F', '3', '2', 'S', 'T'};
constexpr uint32_t kVersion = 1;

struct Header {
    int32_t model, overdamped, lanes, ranks, runs, first_rank, ring_slots, n_cg, nser, pad;
    int64_t ntraj, tick_cap, nframe;
    uint64_t steps, freq_save;
    uint32_t seed, job_id;
    double dt, L, tau, gamma, mass, temperature, kb, x0;
    double heights[2][2], half_width[2], position[2];
    int32_t eq, cg_sizes[LDP_MAX_CG], pad2;
    double eq_constant;
};

int ring_of(const ldp_ctx* ctx) { return ctx->fp32_ring_slots ? ctx->fp32_ring_slots : 64; }
int nser_of(const ldp_params& p) { return 1 + (p.write_x ? 6 : 0); }
int ncg_rows(const ldp_params& p) { return p.n_cg > 0 ? p.n_cg : 1; }

void fill_header(const ldp_job* job, uint64_t steps, Header* h) {
    std::memset(h, 0, sizeof(*h));
    const ldp_params& p = job->p;
    h->model = p.model;
    h->overdamped = p.overdamped;
    h->lanes = job->o.lanes;
    h->ranks = job->o.ranks;
    h->runs = p.number_of_runs;
    h->first_rank = job->o.first_rank;
    h->ring_slots = job->ck_ring_slots;
    h->n_cg = p.n_cg;
    h->nser = nser_of(p);
    h->ntraj = job->ntraj;
    h->tick_cap = job->o.tick_cap;
    h->nframe = (int64_t)(steps / p.freq_save + 1);
    h->steps = steps;
    h->freq_save = p.freq_save;
    h->seed = job->seed;
    h->job_id = job->o.job_id;
    h->dt = p.timestep;
    h->L = p.periodic_length;
    h->tau = p.tau;
    h->gamma = p.gamma;
    h->mass = p.mass;
    h->temperature = p.temperature;
    h->kb = p.kb;
    h->x0 = p.x0;
    std::memcpy(h->heights, p.barrier_heights, sizeof(h->heights));
    std::memcpy(h->half_width, p.barrier_half_width, sizeof(h->half_width));
    std::memcpy(h->position, p.barrier_position, sizeof(h->position));
    h->eq = p.eq;
    std::memcpy(h->cg_sizes, p.cg_sizes, sizeof(h->cg_sizes));
    h->eq_constant = p.eq_constant;
}

// One device array of the file: where it is and how many bytes the file
// holds of it (frame series: the file's frames, a prefix of the job's).
struct Part {
    void* dev;
    size_t bytes;
};

// The arrays in file order.  nframe: frames in the file; the job's own
// frame rows may be more (a continued job), its ticks per trajectory more.
std::vector<Part> parts(ldp_job* job, int64_t nframe_file) {
    const ldp::TrajState& S = job->st;
    const int64_t n = job->ntraj;
    const ldp_params& p = job->p;
    std::vector<Part> v;
    v.push_back({S.counts, sizeof(int64_t) * LDP_NCOUNT * n});
    v.push_back({job->d_ssum, sizeof(int64_t) * LDP_NSUM * n});
    v.push_back({S.state0, sizeof(int32_t) * n});
    v.push_back({S.v0, sizeof(double) * n});
    v.push_back({S.x, sizeof(double) * n});
    v.push_back({S.v, sizeof(double) * n});
    v.push_back({S.state, sizeof(int32_t) * n});
    v.push_back({S.bits, sizeof(int32_t) * n});
    v.push_back({S.fpt_last, sizeof(int64_t) * 4 * n});   // fpt, fpt2, tpt, tpt2 step clocks
    v.push_back({S.wt_tick, sizeof(int64_t) * n});
    v.push_back({job->d_i32b, sizeof(int32_t) * (5 + ncg_rows(p)) * n});
    v.push_back({S.cg_well, sizeof(int64_t) * ncg_rows(p) * n});   // FPTCG step clocks
    const size_t fstride = (size_t)std::max<int64_t>(job->nframe, 1) * n;
    for (int k = 0; k < nser_of(p); ++k)
        v.push_back({(double*)S.fx + k * fstride, sizeof(double) * (size_t)nframe_file * n});
    v.push_back({job->ck_xp, sizeof(int32_t) * 5 * n});   // xp, rv, cell, sw, ckey
    v.push_back({job->ck_cflip, sizeof(int64_t) * 2 * n});
    v.push_back({job->ck_ring, sizeof(int64_t) * 2 * (size_t)job->ck_ring_slots * n});
    return v;
}

ldp_status fail(ldp_job* job, ldp_status st, const std::string& m) {
    ldp_set_error(job->ctx, "%s", m.c_str());
    return st;
}

}  // namespace

extern "C" ldp_status ldp_job_keep_state(ldp_job* job) {
    if (!job) return LDP_ERR_INVALID;
    if (job->o.precision != LDP_PREC_FP32_BATCHED || job->o.mode != LDP_MODE_FIXED_STEPS)
        return fail(job, LDP_ERR_UNSUPPORTED, "kept state is for FP32 batched jobs in fixed-step mode (FP64 plain "
                                              "jobs continue through .restart files)");
    if (job->submitted || job->arena)
        return fail(job, LDP_ERR_INVALID, "ldp_job_keep_state must precede ldp_submit and ldp_job_load_state");
    job->keep_state = true;
    job->ck_ring_slots = ring_of(job->ctx);
    return LDP_OK;
}

extern "C" ldp_status ldp_job_save_state(ldp_job* job, const char* path) {
    if (!job || !path) return LDP_ERR_INVALID;
    if (!job->keep_state || !job->ck_xp) return fail(job, LDP_ERR_INVALID, "the job did not keep its state");
    if (!job->done) {
        const ldp_status st = ldp_wait(job->ctx, job);
        if (st != LDP_OK) return st;
    }
    const uint64_t steps = job->steps_before + job->nsteps;
    Header h;
    fill_header(job, steps, &h);
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(job, LDP_ERR_IO, std::string("can't open state file (") + path + ")");
    cudaSetDevice(job->ctx->device);
    bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&kVersion, 4, 1, f) == 1 &&
              std::fwrite(&h, sizeof(h), 1, f) == 1;
    std::vector<char> buf;
    const auto ps = parts(job, h.nframe);
    for (size_t i = 0; ok && i < ps.size(); ++i) {
        const Part& pt = ps[i];
        const uint64_t b = pt.bytes;
        buf.resize(b);
        if (b && cudaMemcpy(buf.data(), pt.dev, b, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(f);
            return fail(job, LDP_ERR_DEVICE, "copy of the kept state failed");
        }
        ok = std::fwrite(&b, 8, 1, f) == 1 && (b == 0 || std::fwrite(buf.data(), 1, b, f) == b);
    }
    // waiting-time ticks, [ntraj][tick_cap]
    if (ok) {
        const uint64_t b = h.tick_cap > 0 ? sizeof(int64_t) * (size_t)h.tick_cap * job->ntraj : 0;
        buf.resize(b);
        if (b && cudaMemcpy(buf.data(), job->st.ticks, b, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(f);
            return fail(job, LDP_ERR_DEVICE, "copy of the waiting-time ticks failed");
        }
        ok = std::fwrite(&b, 8, 1, f) == 1 && (b == 0 || std::fwrite(buf.data(), 1, b, f) == b);
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? LDP_OK : fail(job, LDP_ERR_IO, std::string("write of state file failed (") + path + ")");
}

extern "C" ldp_status ldp_job_load_state(ldp_job* job, const char* path) {
    if (!job || !path) return LDP_ERR_INVALID;
    if (job->o.precision != LDP_PREC_FP32_BATCHED || job->o.mode != LDP_MODE_FIXED_STEPS)
        return fail(job, LDP_ERR_UNSUPPORTED, "a kept state continues FP32 batched fixed-step jobs");
    if (job->submitted || job->arena) return fail(job, LDP_ERR_INVALID, "ldp_job_load_state must precede ldp_submit");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(job, LDP_ERR_RESTART, std::string("can't open state file (") + path + ")");
    char magic[8];
    uint32_t ver = 0;
    Header h;
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0 || std::fread(&ver, 4, 1, f) != 1 ||
        ver != kVersion || std::fread(&h, sizeof(h), 1, f) != 1) {
        std::fclose(f);
        return fail(job, LDP_ERR_RESTART, std::string("not a state file of this library (") + path + ")");
    }
    job->keep_state = true;   // a continued run can be continued again
    job->ck_ring_slots = ring_of(job->ctx);
    Header want;
    fill_header(job, h.steps, &want);
    const ldp_params& p = job->p;
    std::string bad;
    if (p.number_of_previous_steps != h.steps) bad = "NUMBEROFPREVIOUSSTEPS differs from the steps the file holds";
    else if (h.steps % 4 != 0) bad = "the file's step count is not a multiple of 4";
    else if (h.model != want.model || h.overdamped != want.overdamped) bad = "model";
    else if (h.lanes != want.lanes || h.ranks != want.ranks || h.runs != want.runs || h.first_rank != want.first_rank ||
             h.ntraj != want.ntraj) bad = "layout (lanes, ranks, runs, first_rank)";
    else if (h.ring_slots != want.ring_slots) bad = "cell-table ring slots of the context";
    else if (h.n_cg != want.n_cg || std::memcmp(h.cg_sizes, want.cg_sizes, sizeof(h.cg_sizes)) != 0) bad = "FPTCG";
    else if (h.nser != want.nser) bad = "WRITEX";
    else if (h.seed != want.seed || h.job_id != want.job_id) bad = "RANDOMSEED or job id (the random streams)";
    else if (h.freq_save != want.freq_save) bad = "FREQSAVE";
    else if (h.tick_cap > want.tick_cap) bad = "waiting-time tick capacity";
    else if (h.dt != want.dt || h.L != want.L || h.tau != want.tau || h.gamma != want.gamma || h.mass != want.mass ||
             h.temperature != want.temperature || h.kb != want.kb || h.x0 != want.x0 || h.eq != want.eq ||
             h.eq_constant != want.eq_constant || std::memcmp(h.heights, want.heights, sizeof(h.heights)) ||
             std::memcmp(h.half_width, want.half_width, sizeof(h.half_width)) ||
             std::memcmp(h.position, want.position, sizeof(h.position)))
        bad = "model parameters";
    if (!bad.empty()) {
        std::fclose(f);
        return fail(job, LDP_ERR_RESTART, "state file does not match the job: " + bad + " (" + path + ")");
    }
    cudaSetDevice(job->ctx->device);
    if (ldp_job_arena(job, true) == 0) {
        std::fclose(f);
        return fail(job, LDP_ERR_NOMEM, "device allocation of the job failed");
    }
    if (cudaStreamSynchronize(job->ctx->stream) != cudaSuccess) {
        std::fclose(f);
        return fail(job, LDP_ERR_DEVICE, "job arena set-up failed");
    }
    std::vector<char> buf;
    const auto ps = parts(job, h.nframe);
    bool ok = true;
    for (size_t i = 0; ok && i <= ps.size(); ++i) {
        uint64_t b = 0;
        if (std::fread(&b, 8, 1, f) != 1) { ok = false; break; }
        const bool ticks = i == ps.size();
        const uint64_t want_b = ticks ? (h.tick_cap > 0 ? sizeof(int64_t) * (size_t)h.tick_cap * job->ntraj : 0)
                                      : ps[i].bytes;
        if (b != want_b) { ok = false; break; }
        buf.resize(b);
        if (b && std::fread(buf.data(), 1, b, f) != b) { ok = false; break; }
        if (!b) continue;
        if (!ticks) {
            if (cudaMemcpy(ps[i].dev, buf.data(), b, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
        } else {
            // rows of tick_cap(file) into rows of tick_cap(job)
            const size_t rf = sizeof(int64_t) * (size_t)h.tick_cap, rj = sizeof(int64_t) * (size_t)job->o.tick_cap;
            if (cudaMemcpy2D(job->st.ticks, rj, buf.data(), rf, rf, (size_t)job->ntraj, cudaMemcpyHostToDevice) !=
                cudaSuccess)
                ok = false;
        }
    }
    std::fclose(f);
    if (!ok) return fail(job, LDP_ERR_RESTART, std::string("state file truncated or damaged (") + path + ")");
    job->fp32_resume = true;
    job->restored = true;
    job->steps_before = h.steps;
    return LDP_OK;
}
