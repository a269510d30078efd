// ldp_restart.cpp -- .restart files in the reference's layout; job
// checkpoint and resume on the FP64 plain path.
//
// One file per (virtual rank, trial), named <base>_%05d_%05d.restart, as
// LangevinEquationSIMDMultiple::Write/ReadRestartFile write and read them
// (src/langevinDynamicsSingleBarrier.h:1048-1202,
// src/langevinDynamicsDoubleBarrier.h:1202-1368): a header of the run's
// parameters and step count, the per-lane TrajectoryData
// (S.h:385-576 / D.h:414-640, the overdamped random force S.h:2776-2785),
// the lazily grown barrier table(s) (BarrierStatus S.h:66-118 on
// FiniteInifiniteIntegerTickArray1D, src/DataLocator.h:167-174) and the
// trailer 9990.  Scalars are little-endian int32 / uint64 / float64 as the
// reference's StreamerWriter (src/streamer.h:50-100) emits them.
//
// The layout and the field order have to be the reference's so that files
// move both ways; the code that reads and writes them is this library's.
//
// What the layout does not hold and how it is mapped:
// * The reference keeps every event; the device path keeps counts and sums
//   and, with event_cap > 0, the per-event lists themselves, which are what
//   a written file holds.
// * The reference's barrier table stores (state, step last observed) for
//   every cell between the lowest and highest touched by any lane of the
//   file.  The device ring stores (state when left, pending flip step nb)
//   for the cells a trajectory visited.  Written as (state, S) when nb > S
//   (no flip before the save step S) and (state ^ 1, nb) otherwise (it
//   flipped at nb); cells the trajectory never entered are written as the
//   device would create them (its default state, step 0).  Read back, each
//   cell's pending flip is drawn from its step with the geometric waiting
//   time of its state (exact in law: the flips are memoryless).
// * The reference's MT19937 stream positions (three (renew, progress)
//   pairs) have no meaning for counter-based Philox streams keyed by step;
//   they are written as zeros and ignored on reading.
// * An exact-resume block follows the trailer in files written here: the
//   ring, pending flips, counts and sums of every lane, so that a run
//   chained through a restart file equals the uninterrupted run bit for
//   bit.  The reference's reader stops at the trailer
//   (S.h:1195-1197) and never sees it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ldp_engine.h"
#include "ldp_internal.h"

namespace ldp {
namespace {

constexpr int32_t kSignature = 2345;      // m_Signature, S.h:1011
constexpr int32_t kTrajMark = 9998;       // TrajectoryData block, S.h:434
constexpr int32_t kDoubleMark = 9948;     // after the two tables, D.h:640
constexpr int32_t kTrailer = 9990;        // S.h:1128
constexpr int32_t kExtMagic = 0x5844504c; // "LPDX": exact-resume block
constexpr int32_t kExtVersion = 1;
constexpr int64_t kNever = (int64_t)((1ull << 62) - 1);
constexpr uint32_t kTagInit = 1, kTagCell = 3, kTagResume = 5, kTagResumeCell = 6;

// ---------------------------------------------------------------- bytes
struct Rd {
    const uint8_t* b;
    size_t n, o = 0;
    bool bad = false;
    template <class T>
    T get() {
        T v{};
        if (bad || n - o < sizeof(T)) { bad = true; return v; }
        std::memcpy(&v, b + o, sizeof(T));
        o += sizeof(T);
        return v;
    }
    int32_t i32() { return get<int32_t>(); }
    uint64_t u64() { return get<uint64_t>(); }
    int64_t i64() { return get<int64_t>(); }
    double f64() { return get<double>(); }
    std::vector<double> vec() {
        const uint64_t m = u64();
        if (bad || m > (n - o) / 8) { bad = true; return {}; }
        std::vector<double> v(m);
        if (m) std::memcpy(v.data(), b + o, 8 * m);
        o += 8 * m;
        return v;
    }
};

struct Wr {
    std::vector<uint8_t>& out;
    template <class T>
    void put(T v) {
        const size_t o = out.size();
        out.resize(o + sizeof(T));
        std::memcpy(out.data() + o, &v, sizeof(T));
    }
    void i32(int32_t v) { put(v); }
    void u64(uint64_t v) { put(v); }
    void i64(int64_t v) { put(v); }
    void f64(double v) { put(v); }
    void vec(const std::vector<double>& v) {
        u64(v.size());
        const size_t o = out.size();
        out.resize(o + 8 * v.size());
        if (!v.empty()) std::memcpy(out.data() + o, v.data(), 8 * v.size());
    }
};

// ---------------------------------------------------------------- model
struct Layout {
    bool dbl = false, over = false, tpt = false, cg = false;
};

struct CgData {
    std::vector<double> list;
    double last = 0.0;
    int32_t up = 0, well = 0;
};

struct Lane {
    double x = 0, v = 0, f = 0, e = 0, eta = 0, barrier = 0, xp = 0;
    std::vector<double> series[8];   // X V F PE KE Eta State Barrier
    double state = 0, prev_state = 0;
    std::vector<double> bparams;     // 3 (single) or 10 (double), file order
    double sc[2] = {0, 0};
    double well = 0, cell = 0, well_prev = 0, cell_prev = 0;
    int32_t on_well = 0, on_cell = 0;
    double lb = 0, lb_prev = 0, lb_st = 0, lb_prev_st = 0;
    int32_t on_lb = 0, on_lb_st = 0;
    double v0 = 0, eta0 = 0, state0 = 0;
    double well_st = 0, cell_st = 0, well_prev_st = 0, cell_prev_st = 0;
    int32_t on_well_st = 0, on_cell_st = 0;
    double wt_prev = 0;
    int32_t wt_passed = 0;
    std::vector<double> ticks;
    std::vector<double> fpt, instant, initial;
    double fpt_last = 0;
    int32_t fpt_up = 0;
    double init_state[2] = {0, 0};
    int32_t init_idx[2] = {0, 0};
    std::vector<double> fpt2;
    double fpt2_last = 0;
    int32_t fpt2_up = 0;
    int32_t idx2[2] = {0, 0};
    std::vector<double> tpt;
    double tpt_last = 0;
    int32_t tpt_up = 0;
    std::vector<double> tpt2;
    double tpt2_last = 0;
    int32_t tpt2_up = 0, tpt2_well = 0;
    std::vector<int32_t> cg_sizes;
    std::vector<CgData> cg;
};

struct Table {
    int32_t min_id = 0;
    std::vector<int32_t> state;   // [ncell][W]
    std::vector<uint64_t> step;   // [ncell][W]
    size_t ncell(int W) const { return W ? state.size() / (size_t)W : 0; }
};

struct LaneExt {
    int64_t nflip = 0;
    int32_t bits = 0;
    int64_t counts[LDP_NCOUNT] = {};
    double sums[LDP_NSUM] = {};
    std::vector<int64_t> tag, data;
};

struct File {
    int32_t sig = kSignature, W = 0;
    double x0 = 0, v0 = 0, gamma = 0, kb = 0, T = 0, m = 0, dt = 0;
    uint64_t nsteps = 0;
    int32_t wt = 0;
    uint64_t freq_stat = 1, freq_save = 1;
    int32_t save_x = 1, save_v = 0, save_f = 0, save_e = 0, rand_v = 0, rand_eta = 0;
    double L = 0, H[4] = {0, 0, 0, 0}, init_state = 0, pos[2] = {0, 0}, xc = 0;
    int32_t rand_state = 0, same_init = 0;
    double q = 0.2, tau = 0, eta0 = 0;
    int32_t save_eta = 0, save_state = 0, save_barrier = 0, rank = 0;
    int64_t renew[3] = {0, 0, 0};
    uint64_t progress[3] = {0, 0, 0};
    int32_t lane_wt = 0, lane_fpt = 0;
    std::vector<Lane> lanes;
    Table tables[2];
    std::vector<double> rf;
    bool has_ext = false;
    int32_t ext_slots = 0;
    std::vector<LaneExt> ext;
};

Layout layout_of(const ldp_params& p) {
    Layout L;
    L.dbl = p.model == LDP_MODEL_DOUBLE;
    L.over = p.overdamped != 0;
    L.tpt = p.tpt != 0;
    L.cg = p.fptcg != 0;
    return L;
}

// ---------------------------------------------------------------- decode
bool decode(const std::vector<uint8_t>& bytes, const Layout& Ly, File* f, std::string* err) {
    Rd r{bytes.data(), bytes.size()};
    f->sig = r.i32();
    if (!r.bad && f->sig != kSignature) { *err = "inconsistent signature"; return false; }
    f->W = r.i32();
    if (!r.bad && (f->W < 1 || f->W > 4096)) { *err = "implausible simd width"; return false; }
    f->x0 = r.f64(); f->v0 = r.f64(); f->gamma = r.f64(); f->kb = r.f64(); f->T = r.f64(); f->m = r.f64();
    f->dt = r.f64();
    f->nsteps = r.u64();
    f->wt = r.i32();
    f->freq_stat = r.u64();
    f->freq_save = r.u64();
    f->save_x = r.i32(); f->save_v = r.i32(); f->save_f = r.i32(); f->save_e = r.i32();
    f->rand_v = r.i32(); f->rand_eta = r.i32();
    f->L = r.f64();
    const int nh = Ly.dbl ? 4 : 2;
    for (int i = 0; i < nh; ++i) f->H[i] = r.f64();
    f->init_state = r.f64();
    if (Ly.dbl) { f->pos[0] = r.f64(); f->pos[1] = r.f64(); f->xc = r.f64(); }
    f->rand_state = r.i32(); f->same_init = r.i32();
    f->q = r.f64(); f->tau = r.f64(); f->eta0 = r.f64();
    f->save_eta = r.i32(); f->save_state = r.i32(); f->save_barrier = r.i32();
    f->rank = r.i32();
    for (int i = 0; i < 3; ++i) { f->renew[i] = r.i64(); f->progress[i] = r.u64(); }
    if (r.i32() != kTrajMark && !r.bad) { *err = "restart file corrupted (trajectory block)"; return false; }
    f->lane_wt = r.i32();
    f->lane_fpt = r.i32();
    if (r.bad) { *err = "restart file truncated"; return false; }
    f->lanes.assign(f->W, Lane());
    for (int i = 0; i < f->W && !r.bad; ++i) {
        Lane& a = f->lanes[i];
        a.x = r.f64(); a.v = r.f64(); a.f = r.f64(); a.e = r.f64(); a.eta = r.f64(); a.barrier = r.f64();
        if (Ly.dbl) a.xp = r.f64();
        for (int s = 0; s < 8; ++s) a.series[s] = r.vec();
        a.state = r.f64(); a.prev_state = r.f64();
        a.bparams.resize(Ly.dbl ? 10 : 3);
        for (double& b : a.bparams) b = r.f64();
        a.sc[0] = r.f64(); a.sc[1] = r.f64();
        a.well = r.f64(); a.cell = r.f64(); a.well_prev = r.f64(); a.cell_prev = r.f64();
        a.on_well = r.i32(); a.on_cell = r.i32();
        if (Ly.dbl) {
            a.lb = r.f64(); a.lb_prev = r.f64(); a.on_lb = r.i32();
            a.lb_st = r.f64(); a.lb_prev_st = r.f64(); a.on_lb_st = r.i32();
        }
        a.v0 = r.f64(); a.eta0 = r.f64(); a.state0 = r.f64();
        a.well_st = r.f64(); a.cell_st = r.f64(); a.well_prev_st = r.f64(); a.cell_prev_st = r.f64();
        a.on_well_st = r.i32(); a.on_cell_st = r.i32();
        if (f->lane_wt) { a.wt_prev = r.f64(); a.wt_passed = r.i32(); a.ticks = r.vec(); }
        if (f->lane_fpt) {
            a.fpt = r.vec(); a.instant = r.vec(); a.initial = r.vec();
            a.fpt_last = r.f64(); a.fpt_up = r.i32();
            a.init_state[0] = r.f64(); a.init_state[1] = r.f64();
            a.init_idx[0] = r.i32(); a.init_idx[1] = r.i32();
            a.fpt2 = r.vec(); a.fpt2_last = r.f64(); a.fpt2_up = r.i32();
            a.idx2[0] = r.i32(); a.idx2[1] = r.i32();
        }
        if (Ly.tpt) {
            a.tpt = r.vec(); a.tpt_last = r.f64(); a.tpt_up = r.i32();
            a.tpt2 = r.vec(); a.tpt2_last = r.f64(); a.tpt2_up = r.i32(); a.tpt2_well = r.i32();
        }
        if (Ly.cg) {
            const uint64_t ncg = r.u64();
            if (r.bad || ncg > 1024) { r.bad = true; break; }
            a.cg_sizes.resize(ncg);
            for (auto& s : a.cg_sizes) s = r.i32();
            a.cg.resize(ncg);
            for (auto& c : a.cg) { c.list = r.vec(); c.last = r.f64(); c.up = r.i32(); c.well = r.i32(); }
        }
    }
    const int ntab = Ly.dbl ? 2 : 1;
    for (int t = 0; t < ntab && !r.bad; ++t) {
        const uint64_t nc = r.u64();
        if (r.bad || nc > (r.n - r.o) / 12 / (uint64_t)f->W + 1) { r.bad = true; break; }
        Table& tb = f->tables[t];
        tb.state.resize(nc * f->W);
        tb.step.resize(nc * f->W);
        for (uint64_t c = 0; c < nc; ++c)
            for (int i = 0; i < f->W; ++i) {
                tb.state[c * f->W + i] = r.i32();
                tb.step[c * f->W + i] = r.u64();
            }
        tb.min_id = r.i32();
    }
    if (Ly.dbl && !r.bad && r.i32() != kDoubleMark && !r.bad) { *err = "wrong signiture after the barrier tables"; return false; }
    if (Ly.over) {
        f->rf.resize(f->W);
        for (double& x : f->rf) x = r.f64();
    }
    if (r.bad) { *err = "restart file truncated or of another layout (model / TPT / FPTCG settings)"; return false; }
    if (r.i32() != kTrailer || r.bad) { *err = "restart file corrupted"; return false; }
    f->has_ext = false;
    if (r.o < r.n) {
        if (r.i32() != kExtMagic || r.bad) { *err = "unknown data after the restart trailer"; return false; }
        if (r.i32() != kExtVersion) { *err = "unsupported exact-resume block version"; return false; }
        f->ext_slots = r.i32();
        const int32_t lanes = r.i32();
        if (r.bad || lanes != f->W || f->ext_slots < 1 || f->ext_slots > (1 << 20)) {
            *err = "exact-resume block corrupted";
            return false;
        }
        f->ext.assign(f->W, LaneExt());
        for (auto& e : f->ext) {
            e.nflip = r.i64();
            e.bits = r.i32();
            r.i32();
            for (auto& c : e.counts) c = r.i64();
            for (auto& s : e.sums) s = r.f64();
            e.tag.resize(f->ext_slots);
            e.data.resize(f->ext_slots);
            for (int s = 0; s < f->ext_slots; ++s) { e.tag[s] = r.i64(); e.data[s] = r.i64(); }
        }
        if (r.bad || r.o != r.n) { *err = "exact-resume block corrupted"; return false; }
        f->has_ext = true;
    }
    return true;
}

// ---------------------------------------------------------------- encode
void encode(const File& f, const Layout& Ly, std::vector<uint8_t>* out) {
    out->clear();
    Wr w{*out};
    w.i32(f.sig); w.i32(f.W);
    w.f64(f.x0); w.f64(f.v0); w.f64(f.gamma); w.f64(f.kb); w.f64(f.T); w.f64(f.m);
    w.f64(f.dt);
    w.u64(f.nsteps);
    w.i32(f.wt);
    w.u64(f.freq_stat); w.u64(f.freq_save);
    w.i32(f.save_x); w.i32(f.save_v); w.i32(f.save_f); w.i32(f.save_e);
    w.i32(f.rand_v); w.i32(f.rand_eta);
    w.f64(f.L);
    for (int i = 0; i < (Ly.dbl ? 4 : 2); ++i) w.f64(f.H[i]);
    w.f64(f.init_state);
    if (Ly.dbl) { w.f64(f.pos[0]); w.f64(f.pos[1]); w.f64(f.xc); }
    w.i32(f.rand_state); w.i32(f.same_init);
    w.f64(f.q); w.f64(f.tau); w.f64(f.eta0);
    w.i32(f.save_eta); w.i32(f.save_state); w.i32(f.save_barrier);
    w.i32(f.rank);
    for (int i = 0; i < 3; ++i) { w.i64(f.renew[i]); w.u64(f.progress[i]); }
    w.i32(kTrajMark);
    w.i32(f.lane_wt);
    w.i32(f.lane_fpt);
    for (const Lane& a : f.lanes) {
        w.f64(a.x); w.f64(a.v); w.f64(a.f); w.f64(a.e); w.f64(a.eta); w.f64(a.barrier);
        if (Ly.dbl) w.f64(a.xp);
        for (int s = 0; s < 8; ++s) w.vec(a.series[s]);
        w.f64(a.state); w.f64(a.prev_state);
        for (double b : a.bparams) w.f64(b);
        w.f64(a.sc[0]); w.f64(a.sc[1]);
        w.f64(a.well); w.f64(a.cell); w.f64(a.well_prev); w.f64(a.cell_prev);
        w.i32(a.on_well); w.i32(a.on_cell);
        if (Ly.dbl) {
            w.f64(a.lb); w.f64(a.lb_prev); w.i32(a.on_lb);
            w.f64(a.lb_st); w.f64(a.lb_prev_st); w.i32(a.on_lb_st);
        }
        w.f64(a.v0); w.f64(a.eta0); w.f64(a.state0);
        w.f64(a.well_st); w.f64(a.cell_st); w.f64(a.well_prev_st); w.f64(a.cell_prev_st);
        w.i32(a.on_well_st); w.i32(a.on_cell_st);
        if (f.lane_wt) { w.f64(a.wt_prev); w.i32(a.wt_passed); w.vec(a.ticks); }
        if (f.lane_fpt) {
            w.vec(a.fpt); w.vec(a.instant); w.vec(a.initial);
            w.f64(a.fpt_last); w.i32(a.fpt_up);
            w.f64(a.init_state[0]); w.f64(a.init_state[1]);
            w.i32(a.init_idx[0]); w.i32(a.init_idx[1]);
            w.vec(a.fpt2); w.f64(a.fpt2_last); w.i32(a.fpt2_up);
            w.i32(a.idx2[0]); w.i32(a.idx2[1]);
        }
        if (Ly.tpt) {
            w.vec(a.tpt); w.f64(a.tpt_last); w.i32(a.tpt_up);
            w.vec(a.tpt2); w.f64(a.tpt2_last); w.i32(a.tpt2_up); w.i32(a.tpt2_well);
        }
        if (Ly.cg) {
            w.u64(a.cg_sizes.size());
            for (int32_t s : a.cg_sizes) w.i32(s);
            for (const auto& c : a.cg) { w.vec(c.list); w.f64(c.last); w.i32(c.up); w.i32(c.well); }
        }
    }
    for (int t = 0; t < (Ly.dbl ? 2 : 1); ++t) {
        const Table& tb = f.tables[t];
        const size_t nc = tb.ncell(f.W);
        w.u64(nc);
        for (size_t c = 0; c < nc; ++c)
            for (int i = 0; i < f.W; ++i) {
                w.i32(tb.state[c * f.W + i]);
                w.u64(tb.step[c * f.W + i]);
            }
        w.i32(tb.min_id);
    }
    if (Ly.dbl) w.i32(kDoubleMark);
    if (Ly.over)
        for (double x : f.rf) w.f64(x);
    w.i32(kTrailer);
    if (f.has_ext) {
        w.i32(kExtMagic);
        w.i32(kExtVersion);
        w.i32(f.ext_slots);
        w.i32(f.W);
        for (const auto& e : f.ext) {
            w.i64(e.nflip);
            w.i32(e.bits);
            w.i32(0);
            for (int64_t c : e.counts) w.i64(c);
            for (double s : e.sums) w.f64(s);
            for (int s = 0; s < f.ext_slots; ++s) { w.i64(e.tag[s]); w.i64(e.data[s]); }
        }
    }
}

bool read_file(const std::string& path, std::vector<uint8_t>* bytes) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    bytes->clear();
    uint8_t buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), fp)) > 0) bytes->insert(bytes->end(), buf, buf + k);
    const bool ok = !std::ferror(fp);
    std::fclose(fp);
    return ok;
}

bool write_file(const std::string& path, const std::vector<uint8_t>& bytes) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), fp) == bytes.size();
    return std::fclose(fp) == 0 && ok;
}

std::string file_name(const char* base, int rank, int trial) {
    char tail[32];
    std::snprintf(tail, sizeof(tail), "_%05d_%05d.restart", rank, trial);
    return std::string(base) + tail;
}

// ---------------------------------------------------------------- host RNG
// Philox4x32-10 (Salmon et al., SC'11), the device streams' generator.
void philox_host(uint64_t a, uint32_t g, uint32_t tag, uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c0 = (uint32_t)a, c1 = (uint32_t)(a >> 32), c2 = g, c3 = tag;
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Pending flip step of a barrier in state `st` observed at step s: s + W, W
// geometric with the state's per-step flip probability (1 - e^{ln1m}).
int64_t draw_flip(const KConst& k, uint64_t s, int st, uint32_t hi, uint32_t lo) {
    const double ln1m = k.ln1m[st];
    if (!(ln1m < 0.0)) return kNever;
    const double u = ((double)(((uint64_t)hi << 32) | lo) + 1.0) * 0x1p-64;
    const double q = std::log(u) / ln1m;
    if (!(q < 0x1p61)) return kNever;
    const uint64_t wt = 1ull + (uint64_t)std::floor(q);
    return (wt >= (uint64_t)kNever - s) ? kNever : (int64_t)(s + wt);
}

// The device's state of a never-visited cell (default_state in ldp_fp64.cu,
// BarrierStatus::Initialize S.h:78-96).
int default_state_host(const KConst& k, uint32_t g, int64_t ck) {
    uint32_t w[4];
    if (k.us) {
        if (k.dbl) return k.init_state;
        const int64_t trial = ((int64_t)g / k.lanes) % k.nruns;
        if (trial == 0) return 0;
        if (!k.rs) return k.init_state;
        philox_host(0, g - (uint32_t)k.lanes, kTagInit, k.key0, k.key1, w);
        return ((double)w[0] * 0x1p-32 <= k.p_first) ? 0 : 1;
    }
    philox_host((uint64_t)ck, g, kTagCell, k.key0, k.key1, w);
    return ((double)w[0] * 0x1p-32 < k.p_cell0) ? 0 : 1;
}

// Energy and barrier height at x (EnergyAndForce, S.h:1292-1324 /
// D.h:1464-1522), as the device evaluates them.
void energy_host(const KConst& k, double x, int64_t cell, int s, double* E, double* B) {
    const double xp = x - (double)cell * k.L;
    if (!k.dbl) {
        const double sp = k.slope[s], sn = 0.0 - sp, H = k.Hs[s];
        double e = 0.0;
        if ((xp < 0.0) && (xp > -k.w)) e = H - xp * sn;
        if ((xp < k.w) && (xp > 0.0)) e = H - xp * sp;
        *E = e;
        *B = H;
    } else {
        double e = 0.0, b = 0.0;
        if ((xp < k.xb[0]) && (xp > k.lo0)) { e = xp * k.sN[0][s] + k.iN[0][s]; b = k.Hd[0][s]; }
        if ((xp < k.xc) && (xp > k.xb[0])) { e = xp * k.sP[0][s] + k.iP[0][s]; b = k.Hd[0][s]; }
        if ((xp < k.xb[1]) && (xp > k.xc)) { e = xp * k.sN[1][s] + k.iN[1][s]; b = k.Hd[1][s]; }
        if ((xp < k.hi1) && (xp > k.xb[1])) { e = xp * k.sP[1][s] + k.iP[1][s]; b = k.Hd[1][s]; }
        *E = e;
        *B = b;
    }
}

// Barrier parameters of state s in the file's order (UpdateBarrierStateEta-
// Paramter, S.h:2154-2165 / D.h:2737-2757).
std::vector<double> bparams_of(const KConst& k, int s) {
    if (!k.dbl) return {k.slope[s], 0.0 - k.slope[s], k.Hs[s]};
    return {k.sP[0][s], k.sP[1][s], k.sN[0][s], k.sN[1][s], k.iP[0][s], k.iP[1][s],
            k.iN[0][s], k.iN[1][s], k.Hd[0][s], k.Hd[1][s]};
}

// Header of a file for these parameters (the values LangevinEquationRunner
// hands its engine, S.h:3249-3301): q 0.2, eta0 0 and randomize-eta true
// are fixed by the two mains (src/langevinDynamicsSingleBarrier.cpp:136-147,
// src/langevinDynamicsDoubleBarrier.cpp:144-160); no .inp key changes them.
void fill_header(const ldp_job& job, int rank, uint64_t nsteps, File* f) {
    const ldp_params& p = job.p;
    f->sig = kSignature;
    f->W = job.o.lanes;
    f->x0 = p.x0; f->v0 = p.v0; f->gamma = p.gamma; f->kb = p.kb; f->T = p.temperature; f->m = p.mass;
    f->dt = p.timestep;
    f->nsteps = nsteps;
    f->wt = p.waiting_time ? 1 : 0;
    f->freq_stat = p.freq_stat;
    f->freq_save = p.freq_save;
    f->save_x = 1;
    f->save_v = f->save_f = f->save_e = p.write_x ? 1 : 0;
    if (p.overdamped) f->save_v = 0;   // OverdampedLangevinEquation: m_SaveV = false (S.h:2823)
    f->rand_v = p.randomize_v ? 1 : 0;
    f->rand_eta = 1;
    f->L = p.periodic_length;
    if (p.model == LDP_MODEL_DOUBLE) {
        f->H[0] = p.barrier_heights[0][0]; f->H[1] = p.barrier_heights[0][1];
        f->H[2] = p.barrier_heights[1][0]; f->H[3] = p.barrier_heights[1][1];
        f->pos[0] = p.barrier_position[0]; f->pos[1] = p.barrier_position[1];
        f->xc = job.k.xc;
    } else {
        f->H[0] = p.barrier_heights[0][0]; f->H[1] = p.barrier_heights[0][1];
    }
    f->init_state = (double)p.initial_state;
    f->rand_state = p.randomize_states ? 1 : 0;
    f->same_init = p.uniform_initial_states ? 1 : 0;
    f->q = 0.2; f->tau = p.tau; f->eta0 = 0.0;
    f->save_eta = 0;
    f->save_state = f->save_barrier = p.write_x ? 1 : 0;
    f->rank = rank;
    for (int i = 0; i < 3; ++i) { f->renew[i] = 0; f->progress[i] = 0; }
    f->lane_wt = p.waiting_time ? 1 : 0;
    f->lane_fpt = p.fpt ? 1 : 0;
}

// The checks of ReadRestartFile (S.h:1137-1193 / D.h:1296-1358): a file
// must come from a run with the same parameters.
bool check_header(const ldp_job& job, int rank, const File& f, std::string* err) {
    File h;
    fill_header(job, rank, 0, &h);
    const bool dbl = job.p.model == LDP_MODEL_DOUBLE;
    auto bad = [&](const char* what) { *err = std::string("inconsistent ") + what; return false; };
    if (f.W != job.o.lanes) return bad("simd witdth (the file's lanes differ from the job's lanes)");
    if (f.x0 != h.x0) return bad("x0");
    if (f.v0 != h.v0) return bad("v0");
    if (f.gamma != h.gamma) return bad("gamma0");
    if (f.kb != h.kb) return bad("kb0");
    if (f.T != h.T) return bad("T0");
    if (f.m != h.m) return bad("m0");
    if (f.dt != h.dt) return bad("time step0");
    if (f.wt != h.wt) return bad("bWaitingTimeDistribution");
    if (f.freq_stat != h.freq_stat) return bad("statisticsFreq");
    if (f.freq_save != h.freq_save) return bad("save freq");
    if (f.save_x != h.save_x) return bad("bSaveX");
    if (f.save_f != h.save_f) return bad("bSaveF");
    if (f.save_e != h.save_e) return bad("bSaveE");
    if (f.rand_v != h.rand_v) return bad("randomize velocity");
    if (f.rand_eta != h.rand_eta) return bad("randomize eta");
    if (f.L != h.L) return bad("periodic length0");
    for (int i = 0; i < (dbl ? 4 : 2); ++i)
        if (f.H[i] != h.H[i]) return bad("barrier height0");
    if (f.init_state != h.init_state) return bad("initialState0");
    if (dbl && (f.pos[0] != h.pos[0] || f.pos[1] != h.pos[1])) return bad("barrier position0");
    if (f.rand_state != h.rand_state) return bad("randomizeState0");
    if (f.same_init != h.same_init) return bad("bSameInitialBarrier");
    if (f.q != h.q) return bad("q0");
    if (f.tau != h.tau) return bad("tau0");
    if (f.eta0 != h.eta0) return bad("eta0");
    if (f.save_eta != h.save_eta) return bad("bSaveEta");
    if (f.save_state != h.save_state) return bad("bSaveState");
    if (f.save_barrier != h.save_barrier) return bad("save barrier");
    if (f.rank != rank) return bad("rank");
    if (f.lane_fpt != h.lane_fpt) return bad("bFirstPassageTime");
    return true;
}

double list_sum(const std::vector<double>& v) {
    double s = 0.0;
    for (double x : v) s += x;   // event order, as the device accumulates
    return s;
}

// Counts and sums a job holds for a lane read from a reference-written file
// (no exact-resume block).
void reduce_lane(const Lane& a, uint64_t steps, int n_cg, int64_t* cnt, double* sum) {
    std::fill(cnt, cnt + LDP_NCOUNT, 0);
    std::fill(sum, sum + LDP_NSUM, 0.0);
    cnt[LDP_C_FPT] = (int64_t)a.fpt.size();
    cnt[LDP_C_FPT2] = (int64_t)a.fpt2.size();
    cnt[LDP_C_TPT] = (int64_t)a.tpt.size();
    cnt[LDP_C_TPT2] = (int64_t)a.tpt2.size();
    for (double s : a.initial) cnt[s != 0.0 ? LDP_C_INIT1 : LDP_C_INIT0]++;
    for (double s : a.instant) cnt[s != 0.0 ? LDP_C_INST1 : LDP_C_INST0]++;
    cnt[LDP_C_STATE0] = (int64_t)a.sc[0];
    cnt[LDP_C_STATE1] = (int64_t)a.sc[1];
    cnt[LDP_C_WT] = (int64_t)a.ticks.size();
    cnt[LDP_C_STEPS] = (int64_t)steps;
    sum[LDP_S_FPT] = list_sum(a.fpt);
    sum[LDP_S_FPT2] = list_sum(a.fpt2);
    sum[LDP_S_TPT] = list_sum(a.tpt);
    sum[LDP_S_TPT2] = list_sum(a.tpt2);
    sum[LDP_S_FIRST_FPT] = a.fpt.empty() ? 0.0 : a.fpt[0];
    sum[LDP_S_FIRST_FPT2] = a.fpt2.empty() ? 0.0 : a.fpt2[0];
    sum[LDP_S_FIRST_TPT] = a.tpt.empty() ? 0.0 : a.tpt[0];
    sum[LDP_S_FIRST_TPT2] = a.tpt2.empty() ? 0.0 : a.tpt2[0];
    for (int j = 0; j < n_cg && j < (int)a.cg.size(); ++j) {
        cnt[LDP_C_CG0 + j] = (int64_t)a.cg[j].list.size();
        sum[LDP_S_CG0 + j] = list_sum(a.cg[j].list);
    }
}

bool decode_path(const ldp_params& p, const std::string& path, File* f, std::string* err) {
    std::vector<uint8_t> bytes;
    if (!read_file(path, &bytes)) { *err = "can't open restart file (" + path + ")"; return false; }
    if (!decode(bytes, layout_of(p), f, err)) { *err += " (" + path + ")"; return false; }
    return true;
}

// Host copies of a job's per-trajectory device state.
struct HostState {
    int64_t n = 0;
    std::vector<double> x, v, F, rprev, fpt_last, fpt2_last, tpt_last, tpt2_last, v0;
    std::vector<int64_t> cell, well, init_idx0, init_idx1, idx2_0, idx2_1, tpt2_well, wt_tick, nflip;
    std::vector<int32_t> state, lb, bits, state0;
    std::vector<double> cg_last;
    std::vector<int64_t> cg_well, counts;
    std::vector<double> sums;
    std::vector<int64_t> ring_tag, ring_data, ticks;
    std::vector<double> frames[7];   // fx fv ff fb fpe fke fst
    std::vector<double> ev;
    std::vector<uint8_t> ev_st;
};

void host_alloc(const ldp_job& job, HostState* h) {
    const int64_t n = job.ntraj;
    const int ncg = std::max(1, job.p.n_cg);
    h->n = n;
    for (auto* d : {&h->x, &h->v, &h->F, &h->rprev, &h->fpt_last, &h->fpt2_last, &h->tpt_last, &h->tpt2_last, &h->v0})
        d->assign(n, 0.0);
    for (auto* d : {&h->cell, &h->well, &h->init_idx0, &h->init_idx1, &h->idx2_0, &h->idx2_1, &h->tpt2_well,
                    &h->wt_tick, &h->nflip})
        d->assign(n, 0);
    for (auto* d : {&h->state, &h->lb, &h->bits, &h->state0}) d->assign(n, 0);
    h->cg_last.assign((size_t)ncg * n, 0.0);
    h->cg_well.assign((size_t)ncg * n, 0);
    h->counts.assign((size_t)LDP_NCOUNT * n, 0);
    h->sums.assign((size_t)LDP_NSUM * n, 0.0);
    h->ring_tag.assign((size_t)job.o.table_slots * n, INT64_MIN);
    h->ring_data.assign((size_t)job.o.table_slots * n, 0);
    h->ticks.assign((size_t)std::max<int64_t>(job.o.tick_cap, 1) * n, 0);
    const TrajState& S = job.st;
    const double* fr[7] = {S.fx, S.fv, S.ff, S.fb, S.fpe, S.fke, S.fst};
    for (int s = 0; s < 7; ++s) h->frames[s].assign(fr[s] ? (size_t)job.nframe * n : 0, 0.0);
    const size_t ev_elems = (size_t)std::max<int64_t>(job.o.event_cap, 0) * n;
    h->ev.assign((size_t)(LDP_E_CG0 + job.p.n_cg) * ev_elems, 0.0);
    h->ev_st.assign(ev_elems, 0);
}

// Copies between the host state and the job's device arrays, ordered on
// the context's stream (after the arena's allocation and clearing).
cudaError_t transfer(const ldp_job& job, HostState* h, bool to_device) {
    const TrajState& S = job.st;
    const int64_t n = job.ntraj;
    const int ncg = std::max(1, job.p.n_cg);
    cudaStream_t stream = job.ctx->stream;
    cudaError_t e = cudaSuccess;
    auto mv = [&](void* dev, void* host, size_t bytes) {
        if (e != cudaSuccess || !dev || !bytes) return;
        e = to_device ? cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, stream)
                      : cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, stream);
    };
    const size_t d8 = sizeof(double) * n, i8 = sizeof(int64_t) * n, i4 = sizeof(int32_t) * n;
    mv(S.x, h->x.data(), d8); mv(S.v, h->v.data(), d8); mv(S.F, h->F.data(), d8); mv(S.rprev, h->rprev.data(), d8);
    mv(S.fpt_last, h->fpt_last.data(), d8); mv(S.fpt2_last, h->fpt2_last.data(), d8);
    mv(S.tpt_last, h->tpt_last.data(), d8); mv(S.tpt2_last, h->tpt2_last.data(), d8); mv(S.v0, h->v0.data(), d8);
    mv(S.cell, h->cell.data(), i8); mv(S.well, h->well.data(), i8);
    mv(S.init_idx0, h->init_idx0.data(), i8); mv(S.init_idx1, h->init_idx1.data(), i8);
    mv(S.idx2_0, h->idx2_0.data(), i8); mv(S.idx2_1, h->idx2_1.data(), i8);
    mv(S.tpt2_well, h->tpt2_well.data(), i8); mv(S.wt_tick, h->wt_tick.data(), i8); mv(S.nflip, h->nflip.data(), i8);
    mv(S.state, h->state.data(), i4); mv(S.lb, h->lb.data(), i4); mv(S.bits, h->bits.data(), i4);
    mv(S.state0, h->state0.data(), i4);
    mv(S.cg_last, h->cg_last.data(), sizeof(double) * ncg * n);
    mv(S.cg_well, h->cg_well.data(), sizeof(int64_t) * ncg * n);
    mv(S.counts, h->counts.data(), sizeof(int64_t) * LDP_NCOUNT * n);
    mv(S.sums, h->sums.data(), sizeof(double) * LDP_NSUM * n);
    mv(S.ring_tag, h->ring_tag.data(), sizeof(int64_t) * h->ring_tag.size());
    mv(S.ring_data, h->ring_data.data(), sizeof(int64_t) * h->ring_data.size());
    if (job.o.tick_cap > 0) mv(S.ticks, h->ticks.data(), sizeof(int64_t) * h->ticks.size());
    double* fr[7] = {S.fx, S.fv, S.ff, S.fb, S.fpe, S.fke, S.fst};
    for (int s = 0; s < 7; ++s) mv(fr[s], h->frames[s].data(), sizeof(double) * h->frames[s].size());
    if (!h->ev.empty()) {
        mv(S.ev, h->ev.data(), sizeof(double) * h->ev.size());
        mv(S.ev_st, h->ev_st.data(), h->ev_st.size());
    }
    const cudaError_t es = cudaStreamSynchronize(stream);
    return e != cudaSuccess ? e : es;
}

// Frame series of the file (index in Lane::series) for each device frame
// array fx fv ff fb fpe fke fst (Record, S.h:1707-1765).
constexpr int kSeriesOf[7] = {0, 1, 2, 7, 3, 4, 6};

}  // namespace
}  // namespace ldp

using namespace ldp;

// ---------------------------------------------------------------- restore
extern "C" ldp_status ldp_job_restore(ldp_job* job, const char* base) {
    if (!job || !base) return LDP_ERR_INVALID;
    ldp_ctx* ctx = job->ctx;
    if (job->submitted || job->restored) {
        ldp_set_error(ctx, "restore must precede the job's submission (and happen once)");
        return LDP_ERR_INVALID;
    }
    if (job->o.precision != LDP_PREC_FP64_PLAIN || job->o.mode != LDP_MODE_FIXED_STEPS) {
        ldp_set_error(ctx, "restart files need the FP64 plain path in fixed-step mode");
        return LDP_ERR_UNSUPPORTED;
    }
    const ldp_params& p = job->p;
    const int lanes = job->o.lanes, runs = p.number_of_runs, ranks = job->o.ranks;
    std::vector<File> files((size_t)ranks * runs);
    std::string err;
    uint64_t S0 = 0;
    size_t need_ev = 0, need_ticks = 0;
    for (int r = 0; r < ranks; ++r)
        for (int t = 0; t < runs; ++t) {
            File& f = files[(size_t)r * runs + t];
            const int rg = job->o.first_rank + r;   // the rank in the run
            const std::string path = file_name(base, rg, t);
            if (!decode_path(p, path, &f, &err) || !check_header(*job, rg, f, &err)) {
                if (err.find(path) == std::string::npos) err += " (" + path + ")";
                ldp_set_error(ctx, "%s", err.c_str());
                return LDP_ERR_RESTART;
            }
            if (r == 0 && t == 0) S0 = f.nsteps;
            if (f.nsteps != S0) {
                ldp_set_error(ctx, "restart files of one job hold different step counts (%s)", path.c_str());
                return LDP_ERR_RESTART;
            }
            if (f.has_ext && f.ext_slots != job->o.table_slots) {
                ldp_set_error(ctx, "restart file written with table_slots %d, job has %d (%s)", f.ext_slots,
                              job->o.table_slots, path.c_str());
                return LDP_ERR_RESTART;
            }
            for (const Lane& a : f.lanes) {
                // Values that become integers on the device must be finite
                // and in range (a damaged file must not reach the casts).
                const double idx_max = 0x1p52;
                const double ints[] = {a.cell, a.well, a.lb, a.wt_prev, a.state, a.state0, a.sc[0], a.sc[1]};
                bool ok = std::isfinite(a.x) && std::isfinite(a.v);
                for (double d : ints) ok = ok && std::isfinite(d) && std::fabs(d) < idx_max;
                if (!ok) {
                    ldp_set_error(ctx, "restart file corrupted: non-finite or out-of-range lane state (%s)",
                                  path.c_str());
                    return LDP_ERR_RESTART;
                }
                need_ev = std::max({need_ev, a.fpt.size(), a.fpt2.size(), a.tpt.size(), a.tpt2.size()});
                for (const auto& c : a.cg) need_ev = std::max(need_ev, c.list.size());
                need_ticks = std::max(need_ticks, a.ticks.size());
                const size_t nfr = (size_t)(S0 / p.freq_save) + 1;
                if (a.series[0].size() != nfr) {
                    ldp_set_error(ctx, "restart file holds %zu frames, %llu steps at FREQSAVE %llu make %zu (%s)",
                                  a.series[0].size(), (unsigned long long)S0, (unsigned long long)p.freq_save, nfr,
                                  path.c_str());
                    return LDP_ERR_RESTART;
                }
            }
        }
    if (p.number_of_previous_steps != S0) {
        ldp_set_error(ctx, "NUMBEROFPREVIOUSSTEPS %llu differs from the %llu steps the restart files hold",
                      (unsigned long long)p.number_of_previous_steps, (unsigned long long)S0);
        return LDP_ERR_RESTART;
    }
    if (S0 % p.freq_save != 0) {
        ldp_set_error(ctx, "restart step count %llu is not a multiple of FREQSAVE", (unsigned long long)S0);
        return LDP_ERR_RESTART;
    }
    // Lists carried on: the device lists continue the file's lists.
    if (job->o.event_cap > 0 && (size_t)job->o.event_cap < need_ev) {
        if (!job->ev_auto) {
            ldp_set_error(ctx, "event_cap %lld < %zu events already in the restart files",
                          (long long)job->o.event_cap, need_ev);
            return LDP_ERR_INVALID;
        }
        job->o.event_cap += (int64_t)need_ev;
    }
    if (job->o.tick_cap > 0 && (size_t)job->o.tick_cap < need_ticks) {
        if (!job->tick_auto) {
            ldp_set_error(ctx, "tick_cap %lld < %zu waiting ticks already in the restart files",
                          (long long)job->o.tick_cap, need_ticks);
            return LDP_ERR_INVALID;
        }
        job->o.tick_cap = (int64_t)need_ticks + job->o.tick_cap;
    }
    job->k.ev_cap = job->o.event_cap;
    job->k.tick_cap = job->o.tick_cap;
    cudaSetDevice(ctx->device);
    if (!job->arena && ldp_job_arena(job, true) == 0) {
        ldp_set_error(ctx, "cudaMalloc of %zu bytes failed", ldp_job_arena(job, false));
        return LDP_ERR_NOMEM;
    }
    HostState h;
    host_alloc(*job, &h);
    const KConst& k = job->k;
    const int64_t n = job->ntraj;
    const int slots = job->o.table_slots;
    const int ncg = p.n_cg;
    const int64_t ecap = job->o.event_cap, tcap = job->o.tick_cap;
    for (int r = 0; r < ranks; ++r)
        for (int t = 0; t < runs; ++t) {
            const File& f = files[(size_t)r * runs + t];
            for (int l = 0; l < lanes; ++l) {
                const int64_t i = ((int64_t)r * runs + t) * lanes + l;
                const uint32_t g = (uint32_t)i + k.g0;
                const Lane& a = f.lanes[l];
                h.x[i] = a.x; h.v[i] = a.v; h.F[i] = a.f;
                h.rprev[i] = p.overdamped ? f.rf[l] : 0.0;
                h.cell[i] = (int64_t)a.cell; h.well[i] = (int64_t)a.well;
                h.lb[i] = k.dbl ? (int32_t)a.lb : 0;
                h.state[i] = a.state != 0.0 ? 1 : 0;
                h.state0[i] = a.state0 != 0.0 ? 1 : 0;
                h.v0[i] = a.v0;
                h.fpt_last[i] = a.fpt_last; h.fpt2_last[i] = a.fpt2_last;
                h.tpt_last[i] = a.tpt_last; h.tpt2_last[i] = a.tpt2_last;
                h.init_idx0[i] = a.init_idx[0]; h.init_idx1[i] = a.init_idx[1];
                h.idx2_0[i] = a.idx2[0]; h.idx2_1[i] = a.idx2[1];
                h.tpt2_well[i] = a.tpt2_well;
                h.wt_tick[i] = (int64_t)a.wt_prev;
                for (int j = 0; j < ncg && j < (int)a.cg.size(); ++j) {
                    h.cg_last[(size_t)j * n + i] = a.cg[j].last;
                    h.cg_well[(size_t)j * n + i] = a.cg[j].well;
                }
                // frames (the file's x series and WRITEX series)
                for (int s = 0; s < 7; ++s) {
                    if (h.frames[s].empty()) continue;
                    const std::vector<double>& src = a.series[kSeriesOf[s]];
                    for (size_t fi = 0; fi < src.size() && fi < (size_t)job->nframe; ++fi)
                        h.frames[s][fi * n + i] = src[fi];
                }
                // The overdamped engine keeps no velocity series (S.h:2822);
                // its velocity never changes, so the frames hold a.v.
                if (p.overdamped && !h.frames[1].empty() && a.series[1].empty())
                    for (size_t fi = 0; fi < a.series[0].size() && fi < (size_t)job->nframe; ++fi)
                        h.frames[1][fi * n + i] = a.v;
                for (size_t c = 0; c < a.ticks.size() && (int64_t)c < tcap; ++c)
                    h.ticks[(size_t)i * tcap + c] = (int64_t)a.ticks[c];
                if (ecap > 0) {
                    const std::vector<double>* lists[4] = {&a.fpt, &a.fpt2, &a.tpt, &a.tpt2};
                    for (int L = 0; L < LDP_E_CG0 + ncg; ++L) {
                        const std::vector<double>& src =
                            L < LDP_E_CG0 ? *lists[L] : a.cg[(size_t)(L - LDP_E_CG0)].list;
                        for (size_t c = 0; c < src.size(); ++c) h.ev[((size_t)L * n + i) * ecap + c] = src[c];
                    }
                    for (size_t c = 0; c < a.fpt.size(); ++c)
                        h.ev_st[(size_t)i * ecap + c] = (uint8_t)((c < a.instant.size() && a.instant[c] != 0.0 ? 1 : 0) |
                                                                  (c < a.initial.size() && a.initial[c] != 0.0 ? 2 : 0));
                }
                int64_t* cnt = &h.counts[0];
                double* sum = &h.sums[0];
                if (f.has_ext) {
                    const LaneExt& e = f.ext[l];
                    h.nflip[i] = e.nflip;
                    h.bits[i] = e.bits;
                    for (int c = 0; c < LDP_NCOUNT; ++c) cnt[(size_t)c * n + i] = e.counts[c];
                    for (int c = 0; c < LDP_NSUM; ++c) sum[(size_t)c * n + i] = e.sums[c];
                    for (int s = 0; s < slots; ++s) {
                        h.ring_tag[(size_t)s * n + i] = e.tag[s];
                        h.ring_data[(size_t)s * n + i] = e.data[s];
                    }
                    continue;
                }
                // A file the reference wrote.
                uint32_t bits = 0;
                if (a.fpt_up) bits |= B_FPT_UP;
                if (a.fpt2_up) bits |= B_FPT2_UP;
                if (a.tpt_up) bits |= B_TPT_UP;
                if (a.tpt2_up) bits |= B_TPT2_UP;
                if (a.wt_passed) bits |= B_WT_PASSED;
                if (a.init_state[0] != 0.0) bits |= B_INIT0;
                if (a.init_state[1] != 0.0) bits |= B_INIT1;
                for (int j = 0; j < ncg && j < (int)a.cg.size(); ++j)
                    if (a.cg[j].up) bits |= (B_CG0 << j);
                h.bits[i] = (int32_t)bits;
                int64_t lc[LDP_NCOUNT];
                double ls[LDP_NSUM];
                reduce_lane(a, S0, ncg, lc, ls);
                if ((int64_t)a.ticks.size() > tcap && k.wt) lc[LDP_C_FLAGS] |= LDP_FLAG_TICK_OVERFLOW;
                for (int c = 0; c < LDP_NCOUNT; ++c) cnt[(size_t)c * n + i] = lc[c];
                for (int c = 0; c < LDP_NSUM; ++c) sum[(size_t)c * n + i] = ls[c];
                uint32_t w[4];
                philox_host(S0, g, kTagResume, k.key0, k.key1, w);
                h.nflip[i] = draw_flip(k, S0, h.state[i], w[0], w[1]);
                // The barrier table: every cell of the file, nearest cells
                // last so that they keep their ring slots.
                struct Ent { int64_t key, dist; int st; uint64_t step; };
                std::vector<Ent> ents;
                for (int tb = 0; tb < (k.dbl ? 2 : 1); ++tb) {
                    const Table& T = f.tables[tb];
                    const size_t nc = T.ncell(f.W);
                    for (size_t c = 0; c < nc; ++c) {
                        const int64_t id = (int64_t)T.min_id + (int64_t)c;
                        const int64_t key = k.dbl ? id * 2 + tb : id;
                        ents.push_back({key, std::llabs(id - h.cell[i]), T.state[c * f.W + l] ? 1 : 0,
                                        T.step[c * f.W + l]});
                    }
                }
                std::stable_sort(ents.begin(), ents.end(), [](const Ent& x, const Ent& y) { return x.dist > y.dist; });
                for (const Ent& en : ents) {
                    philox_host((uint64_t)en.key, g, kTagResumeCell, k.key0, k.key1, w);
                    const int64_t nb = draw_flip(k, en.step, en.st, w[0], w[1]);
                    const size_t o = (size_t)(en.key & (int64_t)(slots - 1)) * n + i;
                    h.ring_tag[o] = en.key;
                    h.ring_data[o] = (nb << 1) | en.st;
                }
            }
        }
    const cudaError_t e = transfer(*job, &h, true);
    if (e != cudaSuccess) {
        ldp_set_error(ctx, "restart upload failed: %s", cudaGetErrorString(e));
        return LDP_ERR_DEVICE;
    }
    job->restored = true;
    job->steps_before = S0;
    return LDP_OK;
}

// ---------------------------------------------------------------- save
extern "C" ldp_status ldp_job_save_restart(ldp_job* job, const char* base) {
    if (!job || !base) return LDP_ERR_INVALID;
    ldp_ctx* ctx = job->ctx;
    if (job->o.precision != LDP_PREC_FP64_PLAIN || job->o.mode != LDP_MODE_FIXED_STEPS) {
        ldp_set_error(ctx, "restart files need the FP64 plain path in fixed-step mode");
        return LDP_ERR_UNSUPPORTED;
    }
    if (!job->done) {
        ldp_status st = ldp_wait(ctx, job);
        if (st != LDP_OK) return st;
    }
    const ldp_params& p = job->p;
    const int64_t n = job->ntraj;
    if (job->o.event_cap <= 0) {
        ldp_set_error(ctx, "restart files hold the per-event lists: create the job with event_cap > 0 "
                           "(or -1 with WRITERESTART true)");
        return LDP_ERR_INVALID;
    }
    cudaSetDevice(ctx->device);
    HostState h;
    host_alloc(*job, &h);
    const cudaError_t e = transfer(*job, &h, false);
    if (e != cudaSuccess) {
        ldp_set_error(ctx, "restart download failed: %s", cudaGetErrorString(e));
        return LDP_ERR_DEVICE;
    }
    for (int64_t i = 0; i < n; ++i) {
        const int64_t fl = h.counts[(size_t)LDP_C_FLAGS * n + i];
        if (fl & (LDP_FLAG_EVENT_OVERFLOW | LDP_FLAG_TICK_OVERFLOW)) {
            ldp_set_error(ctx, "trajectory %lld has more events than its lists hold (event_cap %lld, tick_cap %lld): "
                               "the restart file would be incomplete", (long long)i,
                          (long long)job->o.event_cap, (long long)job->o.tick_cap);
            return LDP_ERR_INVALID;
        }
    }
    const KConst& k = job->k;
    const int lanes = job->o.lanes, runs = p.number_of_runs, ranks = job->o.ranks;
    const uint64_t S = job->steps_before + job->nsteps;
    const int slots = job->o.table_slots;
    const int ncg = p.n_cg;
    const int64_t ecap = job->o.event_cap, tcap = job->o.tick_cap;
    const int64_t nfr = (int64_t)(S / p.freq_save) + 1;
    for (int r = 0; r < ranks; ++r)
        for (int t = 0; t < runs; ++t) {
            File f;
            fill_header(*job, job->o.first_rank + r, S, &f);
            f.lanes.assign(lanes, Lane());
            f.has_ext = true;
            f.ext_slots = slots;
            f.ext.assign(lanes, LaneExt());
            if (p.overdamped) f.rf.assign(lanes, 0.0);
            int64_t lo_id[2] = {INT64_MAX, INT64_MAX}, hi_id[2] = {INT64_MIN, INT64_MIN};
            for (int l = 0; l < lanes; ++l) {
                const int64_t i = ((int64_t)r * runs + t) * lanes + l;
                Lane& a = f.lanes[l];
                const int st = h.state[i];
                a.x = h.x[i]; a.v = h.v[i]; a.f = h.F[i];
                energy_host(k, a.x, h.cell[i], st, &a.e, &a.barrier);
                a.eta = 0.0;
                a.xp = a.x - (double)h.cell[i] * k.L;
                for (int s = 0; s < 7; ++s) {
                    // no velocity series for the overdamped engine
                    // (IntegrateInitializeVariables, S.h:2822)
                    if (h.frames[s].empty() || (s == 1 && p.overdamped)) continue;
                    std::vector<double>& dst = a.series[kSeriesOf[s]];
                    dst.resize((size_t)std::min<int64_t>(nfr, job->nframe));
                    for (size_t fi = 0; fi < dst.size(); ++fi) dst[fi] = h.frames[s][fi * n + i];
                }
                a.state = (double)st;
                a.prev_state = (double)st;
                a.bparams = bparams_of(k, st);
                a.sc[0] = (double)h.counts[(size_t)LDP_C_STATE0 * n + i];
                a.sc[1] = (double)h.counts[(size_t)LDP_C_STATE1 * n + i];
                a.well = a.well_prev = a.well_st = a.well_prev_st = (double)h.well[i];
                a.cell = a.cell_prev = a.cell_st = a.cell_prev_st = (double)h.cell[i];
                a.lb = a.lb_prev = a.lb_st = a.lb_prev_st = (double)h.lb[i];
                a.v0 = h.v0[i];
                a.eta0 = 0.0;
                a.state0 = (double)h.state0[i];
                const uint32_t bits = (uint32_t)h.bits[i];
                if (f.lane_wt) {
                    a.wt_prev = (double)h.wt_tick[i];
                    a.wt_passed = (bits & B_WT_PASSED) ? 1 : 0;
                    const int64_t nt = std::min<int64_t>(h.counts[(size_t)LDP_C_WT * n + i], std::max<int64_t>(tcap, 0));
                    a.ticks.resize((size_t)nt);
                    for (int64_t c = 0; c < nt; ++c) a.ticks[c] = (double)h.ticks[(size_t)i * tcap + c];
                }
                auto list = [&](int L, int cfield) {
                    const int64_t m = std::min<int64_t>(h.counts[(size_t)cfield * n + i], ecap);
                    std::vector<double> v((size_t)m);
                    for (int64_t c = 0; c < m; ++c) v[c] = h.ev[((size_t)L * n + i) * ecap + c];
                    return v;
                };
                if (f.lane_fpt) {
                    a.fpt = list(LDP_E_FPT, LDP_C_FPT);
                    a.instant.resize(a.fpt.size());
                    a.initial.resize(a.fpt.size());
                    for (size_t c = 0; c < a.fpt.size(); ++c) {
                        const uint8_t b = h.ev_st[(size_t)i * ecap + c];
                        a.instant[c] = (b & 1) ? 1.0 : 0.0;
                        a.initial[c] = (b & 2) ? 1.0 : 0.0;
                    }
                    a.fpt_last = h.fpt_last[i];
                    a.fpt_up = (bits & B_FPT_UP) ? 1 : 0;
                    a.init_state[0] = (bits & B_INIT0) ? 1.0 : 0.0;
                    a.init_state[1] = (bits & B_INIT1) ? 1.0 : 0.0;
                    a.init_idx[0] = (int32_t)h.init_idx0[i];
                    a.init_idx[1] = (int32_t)h.init_idx1[i];
                    a.fpt2 = list(LDP_E_FPT2, LDP_C_FPT2);
                    a.fpt2_last = h.fpt2_last[i];
                    a.fpt2_up = (bits & B_FPT2_UP) ? 1 : 0;
                    a.idx2[0] = (int32_t)h.idx2_0[i];
                    a.idx2[1] = (int32_t)h.idx2_1[i];
                }
                if (p.tpt) {
                    a.tpt = list(LDP_E_TPT, LDP_C_TPT);
                    a.tpt_last = h.tpt_last[i];
                    a.tpt_up = (bits & B_TPT_UP) ? 1 : 0;
                    a.tpt2 = list(LDP_E_TPT2, LDP_C_TPT2);
                    a.tpt2_last = h.tpt2_last[i];
                    a.tpt2_up = (bits & B_TPT2_UP) ? 1 : 0;
                    a.tpt2_well = (int32_t)h.tpt2_well[i];
                }
                if (p.fptcg) {
                    a.cg_sizes.assign(p.cg_sizes, p.cg_sizes + ncg);
                    a.cg.resize(ncg);
                    for (int j = 0; j < ncg; ++j) {
                        a.cg[j].list = list(LDP_E_CG0 + j, LDP_C_CG0 + j);
                        a.cg[j].last = h.cg_last[(size_t)j * n + i];
                        a.cg[j].up = (bits & (B_CG0 << j)) ? 1 : 0;
                        a.cg[j].well = (int32_t)h.cg_well[(size_t)j * n + i];
                    }
                }
                if (p.overdamped) f.rf[l] = h.rprev[i];
                LaneExt& x = f.ext[l];
                x.nflip = h.nflip[i];
                x.bits = (int32_t)bits;
                for (int c = 0; c < LDP_NCOUNT; ++c) x.counts[c] = h.counts[(size_t)c * n + i];
                for (int c = 0; c < LDP_NSUM; ++c) x.sums[c] = h.sums[(size_t)c * n + i];
                x.tag.resize(slots);
                x.data.resize(slots);
                for (int s = 0; s < slots; ++s) {
                    x.tag[s] = h.ring_tag[(size_t)s * n + i];
                    x.data[s] = h.ring_data[(size_t)s * n + i];
                    if (x.tag[s] == INT64_MIN) continue;
                    const int tb = k.dbl ? (int)(x.tag[s] & 1) : 0;
                    const int64_t id = k.dbl ? (x.tag[s] - tb) / 2 : x.tag[s];
                    lo_id[tb] = std::min(lo_id[tb], id);
                    hi_id[tb] = std::max(hi_id[tb], id);
                }
                // the current cell (and its neighbours, which the FPT
                // bookkeeping reads) belong to the table as well
                for (int tb = 0; tb < (k.dbl ? 2 : 1); ++tb) {
                    lo_id[tb] = std::min(lo_id[tb], h.cell[i] - 1);
                    hi_id[tb] = std::max(hi_id[tb], h.cell[i] + 1);
                }
            }
            for (int tb = 0; tb < (k.dbl ? 2 : 1); ++tb) {
                if (lo_id[tb] < INT32_MIN || hi_id[tb] > INT32_MAX) {
                    ldp_set_error(ctx, "cell indices beyond 32 bits cannot be written to a restart file");
                    return LDP_ERR_INVALID;
                }
                Table& T = f.tables[tb];
                T.min_id = (int32_t)lo_id[tb];
                const size_t nc = (size_t)(hi_id[tb] - lo_id[tb] + 1);
                T.state.assign(nc * lanes, 0);
                T.step.assign(nc * lanes, 0);
                for (int l = 0; l < lanes; ++l) {
                    const int64_t i = ((int64_t)r * runs + t) * lanes + l;
                    const uint32_t g = (uint32_t)i + k.g0;
                    for (size_t c = 0; c < nc; ++c) {
                        const int64_t id = lo_id[tb] + (int64_t)c;
                        const int64_t key = k.dbl ? id * 2 + tb : id;
                        const size_t o = (size_t)(key & (int64_t)(slots - 1)) * n + i;
                        int st;
                        uint64_t step;
                        if (key == (k.dbl ? h.cell[i] * 2 + h.lb[i] : h.cell[i])) {
                            st = h.state[i];       // the current barrier
                            step = S;
                        } else if (h.ring_tag[o] == key) {
                            const int ps = (int)(h.ring_data[o] & 1);
                            const int64_t nb = h.ring_data[o] >> 1;
                            if (nb > (int64_t)S) { st = ps; step = S; }
                            else { st = ps ^ 1; step = (uint64_t)nb; }
                        } else {
                            st = default_state_host(k, g, key);
                            step = 0;
                        }
                        T.state[c * lanes + l] = st;
                        T.step[c * lanes + l] = step;
                    }
                }
            }
            std::vector<uint8_t> bytes;
            encode(f, layout_of(p), &bytes);
            const std::string path = file_name(base, job->o.first_rank + r, t);
            if (!write_file(path, bytes)) {
                ldp_set_error(ctx, "can't open restart file (%s)", path.c_str());
                return LDP_ERR_IO;
            }
        }
    return LDP_OK;
}

// ---------------------------------------------------------------- files
extern "C" ldp_status ldp_restart_inspect(const ldp_params* p, const char* path, ldp_restart_summary* s,
                                          int64_t* counts, double* sums, char* err, size_t errlen) {
    if (!p || !path || !s) return LDP_ERR_INVALID;
    File f;
    std::string e;
    if (!decode_path(*p, path, &f, &e)) {
        if (err && errlen) std::snprintf(err, errlen, "%s", e.c_str());
        return LDP_ERR_RESTART;
    }
    std::memset(s, 0, sizeof(*s));
    s->lanes = f.W;
    s->rank = f.rank;
    s->steps = f.nsteps;
    s->has_exact_resume = f.has_ext ? 1 : 0;
    s->frames = f.lanes.empty() ? 0 : (int64_t)f.lanes[0].series[0].size();
    for (int t = 0; t < 2; ++t) {
        s->ncell[t] = (int64_t)f.tables[t].ncell(f.W);
        s->min_id[t] = f.tables[t].min_id;
    }
    const int64_t W = f.W;
    for (int l = 0; l < f.W; ++l) {
        int64_t lc[LDP_NCOUNT];
        double ls[LDP_NSUM];
        reduce_lane(f.lanes[l], f.nsteps, p->n_cg, lc, ls);
        if (f.has_ext) {
            std::copy(f.ext[l].counts, f.ext[l].counts + LDP_NCOUNT, lc);
            std::copy(f.ext[l].sums, f.ext[l].sums + LDP_NSUM, ls);
        }
        if (counts)
            for (int c = 0; c < LDP_NCOUNT; ++c) counts[c * W + l] = lc[c];
        if (sums)
            for (int c = 0; c < LDP_NSUM; ++c) sums[c * W + l] = ls[c];
    }
    return LDP_OK;
}

extern "C" ldp_status ldp_restart_rewrite(const ldp_params* p, const char* in, const char* out, char* err,
                                          size_t errlen) {
    if (!p || !in || !out) return LDP_ERR_INVALID;
    File f;
    std::string e;
    if (!decode_path(*p, in, &f, &e)) {
        if (err && errlen) std::snprintf(err, errlen, "%s", e.c_str());
        return LDP_ERR_RESTART;
    }
    std::vector<uint8_t> bytes;
    encode(f, layout_of(*p), &bytes);
    if (!write_file(out, bytes)) {
        if (err && errlen) std::snprintf(err, errlen, "can't open restart file (%s)", out);
        return LDP_ERR_IO;
    }
    return LDP_OK;
}
