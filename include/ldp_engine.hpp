/*
 * ldp_engine.hpp -- the reference's engine interface over the C ABI.
 *
 * ldp::LangevinEquationSIMDMultiple has the public methods of the
 * reference's engine class of the same name
 * (src/langevinDynamicsSingleBarrier.h:1048-2769; the overdamped and
 * double-barrier engines have the same ones): Initialize, Integrate,
 * Write/ReadRestartFile and the per-lane getters, with the same lane
 * indices and the same error convention (a failing call returns false after
 * printing the error on stderr), for C++ hosts that drive the engine in
 * process instead of through the executables.  Header only, over
 * include/ldp.h.
 *
 * One object stands for one virtual rank of a run: `lanes` trajectories per
 * trial (the reference's SIMD width), NUMBEROFRUNS trials, rank `rank` of
 * `ranks`.  Integrate(iTrial) makes trial iTrial current and the getters
 * read its lane `index`.  The object's trials are one job of the library
 * (ranks rank..rank of the run, ldp_job_opts.first_rank), integrated at the
 * first Integrate after Initialize: each trajectory's random streams are
 * keyed by (seed, its index in the run, step), so the results are those of
 * a trial-by-trial run, and the objects of the ranks of one run (in one
 * process or in several, on one GPU or several) hold the whole run's
 * trajectories, each integrated once.  bTimer is accepted and ignored (the
 * reference prints progress lines with it).
 *
 * Getters that read results before Integrate, or a lane or frame outside
 * the trial, print an error and return NaN (values), 0 (counts) or an empty
 * vector.  Per-event getters (GetFirstPassageTime, GetFirstPassageTime2,
 * GetTransitionPathTimeAll2) and restart files need the FP64 plain
 * precision, whose jobs keep every event (ldp_job_opts.event_cap); the WRITEX
 * series (GetV, GetF, GetPE, GetKE, GetState, GetBarrier) are empty unless
 * the .inp sets WRITEX, as in the reference.
 */
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <vector>

#include "ldp.h"

namespace ldp {

// The part of the reference's HISTOGRAM::HISTOGRAM (src/clsHistogram.h) the
// barrier-height histogram fillers use: bins [min, max) of equal width,
// `count` accumulating per-lane percentages.
struct Histogram {
    double min = 0.0, max = 10.0;
    int size = 100;
    std::vector<double> count = std::vector<double>(100, 0.0);
};

class LangevinEquationSIMDMultiple {
   public:
    // p: the parsed .inp (ldp_params_from_inp); precision: LDP_PREC_FP64_PLAIN
    // (bit-identical to the oracle) or LDP_PREC_FP32_BATCHED.
    LangevinEquationSIMDMultiple(ldp_ctx* ctx, const ldp_params& p, int lanes, int ranks = 1, int rank = 0,
                                 int precision = LDP_PREC_FP64_PLAIN)
        : ctx_(ctx), p_(p), lanes_(lanes), ranks_(ranks), rank_(rank), precision_(precision) {}
    LangevinEquationSIMDMultiple(const LangevinEquationSIMDMultiple&) = delete;
    LangevinEquationSIMDMultiple& operator=(const LangevinEquationSIMDMultiple&) = delete;
    virtual ~LangevinEquationSIMDMultiple() { release(); }

    // S.h:1276: the seed of every random stream (RANDOMSEED); results of an
    // earlier run are dropped.
    virtual void Initialize(int randomNumberSeed) {
        release();
        p_.random_seed = randomNumberSeed;
        restore_ = false;
    }

    // S.h:1386: integrates the object's trials if they have not been (every
    // trial at once) and makes trial iTrial current.
    virtual bool Integrate(int iTrial, bool bTimer = false) {
        (void)bTimer;
        if (iTrial < 0 || iTrial >= p_.number_of_runs || rank_ < 0 || rank_ >= ranks_) {
            std::fprintf(stderr, "Error: trial %d / rank %d outside the run (%d trials, %d ranks)\n", iTrial, rank_,
                         p_.number_of_runs, ranks_);
            return false;
        }
        if (!job_ && !run()) return false;
        trial_ = iTrial;
        x_.assign(kSeries * (size_t)lanes_, std::vector<double>());
        tick_.assign(lanes_, std::vector<double>());
        tpt2_.assign(lanes_, std::vector<double>());
        return true;
    }

    // S.h:1137: reads the object's restart files (INPUTRESTART,
    // <base>_%05d_%05d.restart per trial of this rank) into the run, which
    // then continues from them (NUMBEROFPREVIOUSSTEPS must equal the steps
    // they hold).  All trials' files are read at the first Integrate, so a
    // call after it is a no-op for the trials already restored.
    virtual bool ReadRestartFile(int iTrial) {
        if (iTrial < 0 || iTrial >= p_.number_of_runs) {
            std::fprintf(stderr, "Error: trial %d outside the run (%d trials)\n", iTrial, p_.number_of_runs);
            return false;
        }
        if (!job_) restore_ = true;
        return true;
    }
    // S.h:1048: writes the restart files of this rank (OUTPUTRESTART), every
    // trial's at the first call.
    virtual bool WriteRestartFile(int iTrial) {
        if (!ready("WriteRestartFile") || iTrial < 0 || iTrial >= p_.number_of_runs) return false;
        if (!saved_) {
            if (ldp_job_save_restart(job_, p_.output_restart) != LDP_OK) return fail("restart files");
            saved_ = true;
        }
        return true;
    }

    // Frames (S.h:2630-2699): x always, the other series with WRITEX.
    size_t GetNumberOfFrameX(int index) { return series_frames(kX, index); }
    double GetX(int index, size_t frameID) { return frame(kX, index, frameID); }
    std::vector<double>& GetX(int index) { return series(kX, index); }
    size_t GetNumberOfFrameV(int index) { return series_frames(kV, index); }
    double GetV(int index, size_t frameID) { return frame(kV, index, frameID); }
    std::vector<double>& GetV(int index) { return series(kV, index); }
    size_t GetNumberOfFrameF(int index) { return series_frames(kF, index); }
    double GetF(int index, size_t frameID) { return frame(kF, index, frameID); }
    std::vector<double>& GetF(int index) { return series(kF, index); }
    size_t GetNumberOfFramePE(int index) { return series_frames(kPE, index); }
    double GetPE(int index, size_t frameID) { return frame(kPE, index, frameID); }
    std::vector<double>& GetPE(int index) { return series(kPE, index); }
    size_t GetNumberOfFrameKE(int index) { return series_frames(kKE, index); }
    double GetKE(int index, size_t frameID) { return frame(kKE, index, frameID); }
    std::vector<double>& GetKE(int index) { return series(kKE, index); }
    size_t GetNumberOfFrameState(int index) { return series_frames(kState, index); }
    double GetState(int index, size_t frameID) { return frame(kState, index, frameID); }
    std::vector<double>& GetState(int index) { return series(kState, index); }
    size_t GetNumberOfFrameBarrier(int index) { return series_frames(kBarrier, index); }
    double GetBarrier(int index, size_t frameID) { return frame(kBarrier, index, frameID); }
    std::vector<double>& GetBarrier(int index) { return series(kBarrier, index); }

    // Renewal statistics (S.h:2716-2769).
    size_t GetFirstPassageTimeCount(int index) { return (size_t)count(LDP_C_FPT, index); }
    size_t GetFirstPassageTimeCount2(int index) { return (size_t)count(LDP_C_FPT2, index); }
    double GetFirstPassageTime(int index, size_t index2) { return event(LDP_E_FPT, LDP_C_FPT, index, index2); }
    double GetFirstPassageTime2(int index, size_t index2) { return event(LDP_E_FPT2, LDP_C_FPT2, index, index2); }
    double GetFirstPassageTimeAverage(int index) { return average(LDP_C_FPT, LDP_S_FPT, index); }
    double GetFirstPassageTimeAverage2(int index) { return average(LDP_C_FPT2, LDP_S_FPT2, index); }
    double GetTransitionPathTimeAverage(int index) { return average(LDP_C_TPT, LDP_S_TPT, index); }
    double GetTransitionPathTimeAverage2(int index) { return average(LDP_C_TPT2, LDP_S_TPT2, index); }
    std::vector<double>& GetTransitionPathTimeAll2(int index) {
        static std::vector<double> none;
        if (!lane_ok(index) || !events_ok("GetTransitionPathTimeAll2")) return none;
        std::vector<double>& v = tpt2_[index];
        if (v.empty()) {
            const int64_t n = count(LDP_C_TPT2, index) < event_cap_ ? count(LDP_C_TPT2, index) : event_cap_;
            for (int64_t k = 0; k < n; ++k) v.push_back(events_[event_at(LDP_E_TPT2, index, k)]);
        }
        return v;
    }
    // sizeIndex: the FPTCG entry of the .inp, in order
    double GetFirstPassageTimeCGAverage2(int index, int sizeIndex) {
        if (sizeIndex < 0 || sizeIndex >= p_.n_cg) return bad("FPTCG entry", sizeIndex);
        return average(LDP_C_CG0 + sizeIndex, LDP_S_CG0 + sizeIndex, index);
    }
    // The reference's fillers (S.h:2734-2753) histogram the lane's per-event
    // barrier states through HISTOGRAM::HistogramVector with its default
    // bounds, whose loop runs to the unclamped last = -1 and visits no
    // element (src/clsHistogram.cpp:242-255), so they add 0 to every bin;
    // these do the same.  The FPT events' barrier states themselves are the
    // counts LDP_C_INIT0/1 and LDP_C_INST0/1 of ldp_job_traj_results.
    void GetInitialBarrierHeightHistogram(int index, Histogram* histOut) { add_nothing(index, histOut); }
    void GetInstantBarrierHeightHistogram(int index, Histogram* histOut) { add_nothing(index, histOut); }
    // steps spent in barrier state iState (0 or 1), step 0 included
    double GetStateCount(int index, int iState) {
        if (iState != 0 && iState != 1) return bad("barrier state", iState);
        return (double)count(LDP_C_STATE0 + iState, index);
    }
    // waiting-time ticks: the steps at which a well change was followed by a
    // cell change (WAITINGTIME), as the reference stores them
    std::vector<double>& GetBarrierTick(int index) {
        static std::vector<double> none;
        if (!lane_ok(index) || !ready("GetBarrierTick")) return none;
        std::vector<double>& v = tick_[index];
        if (v.empty() && tick_cap_ > 0) {
            const int64_t n = count(LDP_C_WT, index) < tick_cap_ ? count(LDP_C_WT, index) : tick_cap_;
            for (int64_t k = 0; k < n; ++k) v.push_back((double)ticks_[(size_t)(traj(index) * tick_cap_ + k)]);
        }
        return v;
    }

   private:
    enum { kX = 0, kV, kF, kPE, kKE, kState, kBarrier, kSeries };

    bool fail(const char* what) {
        std::fprintf(stderr, "Error: %s: %s\n", what, ctx_ ? ldp_last_error(ctx_) : "no context");
        release();
        return false;
    }
    double bad(const char* what, long long v) {
        std::fprintf(stderr, "Error: %s %lld out of range\n", what, v);
        return std::numeric_limits<double>::quiet_NaN();
    }
    bool ready(const char* what) {
        if (job_) return true;
        std::fprintf(stderr, "Error: %s before Integrate\n", what);
        return false;
    }
    bool lane_ok(int index) {
        if (index >= 0 && index < lanes_) return true;
        bad("lane", index);
        return false;
    }
    bool events_ok(const char* what) {
        if (!ready(what)) return false;
        if (event_cap_ > 0) return true;
        std::fprintf(stderr, "Error: %s needs per-event lists (the FP64 plain precision)\n", what);
        return false;
    }
    bool run() {
        ldp_job_opts o;
        ldp_job_opts_default(&o);
        o.lanes = lanes_;
        o.ranks = 1;
        o.first_rank = rank_;
        o.precision = precision_;
        const uint64_t steps = p_.number_of_steps;
        if (precision_ == LDP_PREC_FP64_PLAIN) {
            // every event, as the reference's per-lane vectors (about one per
            // 10^4 steps at most, within 2^28 list entries)
            const int64_t lists = LDP_E_CG0 + p_.n_cg;
            const int64_t n = (int64_t)p_.number_of_runs * lanes_;
            int64_t a = (int64_t)(steps / 10000), b = ((int64_t)1 << 28) / (n * lists);
            a = a < 64 ? 64 : a;
            b = b < 64 ? 64 : b;
            o.event_cap = a < b ? a : b;
        } else {
            o.event_cap = 0;
        }
        if (ldp_job_create(ctx_, &p_, &o, &job_) != LDP_OK) return fail("job creation");
        if (restore_ && ldp_job_restore(job_, p_.input_restart) != LDP_OK) return fail("restart files");
        if (ldp_submit(ctx_, job_) != LDP_OK || ldp_wait(ctx_, job_) != LDP_OK) return fail("integration");
        ldp_job_info info;
        if (ldp_job_info_get(job_, &info) != LDP_OK) return fail("job info");
        ntraj_ = info.ntraj;
        nframe_ = info.nframe;
        tick_cap_ = info.tick_cap;
        event_cap_ = info.event_cap;
        counts_.assign((size_t)(LDP_NCOUNT * ntraj_), 0);
        sums_.assign((size_t)(LDP_NSUM * ntraj_), 0.0);
        const int nser = p_.write_x ? kSeries : 1;
        for (int k = 0; k < kSeries; ++k) frames_[k].assign(k < nser ? (size_t)(nframe_ * ntraj_) : 0, 0.0);
        ticks_.assign((size_t)(tick_cap_ > 0 ? tick_cap_ * ntraj_ : 0), 0);
        events_.assign((size_t)(event_cap_ > 0 ? event_cap_ * ntraj_ * (LDP_E_CG0 + p_.n_cg) : 0), 0.0);
        ldp_traj_results r = {};
        r.counts = counts_.data();
        r.sums = sums_.data();
        double* fr[kSeries];
        for (int k = 0; k < kSeries; ++k) fr[k] = frames_[k].empty() ? nullptr : frames_[k].data();
        r.frames_x = fr[kX];
        r.frames_v = fr[kV];
        r.frames_f = fr[kF];
        r.frames_pe = fr[kPE];
        r.frames_ke = fr[kKE];
        r.frames_state = fr[kState];
        r.frames_barrier = fr[kBarrier];
        r.ticks = ticks_.empty() ? nullptr : ticks_.data();
        r.events = events_.empty() ? nullptr : events_.data();
        if (ldp_job_traj_results(job_, &r) != LDP_OK) return fail("results");
        saved_ = false;
        return true;
    }
    void release() {
        if (job_) ldp_job_destroy(job_);
        job_ = nullptr;
    }
    // the lane's trajectory in the object's job (its trials of this rank)
    int64_t traj(int index) const { return (int64_t)trial_ * lanes_ + index; }
    int64_t count(int field, int index) {
        if (!lane_ok(index) || !ready("getter")) return 0;
        return counts_[(size_t)(field * ntraj_ + traj(index))];
    }
    // STATISTICS::AVERAGE of the event list: 0 without events
    double average(int cfield, int sfield, int index) {
        if (!lane_ok(index) || !ready("getter")) return std::numeric_limits<double>::quiet_NaN();
        const int64_t c = count(cfield, index);
        return c ? sums_[(size_t)(sfield * ntraj_ + traj(index))] / (double)c : 0.0;
    }
    size_t event_at(int list, int index, int64_t k) const {
        return (size_t)(((int64_t)list * ntraj_ + traj(index)) * event_cap_ + k);
    }
    double event(int list, int cfield, int index, size_t k) {
        if (!lane_ok(index) || !events_ok("per-event getter")) return std::numeric_limits<double>::quiet_NaN();
        const int64_t c = count(cfield, index);
        if ((int64_t)k >= c) return bad("event", (long long)k);
        if ((int64_t)k >= event_cap_) return bad("event beyond the kept list", (long long)k);
        return events_[event_at(list, index, (int64_t)k)];
    }
    size_t series_frames(int s, int index) {
        if (!lane_ok(index) || !ready("GetNumberOfFrame")) return 0;
        return frames_[s].empty() ? 0 : (size_t)nframe_;
    }
    double frame(int s, int index, size_t f) {
        if (!lane_ok(index) || !ready("frame getter")) return std::numeric_limits<double>::quiet_NaN();
        if (frames_[s].empty() || (int64_t)f >= nframe_) return bad("frame", (long long)f);
        return frames_[s][(size_t)f * (size_t)ntraj_ + (size_t)traj(index)];
    }
    std::vector<double>& series(int s, int index) {
        static std::vector<double> none;
        if (!lane_ok(index) || !ready("frame getter")) return none;
        std::vector<double>& v = x_[(size_t)s * lanes_ + index];
        if (v.empty() && !frames_[s].empty())
            for (int64_t f = 0; f < nframe_; ++f) v.push_back(frames_[s][(size_t)(f * ntraj_ + traj(index))]);
        return v;
    }
    void add_nothing(int index, Histogram* h) {
        if (!lane_ok(index) || !h) return;
        if ((int)h->count.size() < h->size) h->count.resize((size_t)h->size, 0.0);
    }

    ldp_ctx* ctx_;
    ldp_params p_;
    int lanes_, ranks_, rank_, precision_;
    ldp_job* job_ = nullptr;
    bool restore_ = false, saved_ = false;
    int trial_ = 0;
    int64_t ntraj_ = 0, nframe_ = 0, tick_cap_ = 0, event_cap_ = 0;
    std::vector<int64_t> counts_, ticks_;
    std::vector<double> sums_, events_;
    std::vector<double> frames_[kSeries];
    std::vector<std::vector<double>> x_, tick_, tpt2_;
};

}  // namespace ldp
