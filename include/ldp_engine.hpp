/*
 * ldp_engine.hpp -- the reference's engine interface over the C ABI.
 *
 * ldp::LangevinEquationSIMDMultiple has the public methods of the
 * reference's engine class of the same name
 * (src/langevinDynamicsSingleBarrier.h:1276-2769; the overdamped and
 * double-barrier engines have the same ones): Initialize, Integrate and the
 * per-lane getters, with the same lane indices and the same error
 * convention (Integrate returns false after printing the error on stderr),
 * for C++ hosts that drive the engine in process instead of through the
 * executables.  Header only, over include/ldp.h.
 *
 * One object stands for one virtual rank of a run: `lanes` trajectories per
 * trial (the reference's SIMD width), NUMBEROFRUNS trials, `ranks` ranks.
 * Integrate(iTrial) makes trial iTrial current and the getters read its
 * lane `index`.  The whole run (every trial of every rank) is one job of the
 * library, integrated at the first Integrate after Initialize: each
 * trajectory's random streams are keyed by (seed, trajectory, step), so the
 * results are those of a trial-by-trial run.  bTimer is accepted and
 * ignored (the reference prints progress lines with it).
 */
#pragma once

#include <cstdint>
#include <cstdio>
#include <vector>

#include "ldp.h"

namespace ldp {

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
    }

    // S.h:1386: integrates the run if it has not been (every trial at once)
    // and makes trial iTrial current.
    virtual bool Integrate(int iTrial, bool bTimer = false) {
        (void)bTimer;
        if (iTrial < 0 || iTrial >= p_.number_of_runs || rank_ < 0 || rank_ >= ranks_) {
            std::fprintf(stderr, "Error: trial %d / rank %d outside the run (%d trials, %d ranks)\n", iTrial, rank_,
                         p_.number_of_runs, ranks_);
            return false;
        }
        if (!job_ && !run()) return false;
        trial_ = iTrial;
        x_.assign(lanes_, std::vector<double>());
        tick_.assign(lanes_, std::vector<double>());
        return true;
    }

    size_t GetNumberOfFrameX(int index) { return lane_ok(index) ? (size_t)nframe_ : 0; }
    double GetX(int index, size_t frameID) { return frames_[frameID * (size_t)ntraj_ + (size_t)traj(index)]; }
    std::vector<double>& GetX(int index) {
        std::vector<double>& v = x_[index];
        if (v.empty())
            for (int64_t f = 0; f < nframe_; ++f) v.push_back(frames_[(size_t)(f * ntraj_ + traj(index))]);
        return v;
    }
    size_t GetFirstPassageTimeCount(int index) { return (size_t)count(LDP_C_FPT, index); }
    size_t GetFirstPassageTimeCount2(int index) { return (size_t)count(LDP_C_FPT2, index); }
    double GetFirstPassageTimeAverage(int index) { return average(LDP_C_FPT, LDP_S_FPT, index); }
    double GetFirstPassageTimeAverage2(int index) { return average(LDP_C_FPT2, LDP_S_FPT2, index); }
    double GetTransitionPathTimeAverage(int index) { return average(LDP_C_TPT, LDP_S_TPT, index); }
    double GetTransitionPathTimeAverage2(int index) { return average(LDP_C_TPT2, LDP_S_TPT2, index); }
    // sizeIndex: the FPTCG entry of the .inp, in order
    double GetFirstPassageTimeCGAverage2(int index, int sizeIndex) {
        return average(LDP_C_CG0 + sizeIndex, LDP_S_CG0 + sizeIndex, index);
    }
    // steps spent in barrier state iState (0 or 1), step 0 included
    double GetStateCount(int index, int iState) { return (double)count(LDP_C_STATE0 + iState, index); }
    // waiting-time ticks: the steps at which a well change was followed by a
    // cell change (WAITINGTIME), as the reference stores them
    std::vector<double>& GetBarrierTick(int index) {
        std::vector<double>& v = tick_[index];
        if (v.empty() && tick_cap_ > 0) {
            const int64_t n = count(LDP_C_WT, index) < tick_cap_ ? count(LDP_C_WT, index) : tick_cap_;
            for (int64_t k = 0; k < n; ++k) v.push_back((double)ticks_[(size_t)(traj(index) * tick_cap_ + k)]);
        }
        return v;
    }

   private:
    bool fail(const char* what) {
        std::fprintf(stderr, "Error: %s: %s\n", what, ctx_ ? ldp_last_error(ctx_) : "no context");
        release();
        return false;
    }
    bool run() {
        ldp_job_opts o;
        ldp_job_opts_default(&o);
        o.lanes = lanes_;
        o.ranks = ranks_;
        o.precision = precision_;
        if (ldp_job_create(ctx_, &p_, &o, &job_) != LDP_OK) return fail("job creation");
        if (ldp_submit(ctx_, job_) != LDP_OK || ldp_wait(ctx_, job_) != LDP_OK) return fail("integration");
        ldp_job_info info;
        if (ldp_job_info_get(job_, &info) != LDP_OK) return fail("job info");
        ntraj_ = info.ntraj;
        nframe_ = info.nframe;
        tick_cap_ = info.tick_cap;
        counts_.assign((size_t)(LDP_NCOUNT * ntraj_), 0);
        sums_.assign((size_t)(LDP_NSUM * ntraj_), 0.0);
        frames_.assign((size_t)(nframe_ * ntraj_), 0.0);
        ticks_.assign((size_t)(tick_cap_ > 0 ? tick_cap_ * ntraj_ : 0), 0);
        ldp_traj_results r = {};
        r.counts = counts_.data();
        r.sums = sums_.data();
        r.frames_x = frames_.empty() ? nullptr : frames_.data();
        r.ticks = ticks_.empty() ? nullptr : ticks_.data();
        if (ldp_job_traj_results(job_, &r) != LDP_OK) return fail("results");
        return true;
    }
    void release() {
        if (job_) ldp_job_destroy(job_);
        job_ = nullptr;
    }
    bool lane_ok(int index) const { return index >= 0 && index < lanes_; }
    int64_t traj(int index) const { return ((int64_t)rank_ * p_.number_of_runs + trial_) * lanes_ + index; }
    int64_t count(int field, int index) const { return counts_[(size_t)(field * ntraj_ + traj(index))]; }
    // STATISTICS::AVERAGE of the event list: 0 without events
    double average(int cfield, int sfield, int index) const {
        const int64_t c = count(cfield, index);
        return c ? sums_[(size_t)(sfield * ntraj_ + traj(index))] / (double)c : 0.0;
    }

    ldp_ctx* ctx_;
    ldp_params p_;
    int lanes_, ranks_, rank_, precision_;
    ldp_job* job_ = nullptr;
    int trial_ = 0;
    int64_t ntraj_ = 0, nframe_ = 0, tick_cap_ = 0;
    std::vector<int64_t> counts_, ticks_;
    std::vector<double> sums_, frames_;
    std::vector<std::vector<double>> x_, tick_;
};

}  // namespace ldp
