// Drives ldp::LangevinEquationSIMDMultiple (include/ldp_engine.hpp) the way
// the reference's runner drives its engine: Initialize(seed), then
// Integrate(iTrial) per trial and the per-lane getters.  Prints one line per
// (trial, lane): FPT count and average, FPT2 average, TPT average, state
// counts, last frame, the mean of the lane's per-event FPT list (GetFirst-
// PassageTime summed in order over the count; -1 without events), the size
// of its TPT2 list, whether a frame past the last one is rejected (NaN),
// the number of velocity frames and the first one (WRITEX).  Without a
// device context Integrate must fail with a message (the reference's error
// convention) and a getter before Integrate gives NaN; argv[3] == "nodevice"
// checks exactly that.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ldp_engine.hpp"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    char err[512];
    ldp_params p;
    if (ldp_params_from_inp(argv[1], LDP_MODEL_SINGLE, &p, err, sizeof err) != LDP_OK) {
        std::fprintf(stderr, "%s\n", err);
        return 2;
    }
    p.number_of_steps = std::strtoull(argv[2], nullptr, 10);
    p.freq_save = p.number_of_steps / 2000;   // 2001 frames
    p.random_seed = 1234;
    const bool nodevice = argc > 3 && std::strcmp(argv[3], "nodevice") == 0;
    ldp_ctx* ctx = nullptr;
    if (!nodevice && ldp_create(&ctx, 0) != LDP_OK) return 3;
    int rc = 0;
    {
        ldp::LangevinEquationSIMDMultiple e(ctx, p, 8, 2, 1);   // rank 1 of 2, 8 lanes
        e.Initialize((int)p.random_seed);
        if (nodevice) {
            const bool a = e.Integrate(0);
            const bool b = e.Integrate(p.number_of_runs);   // past the last trial
            const bool c = std::isnan(e.GetX(0, 0));          // before Integrate
            std::printf("%d %d %d\n", (int)a, (int)b, (int)c);
            rc = (a || b || !c) ? 1 : 0;
        } else {
            for (int trial = 0; trial < p.number_of_runs && rc == 0; ++trial) {
                if (!e.Integrate(trial)) { rc = 1; break; }
                for (int lane = 0; lane < 8; ++lane) {
                    const size_t nfpt = e.GetFirstPassageTimeCount(lane);
                    double sum = 0.0;
                    for (size_t k = 0; k < nfpt; ++k) sum += e.GetFirstPassageTime(lane, k);
                    const double ev_mean = nfpt ? sum / (double)nfpt : -1.0;
                    const size_t nf = e.GetNumberOfFrameX(lane);
                    std::printf("%d %d %zu %.17g %.17g %.17g %.17g %.17g %.17g %.17g %zu %d %zu %.17g\n", trial,
                                lane, nfpt, e.GetFirstPassageTimeAverage(lane), e.GetFirstPassageTimeAverage2(lane),
                                e.GetTransitionPathTimeAverage(lane), e.GetStateCount(lane, 0),
                                e.GetStateCount(lane, 1), e.GetX(lane).back(), ev_mean,
                                e.GetTransitionPathTimeAll2(lane).size(), (int)std::isnan(e.GetX(lane, nf)),
                                e.GetNumberOfFrameV(lane), e.GetNumberOfFrameV(lane) ? e.GetV(lane, 0) : 0.0);
                }
            }
        }
    }
    if (ctx) ldp_destroy(ctx);
    return rc;
}
