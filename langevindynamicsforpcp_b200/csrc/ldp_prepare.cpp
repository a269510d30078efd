// ldp_prepare.cpp -- per-job constants (host).
//
// Restates IntegrateInitializeVariables of the reference engines
// (src/langevinDynamicsSingleBarrier.h:1520-1618, overdamped 2812-2824;
// src/langevinDynamicsDoubleBarrier.h:1733-1937 with GetXc at 1722-1732,
// overdamped 3427-3439) plus the few run-level facts the kernels need.
#include <cmath>
#include <cstring>
#include "ldp_engine.h"

namespace ldp {

uint64_t effective_steps(const ldp_params& p) {
    // With FREQSAVE >= 10 the reference integrates whole FREQSAVE groups only
    // (S.h:1409-1456); otherwise every step (S.h:1457-1511).
    if (p.freq_save >= 10) return (p.number_of_steps / p.freq_save) * p.freq_save;
    return p.number_of_steps;
}

// Frames of the run, the previous steps of a restart included: the count
// the runner analyses (CalculateNumberOfFrame(numberOfStep +
// numberOfStepPrevious, saveFreq), S.h:3220 with S.h:1811).
int64_t frame_count(const ldp_params& p) {
    return (int64_t)((p.number_of_steps + p.number_of_previous_steps) / p.freq_save + 1);
}

static uint64_t to_u64_threshold(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return ~0ull;
    return (uint64_t)std::ldexp(p, 64);
}

void prepare_kconst(const ldp_params& p, const ldp_job_opts& o, uint32_t seed, KConst* k) {
    std::memset(k, 0, sizeof(*k));
    k->dbl = p.model == LDP_MODEL_DOUBLE;
    k->over = p.overdamped != 0;
    k->eta = p.tau != 0.0;
    k->eq = p.eq != 0;
    k->rv = p.randomize_v != 0;
    k->rs = p.randomize_states != 0;
    k->us = p.uniform_initial_states != 0;
    k->init_state = p.initial_state;
    // The double-barrier engine clears its waiting-time, bottom-to-top FPT and
    // TPT lists every step (D.h:2950-2953, 2962-2963, 3149-3153): they stay
    // empty, so they are not accumulated at all.
    k->wt = (p.waiting_time != 0) && !k->dbl;
    k->fpt = p.fpt != 0;
    k->tpt = (p.tpt != 0) && !k->dbl;
    k->cg = p.fptcg != 0;
    k->n_cg = p.n_cg;
    for (int j = 0; j < p.n_cg && j < LDP_MAX_CG; ++j) k->cg_size[j] = p.cg_sizes[j];
    k->write_x = p.write_x != 0;
    k->fp_mode = o.mode == LDP_MODE_FIRST_PASSAGE;
    k->lanes = o.lanes;
    k->nruns = p.number_of_runs;
    k->slots = o.table_slots;
    k->g0 = (uint32_t)((int64_t)o.first_rank * p.number_of_runs * o.lanes);
    k->key0 = seed;
    k->key1 = o.job_id;

    k->x0 = p.x0;
    k->v0 = p.v0;
    k->dt = p.timestep;
    k->L = p.periodic_length;
    k->invL = 1.0 / k->L;
    const double halfL = k->L * 0.5;
    if (!k->dbl) {
        k->w = p.barrier_half_width[0];
        k->Hs[0] = p.barrier_heights[0][0];
        k->Hs[1] = p.barrier_heights[0][1];
        k->slope[0] = k->Hs[0] / k->w;   // m_StateBarrierSlope_0, S.h:1589
        k->slope[1] = k->Hs[1] / k->w;
    } else {
        const double x1b = p.barrier_position[0], w1 = p.barrier_half_width[0];
        const double x2b = p.barrier_position[1], w2 = p.barrier_half_width[1];
        const double y1 = p.barrier_heights[0][0], y2 = p.barrier_heights[1][0];
        // Meeting point of the two inner flanks, from the state-0 heights.
        const double x1h = x1b + w1, x2l = x2b - w2;
        const double xc = (x1h * y1 * (x2b - x2l) + x2l * y2 * (x1h - x1b)) /
                          (y1 * (x2b - x2l) + y2 * (x1h - x1b));
        const double yc = (x1h - xc) / (x1h - x1b) * y1;
        k->xc = xc;
        k->xb[0] = x1b;
        k->xb[1] = x2b;
        const double lo[2] = {x1b - w1, x2b - w2}, hi[2] = {x1b + w1, x2b + w2};
        k->lo0 = lo[0];
        k->hi1 = hi[1];
        const double xb_xl0 = k->xb[0] - lo[0];
        const double xh_xb1 = hi[1] - k->xb[1];
        for (int s = 0; s < 2; ++s) {
            const double h0 = p.barrier_heights[0][s], h1 = p.barrier_heights[1][s];
            k->Hd[0][s] = h0;
            k->Hd[1][s] = h1;
            // Slopes and intercepts of the four flanks (D.h:1863-1899).
            k->sN[0][s] = h0 / xb_xl0;
            k->sP[0][s] = (yc - h0) / (xc - k->xb[0]);
            k->sN[1][s] = (h1 - yc) / (k->xb[1] - xc);
            k->sP[1][s] = 0.0 - h1 / xh_xb1;
            k->iN[0][s] = 0.0 - h0 * (lo[0] / xb_xl0);
            k->iP[0][s] = (xc * h0 - yc * k->xb[0]) / (xc - k->xb[0]);
            k->iN[1][s] = (yc * k->xb[1] - xc * h1) / (k->xb[1] - xc);
            k->iP[1][s] = h1 * (hi[1] / xh_xb1);
        }
    }
    const double m = p.mass, g = p.gamma;
    k->invM = 1.0 / m;
    k->hdt = k->dt * 0.5;
    k->mhalf = m * 0.5;
    k->expg = std::exp(-g * k->dt);
    k->sig_v = std::sqrt(p.kb * p.temperature / m * (1.0 - std::exp(-2.0 * g * k->dt)));
    const double mgi = 1.0 / (m * g);
    k->c_drift = k->dt * mgi;
    k->sig_r = std::sqrt(p.kb * p.temperature * mgi * k->dt * 0.5);
    k->sig_v0 = std::sqrt(p.kb * p.temperature / m);
    const double K = p.eq_constant;
    // Flip probabilities (S.h:1542-1584); 1 - exp(a) is evaluated as
    // -expm1(a), which keeps its accuracy when dt/TAU is small.
    if (k->eq) {
        k->a_lap = -2.0 * k->dt / p.tau;
        k->T_eq = k->eta ? to_u64_threshold(0.5 * -std::expm1(-2.0 * k->dt / p.tau)) : 0;
        k->c_lap[0] = k->c_lap[1] = 0.5;
        k->p_first = 0.5;
    } else {
        k->a_lap = -(K + 1.0) * k->dt / p.tau;
        const double e = -std::expm1(k->a_lap);
        k->T_as[0] = k->eta ? to_u64_threshold(K / (1.0 + K) * e) : 0;
        k->T_as[1] = k->eta ? to_u64_threshold(1.0 / (1.0 + K) * e) : 0;
        k->c_lap[0] = K / (1.0 + K);
        k->c_lap[1] = 1.0 / (1.0 + K);
        k->p_first = 1.0 / (1.0 + K);
    }
    // Waiting times between flips (geometric in the per-step probability).
    for (int s = 0; s < 2; ++s) {
        double pf = 0.0;
        if (k->eta) pf = k->eq ? 0.5 * -std::expm1(-2.0 * k->dt / p.tau) : k->c_lap[s] * -std::expm1(k->a_lap);
        k->ln1m[s] = (pf > 0.0) ? std::log1p(-pf) : 0.0;
    }
    k->p_cell0 = 1.0 / (1.0 + K);   // BarrierStatus::Initialize, S.h:90
    // Math::Modulo(X0, L) == L/2 (S.h:2184, src/mathdef.h:20).
    k->at_bottom = std::fmod(std::fmod(k->x0, k->L) + k->L, k->L) == halfL;
    k->nsteps = effective_steps(p);
    k->freq_save = p.freq_save;
    k->step_cap = o.step_cap;
    k->nframe = frame_count(p);
    k->tick_cap = o.tick_cap;

    // FP32 cell-local constants.
    k->fL = (float)k->L;
    k->fhalfL = (float)halfL;
    k->fw = (float)k->w;
    k->fslope[0] = (float)k->slope[0];
    k->fslope[1] = (float)k->slope[1];
    k->fxb[0] = (float)k->xb[0];
    k->fxb[1] = (float)k->xb[1];
    k->flo0 = (float)k->lo0;
    k->fhi1 = (float)k->hi1;
    k->fxc = (float)k->xc;
    for (int b = 0; b < 2; ++b)
        for (int s = 0; s < 2; ++s) { k->fsN[b][s] = (float)k->sN[b][s]; k->fsP[b][s] = (float)k->sP[b][s]; }
    k->fc_drift = (float)k->c_drift;
    k->fsig_r = (float)k->sig_r;
    k->fhdt_invM = (float)(k->invM * k->hdt);
    k->fhdt = (float)k->hdt;
    k->fexpg = (float)k->expg;
    k->fsig_v = (float)k->sig_v;
}

}  // namespace ldp
