// ldp_fp32.cu -- FP32 batched persistent trajectory kernel.
//
// Same model as the FP64 plain path (src/langevinDynamicsSingleBarrier.h:
// 1292-1324, 1680-1706, 1861-1884, 1998-2165, 2334-2592, 2860-2886 and the
// double-barrier counterparts in src/langevinDynamicsDoubleBarrier.h), with
// the step in FP32:
//  * position = cell * L + xp with an int cell index and an FP32 cell-local
//    coordinate xp in [-L/2, L/2) (no FP32 absolute position);
//  * Box-Muller noise on the special-function units (__logf, __sincosf) from
//    the same Philox words the FP64 path uses, so both paths integrate the
//    same noise sequence;
//  * an exact integer step counter as the clock; event durations are summed
//    as integer step counts (exact), frames are saved as FP64 cell*L + xp.
// The rare paths (cell entry catch-up, renewal statistics, frame records,
// trajectory start/retire) are out-of-line functions so that the hot loop
// keeps few registers.
//
// Batching: each thread is a slot that owns one trajectory; when it retires
// (fixed step count reached, or first passage in FIRST_PASSAGE mode) the
// warp's retired lanes claim new trajectories from the device work queue
// with one compare-and-swap per warp and a ballot/popc prefix.
#include <cuda_runtime.h>

#include "ldp_device.cuh"
#include "ldp_fp32.h"

namespace ldp {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kClaimTries = 1 << 16;   // bound of the claim retry loop

__device__ __forceinline__ int64_t fkey(bool dbl, int cell, int lb) {
    return dbl ? (int64_t)cell * 2 + lb : (int64_t)cell;
}

__device__ int f_default_state(const JobF& J, bool dbl, uint32_t g, int64_t ck) {
    if (J.us) {
        if (dbl) return J.init_state;
        const int64_t trial = ((int64_t)g / J.lanes) % J.nruns;
        if (trial == 0) return 0;
        if (!J.rs) return J.init_state;
        const Words w = philox_at(0, g - (uint32_t)J.lanes, TAG_INIT, J.key0, J.key1);
        return ((double)w.w0 * 0x1p-32 <= J.p_first) ? 0 : 1;
    }
    const Words w = philox_at((uint64_t)ck, g, TAG_CELL, J.key0, J.key1);
    return ((double)w.w0 * 0x1p-32 < J.p_cell0) ? 0 : 1;
}

__device__ void f_ring_load(const JobF& J, const SlotsDev& S, int64_t slot, bool dbl, uint32_t g, int64_t ck,
                            int* state, int64_t* stamp) {
    const int64_t r = ck & (int64_t)(S.ring_slots - 1);
    const int64_t o = r * S.nslots + slot;
    if (S.ring_tag[o] == ck) {
        const int64_t d = S.ring_data[o];
        *state = (int)(d & 1);
        *stamp = d >> 1;
    } else {
        *state = f_default_state(J, dbl, g, ck);
        *stamp = 0;
    }
}

__device__ void f_ring_store(const JobF& J, const SlotsDev& S, int64_t slot, int64_t traj, int64_t ck, int state,
                             int64_t stamp) {
    const int64_t r = ck & (int64_t)(S.ring_slots - 1);
    const int64_t o = r * S.nslots + slot;
    const int64_t old = S.ring_tag[o];
    if (old != ck && old != INT64_MIN) J.counts[(int64_t)LDP_C_EVICT * J.ntraj + traj] += 1;
    S.ring_tag[o] = ck;
    S.ring_data[o] = (stamp << 1) | (int64_t)state;
}

// Cell (double model: local barrier) entry: save the state of the cell left,
// load the entered cell and catch it up over the steps it was not observed
// (UpdateBarrierStateEta, S.h:2025-2068 / D.h:2468-2517).  The catch-up
// probability is evaluated in FP64 exactly as in the FP64 path.
__device__ __noinline__ int f_enter_cell(const JobF* Jp, const SlotsDev S, int64_t slot, int64_t traj, bool dbl,
                                         uint32_t g, int64_t key_prev, int state, int64_t key_cur, uint64_t s) {
    const JobF& J = *Jp;
    f_ring_store(J, S, slot, traj, key_prev, state, (int64_t)s);
    int ps;
    int64_t stamp;
    f_ring_load(J, S, slot, dbl, g, key_cur, &ps, &stamp);
    if (!J.eta) return ps;
    const double lap = (double)((int64_t)s - stamp);
    const double pl = J.c_lap[J.eq ? 0 : ps] * -expm1_f64(J.a_lap * lap);
    const uint64_t Tl = prob_to_u64(pl);
    const Words wc = philox_at(s, g, TAG_CATCHUP, J.key0, J.key1);
    const uint64_t U = ((uint64_t)wc.w0 << 32) | wc.w1;
    return (U < Tl) ? (ps ^ 1) : ps;
}

__device__ __noinline__ bool f_refine_flip(const JobF* Jp, uint32_t g, uint64_t s, uint32_t tlo) {
    const Words wr = philox_at(s, g, TAG_REFINE, Jp->key0, Jp->key1);
    return wr.w0 < tlo;
}

// FP32 force constants of one job, kept in registers by the hot loop.
struct ForceC {
    float w, sl0, sl1;                       // single barrier
    float xb0, xb1, lo0, hi1, xc;            // double barrier geometry
    float n0[2], p0[2], n1[2], p1[2];        // double barrier slopes by state
};

__device__ __forceinline__ ForceC f_force_consts(const JobF& J) {
    ForceC c;
    c.w = J.w; c.sl0 = J.slope[0]; c.sl1 = J.slope[1];
    c.xb0 = J.xb[0]; c.xb1 = J.xb[1]; c.lo0 = J.lo0; c.hi1 = J.hi1; c.xc = J.xc;
    for (int s = 0; s < 2; ++s) { c.n0[s] = J.sN[0][s]; c.p0[s] = J.sP[0][s]; c.n1[s] = J.sN[1][s]; c.p1[s] = J.sP[1][s]; }
    return c;
}

// FP32 force of the current state (EnergyAndForce, S.h:1292-1324 /
// D.h:1464-1522).
template <bool DBL>
__device__ __forceinline__ float f_force(const ForceC& c, float xp, int state) {
    if (!DBL) {
        const float a = fabsf(xp);
        const float sl = state ? c.sl1 : c.sl0;
        return (a < c.w && a > 0.0f) ? copysignf(sl, xp) : 0.0f;
    } else {
        float f = 0.0f;
        if (xp < c.xb0 && xp > c.lo0) f = state ? c.n0[1] : c.n0[0];
        if (xp < c.xc && xp > c.xb0) f = state ? c.p0[1] : c.p0[0];
        if (xp < c.xb1 && xp > c.xc) f = state ? c.n1[1] : c.n1[0];
        if (xp < c.hi1 && xp > c.xb1) f = state ? c.p1[1] : c.p1[0];
        return -f;
    }
}

template <bool DBL>
__device__ void f_energy(const JobF& J, double xp, int s, double* E, double* B) {
    if (!DBL) {
        const double sp = J.Hs[s] / J.wd, sn = -sp;
        double e = 0.0;
        if (xp < 0.0 && xp > -J.wd) e = J.Hs[s] - xp * sn;
        if (xp < J.wd && xp > 0.0) e = J.Hs[s] - xp * sp;
        *E = e;
        *B = J.Hs[s];
    } else {
        double e = 0.0, b = 0.0;
        if (xp < J.xbd[0] && xp > J.lo0d) { e = xp * J.sNd[0][s] + J.iN[0][s]; b = J.Hd[0][s]; }
        if (xp < J.xcd && xp > J.xbd[0]) { e = xp * J.sPd[0][s] + J.iP[0][s]; b = J.Hd[0][s]; }
        if (xp < J.xbd[1] && xp > J.xcd) { e = xp * J.sNd[1][s] + J.iN[1][s]; b = J.Hd[1][s]; }
        if (xp < J.hi1d && xp > J.xbd[1]) { e = xp * J.sPd[1][s] + J.iP[1][s]; b = J.Hd[1][s]; }
        *E = e;
        *B = b;
    }
}

template <bool DBL>
__device__ __noinline__ void f_record(const JobF* Jp, int64_t traj, int64_t frame, int cell, float xp, float v,
                                      float F, int state) {
    const JobF& J = *Jp;
    const int64_t o = frame * J.ntraj + traj;
    const double x = (double)cell * J.Ld + (double)xp;
    if (J.fx) J.fx[o] = x;
    if (J.write_x) {
        double E, B;
        f_energy<DBL>(J, (double)xp, state, &E, &B);
        if (J.fv) J.fv[o] = (double)v;
        if (J.ff) J.ff[o] = (double)F;
        if (J.fb) J.fb[o] = B;
        if (J.fpe) J.fpe[o] = E;
        if (J.fke) J.fke[o] = J.mhalf * ((double)v * (double)v);
        if (J.fst) J.fst[o] = (double)state;
    }
}

__device__ __forceinline__ bool cg_hit32(int well, int size) { return (well % size) == 0; }

// FPT initial-barrier bookkeeping (S.h:2187-2211, 2364-2388).
__device__ void f_fpt_initial(const JobF& J, const SlotsDev& S, int64_t slot, uint32_t g, int64_t traj, int cell,
                              int well, int state, uint32_t* bits) {
    int s0, s1;
    int64_t stamp;
    if (well == cell) {
        s0 = state;
        J.init_idx0[traj] = cell;
        f_ring_load(J, S, slot, false, g, (int64_t)cell + 1, &s1, &stamp);
        J.init_idx1[traj] = cell + 1;
    } else {
        f_ring_load(J, S, slot, false, g, (int64_t)cell - 1, &s0, &stamp);
        J.init_idx0[traj] = cell - 1;
        s1 = state;
        J.init_idx1[traj] = cell;
    }
    *bits = (*bits & ~(B_INIT0 | B_INIT1)) | (s0 ? B_INIT0 : 0u) | (s1 ? B_INIT1 : 0u);
}

__device__ __forceinline__ void f_fpt2_idx(const JobF& J, int64_t traj, int cell, int well) {
    if (well == cell) { J.idx2_0[traj] = cell; J.idx2_1[traj] = cell + 1; }
    else { J.idx2_0[traj] = cell - 1; J.idx2_1[traj] = cell; }
}

// Renewal statistics (UpdateStatistics, S.h:2334-2592 / D.h:2931-3209) with
// integer step clocks.  Returns true when a FIRST_PASSAGE trajectory ends.
template <bool DBL>
__device__ __noinline__ bool f_events(const JobF* Jp, const SlotsDev S, int64_t slot, uint32_t g, int64_t traj,
                                      uint64_t s, bool dWell, bool dCell, int cell, int well, int state) {
    const JobF& J = *Jp;
    const int64_t n = J.ntraj;
    uint32_t bits = (uint32_t)J.bits[traj];
    bool done = false;
    const int64_t now = (int64_t)s;
    if (!DBL && J.wt && !J.fp_mode) {
        if (dWell) { J.wt_tick[traj] = now; bits |= B_WT_PASSED; }
        else if (dCell && (bits & B_WT_PASSED)) {
            int64_t& nwt = J.counts[(int64_t)LDP_C_WT * n + traj];
            if (nwt < J.tick_cap) J.ticks[traj * J.tick_cap + nwt] = J.wt_tick[traj];
            else J.counts[(int64_t)LDP_C_FLAGS * n + traj] |= LDP_FLAG_TICK_OVERFLOW;
            nwt += 1;
            bits &= ~B_WT_PASSED;
        }
    }
    if (J.fpt || J.fp_mode) {
        if (!DBL && !J.fp_mode) {
            if ((bits & B_FPT_UP) && dCell) {
                bits &= ~B_FPT_UP;
                J.fpt_last[traj] = now;
                f_fpt_initial(J, S, slot, g, traj, cell, well, state, &bits);
            }
            if (!(bits & B_FPT_UP) && dWell) {
                bits |= B_FPT_UP;
                if (J.counts[(int64_t)LDP_C_FPT * n + traj] == 0)
                    J.ssum[(int64_t)LDP_S_FIRST_FPT * n + traj] = now - J.fpt_last[traj];
                J.ssum[(int64_t)LDP_S_FPT * n + traj] += now - J.fpt_last[traj];
                J.counts[(int64_t)LDP_C_FPT * n + traj] += 1;
                const bool ib = (cell == J.init_idx0[traj]) ? ((bits & B_INIT0) != 0) : ((bits & B_INIT1) != 0);
                J.counts[(int64_t)(ib ? LDP_C_INIT1 : LDP_C_INIT0) * n + traj] += 1;
                J.counts[(int64_t)(state ? LDP_C_INST1 : LDP_C_INST0) * n + traj] += 1;
            }
        }
        if ((bits & B_FPT2_UP) && dCell) {
            bits &= ~B_FPT2_UP;
            J.fpt2_last[traj] = now;
            f_fpt2_idx(J, traj, cell, well);
        }
        if (dCell && !(bits & B_FPT2_UP) && J.idx2_0[traj] != cell && J.idx2_1[traj] != cell) {
            if (J.counts[(int64_t)LDP_C_FPT2 * n + traj] == 0)
                J.ssum[(int64_t)LDP_S_FIRST_FPT2 * n + traj] = now - J.fpt2_last[traj];
            J.ssum[(int64_t)LDP_S_FPT2 * n + traj] += now - J.fpt2_last[traj];
            J.counts[(int64_t)LDP_C_FPT2 * n + traj] += 1;
            J.fpt2_last[traj] = now;
            f_fpt2_idx(J, traj, cell, well);
            if (J.fp_mode) done = true;
        }
    }
    if (!DBL && J.tpt && !J.fp_mode) {
        if (dCell) { bits &= ~B_TPT_UP; J.tpt_last[traj] = now; }
        if (!(bits & B_TPT_UP) && dWell) {
            bits |= B_TPT_UP;
            if (J.counts[(int64_t)LDP_C_TPT * n + traj] == 0)
                J.ssum[(int64_t)LDP_S_FIRST_TPT * n + traj] = now - J.tpt_last[traj];
            J.ssum[(int64_t)LDP_S_TPT * n + traj] += now - J.tpt_last[traj];
            J.counts[(int64_t)LDP_C_TPT * n + traj] += 1;
        }
        if (dCell) {
            if (bits & B_TPT2_UP) bits &= ~B_TPT2_UP;
            else if (well != J.tpt2_well[traj]) {
                if (J.counts[(int64_t)LDP_C_TPT2 * n + traj] == 0)
                    J.ssum[(int64_t)LDP_S_FIRST_TPT2 * n + traj] = now - J.tpt2_last[traj];
                J.ssum[(int64_t)LDP_S_TPT2 * n + traj] += now - J.tpt2_last[traj];
                J.counts[(int64_t)LDP_C_TPT2 * n + traj] += 1;
            }
            J.tpt2_last[traj] = now;
            J.tpt2_well[traj] = well;
        }
    }
    if (J.cg && !J.fp_mode && dCell) {
        for (int jj = 0; jj < J.n_cg; ++jj) {
            if (cg_hit32(well, J.cg_size[jj])) {
                const int64_t o = (int64_t)jj * n + traj;
                if (bits & (B_CG0 << jj)) {
                    bits &= ~(B_CG0 << jj);
                    J.cg_last[o] = now;
                    J.cg_well[o] = well;
                } else if (well != J.cg_well[o]) {
                    J.ssum[(int64_t)(LDP_S_CG0 + jj) * n + traj] += now - J.cg_last[o];
                    J.counts[(int64_t)(LDP_C_CG0 + jj) * n + traj] += 1;
                    J.cg_last[o] = now;
                    J.cg_well[o] = well;
                }
            }
        }
    }
    J.bits[traj] = (int32_t)bits;
    return done;
}

// Step 0 of a trajectory (IntegrateStep0 + InitializeBarrierState +
// InitializeStatistics), FP64 where it is cheap and exact, then the hot
// state is rounded to FP32.
template <bool DBL, bool OVER>
__device__ __noinline__ void f_start(const JobF* Jp, const SlotsDev S, int64_t slot, int64_t traj, float* xp,
                                     float* rv, int* cell, int* state, int* lb) {
    const JobF& J = *Jp;
    const uint32_t g = (uint32_t)traj;
    for (int r = 0; r < S.ring_slots; ++r) S.ring_tag[(int64_t)r * S.nslots + slot] = INT64_MIN;
    const double red = J.x0 * J.invL;
    const int64_t c = (int64_t)rint(red);
    const int64_t well = (int64_t)floor(red);
    const double xpd = J.x0 - (double)c * J.Ld;
    int l = 0;
    if (DBL) l = (xpd < J.xcd) ? 0 : 1;
    const Words w0 = philox_at(0, g, TAG_INIT, J.key0, J.key1);
    const int st = J.rs ? (((double)w0.w0 * 0x1p-32 <= J.p_first) ? 0 : 1) : J.init_state;
    double zv, zr;
    gauss_pair_f64(w0.w1, w0.w2, &zv, &zr);
    const double v = J.rv ? J.sig_v0 * zv : J.v0;
    J.state0[traj] = st;
    J.v0s[traj] = v;
    uint32_t bits = 0;
    if (J.at_bottom) {
        if (!DBL && J.fpt && !J.fp_mode)
            f_fpt_initial(J, S, slot, g, traj, (int)c, (int)well, st, &bits);
        f_fpt2_idx(J, traj, (int)c, (int)well);
    } else {
        bits |= B_FPT_UP | B_FPT2_UP;
    }
    if (!J.at_bottom) bits |= B_TPT_UP | B_TPT2_UP;
    J.tpt2_well[traj] = (int32_t)well;
    J.fpt_last[traj] = 0;
    J.fpt2_last[traj] = 0;
    J.tpt_last[traj] = 0;
    J.tpt2_last[traj] = 0;
    J.wt_tick[traj] = 0;
    for (int j = 0; j < J.n_cg; ++j) {
        J.cg_last[(int64_t)j * J.ntraj + traj] = 0;
        J.cg_well[(int64_t)j * J.ntraj + traj] = (int32_t)well;
        if (!(J.at_bottom && cg_hit32((int)well, J.cg_size[j]))) bits |= (B_CG0 << j);
    }
    J.bits[traj] = (int32_t)bits;
    *xp = (float)xpd;
    *cell = (int)c;
    *state = st;
    *lb = l;
    *rv = OVER ? (float)(J.sig_r_d * zr) : (float)v;
    if (!J.fp_mode) {
        const float F = f_force<DBL>(f_force_consts(J), *xp, st);
        f_record<DBL>(Jp, traj, 0, (int)c, *xp, OVER ? 0.0f : (float)v, F, st);
    }
}

__device__ __noinline__ void f_retire(const JobF* Jp, const SlotsDev S, int64_t traj, uint64_t steps_done,
                                      int64_t sc1, int cell, float xp, float v, int state, uint32_t flags) {
    const JobF& J = *Jp;
    const int64_t n = J.ntraj;
    J.counts[(int64_t)LDP_C_STATE1 * n + traj] = sc1;
    J.counts[(int64_t)LDP_C_STATE0 * n + traj] = (int64_t)steps_done + 1 - sc1;
    J.counts[(int64_t)LDP_C_STEPS * n + traj] = (int64_t)steps_done;
    if (flags) J.counts[(int64_t)LDP_C_FLAGS * n + traj] |= (int64_t)flags;
    J.x_final[traj] = (double)cell * J.Ld + (double)xp;
    J.v_final[traj] = (double)v;
    J.state_final[traj] = state;
    atomicAdd(J.remaining, ~0ull);   // -1 modulo 2^64
    atomicAdd(S.retired, 1ull);
}

// Resolves a claimed queue index to (job, trajectory).
__device__ __noinline__ void f_resolve(const QueueDev q, int64_t idx, int* job, int64_t* traj) {
    int lo = 0, hi = *(volatile int32_t*)q.nranges - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (q.range_end[mid] > idx) hi = mid; else lo = mid + 1;
    }
    const int64_t begin = lo ? q.range_end[lo - 1] : 0;
    *job = q.range_job[lo];
    *traj = q.range_first[lo] + (idx - begin);
}

}  // namespace

template <bool DBL, bool OVER>
__global__ void __launch_bounds__(256) fp32_persistent_kernel(const QueueDev q, const SlotsDev S,
                                                              uint64_t pair_budget) {
    const int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned lane = threadIdx.x & 31u;
    const bool in_range = slot < S.nslots;

    // ---- slot state ----
    int job = in_range ? S.job[slot] : -1;
    int64_t traj = 0;
    uint64_t s = 1;
    float xp = 0.f, rv = 0.f;
    int cell = 0, state = 0, lb = 0;
    int64_t sc1 = 0;
    if (job >= 0) {
        traj = S.traj[slot];
        s = (uint64_t)S.step[slot];
        xp = S.xp[slot];
        rv = S.rv[slot];
        cell = S.cell[slot];
        const int st = S.st[slot];
        state = st & 1;
        lb = (st >> 1) & 1;
        sc1 = S.sc1[slot];
    }
    // Hot per-job constants in registers.
    const JobF* J = nullptr;
    float L = 0.f, halfL = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f, c4 = 0.f;
    ForceC fc{};
    uint32_t key0 = 0, key1 = 0, thi0 = 0, thi1 = 0, g = 0;
    uint64_t nsteps = 0, fs = 0, to_rec = 0;
    int well = 0;
    float F = 0.f;
    auto bind = [&]() {
        J = &q.jobs[job];
        L = J->L; halfL = J->halfL;
        if (OVER) { c1 = J->c_drift; c2 = J->sig_r; }
        else { c1 = J->hdt_invM; c2 = J->hdt; c3 = J->expg; c4 = J->sig_v; }
        fc = f_force_consts(*J);
        key0 = J->key0; key1 = J->key1;
        const uint64_t T0 = J->eq ? J->T_eq : J->T_as[0];
        const uint64_t T1 = J->eq ? J->T_eq : J->T_as[1];
        thi0 = (uint32_t)(T0 >> 32);
        thi1 = (uint32_t)(T1 >> 32);
        nsteps = J->nsteps;
        fs = J->fp_mode ? 0 : J->freq_save;
        g = (uint32_t)traj;
        well = cell - (xp < 0.0f ? 1 : 0);
        F = f_force<DBL>(fc, xp, state);
        to_rec = fs ? fs - ((s - 1) % fs) : ~0ull;
    };
    if (job >= 0) bind();

    bool dry = false;   // the queue had nothing left for this warp
    uint32_t flags = 0;
    for (uint64_t it = 0; it < pair_budget; ++it) {
        // ---- warp-aggregated refill ----
        const bool need = in_range && job < 0 && !dry;
        const unsigned m = __ballot_sync(kFull, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0, got = 0;
            if ((int)lane == leader) {
                const unsigned long long tail = *(volatile unsigned long long*)q.tail;
                unsigned long long old = *(volatile unsigned long long*)q.head;
                for (int tries = 0; tries < kClaimTries; ++tries) {
                    if (old >= tail) break;
                    const unsigned long long want = min((unsigned long long)__popc(m), tail - old);
                    const unsigned long long prev = atomicCAS(q.head, old, old + want);
                    if (prev == old) { base = old; got = want; break; }
                    old = prev;
                }
            }
            base = __shfl_sync(kFull, base, leader);
            got = __shfl_sync(kFull, got, leader);
            if (got < (unsigned long long)__popc(m)) dry = true;
            if (need) {
                const unsigned rank = __popc(m & ((1u << lane) - 1u));
                if (rank < got) {
                    int64_t t;
                    f_resolve(q, (int64_t)(base + rank), &job, &t);
                    traj = t;
                    f_start<DBL, OVER>(&q.jobs[job], S, slot, traj, &xp, &rv, &cell, &state, &lb);
                    s = 1;
                    sc1 = state;
                    flags = 0;
                    bind();
                }
            }
        }
        if (__all_sync(kFull, job < 0)) {
            if (dry || !__any_sync(kFull, need)) break;
            continue;
        }
        if (job < 0) continue;

        // ---- one Philox call, two steps ----
        const uint64_t j = (s - 1) >> 1;
        const Words w = philox((uint32_t)j, (uint32_t)(j >> 32), g, TAG_STEP, key0, key1);
        float za, zb;
        gauss_pair_f32(w.w0, w.w1, &za, &zb);
        bool finished = false;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 1 && (finished || s > nsteps)) break;
            const float z = h ? zb : za;
            const uint32_t fw = h ? w.w3 : w.w2;
            const int cell_prev = cell, well_prev = well, lb_prev = lb;
            if (OVER) {
                const float rf = c2 * z;
                xp = fmaf(F, c1, xp);
                xp = xp + rf;
                xp = xp + rv;
                rv = rf;
            } else {
                rv = fmaf(F, c1, rv);
                xp = fmaf(rv, c2, xp);
                rv = fmaf(c3, rv, c4 * z);
                xp = fmaf(rv, c2, xp);
            }
            if (!isfinite(xp)) {
                flags |= LDP_FLAG_NONFINITE;
                finished = true;
                break;
            }
            if (xp >= halfL) { xp -= L; ++cell; }
            else if (xp < -halfL) { xp += L; --cell; }
            well = cell - (xp < 0.0f ? 1 : 0);
            if (DBL) lb = (xp < fc.xc) ? 0 : 1;
            const bool dCell = cell != cell_prev;
            const bool dWell = well != well_prev;
            const bool dKey = DBL ? (lb != lb_prev) : dCell;
            // per-step dichotomic flip: 64-bit Bernoulli, high word first
            const uint32_t thi = state ? thi1 : thi0;
            bool flip = fw < thi;
            if (fw == thi) {
                const uint64_t T = J->eq ? J->T_eq : J->T_as[state];
                flip = f_refine_flip(J, g, s, (uint32_t)T);
            }
            state ^= (int)flip;
            if (dKey)
                state = f_enter_cell(J, S, slot, traj, DBL, g, fkey(DBL, cell_prev, lb_prev), state,
                                     fkey(DBL, cell, lb), s);
            sc1 += state;
            F = f_force<DBL>(fc, xp, state);
            if (!OVER) rv = fmaf(F, c1, rv);
            if (dCell || dWell) finished = f_events<DBL>(J, S, slot, g, traj, s, dWell, dCell, cell, well, state);
            if (--to_rec == 0) {
                f_record<DBL>(J, traj, (int64_t)(s / fs), cell, xp, OVER ? 0.0f : rv, F, state);
                to_rec = fs;
            }
            if (s == nsteps) finished = true;
            ++s;
        }
        if (finished) {
            const uint64_t done = s - 1;
            if (J->fp_mode && !(flags & LDP_FLAG_NONFINITE) && J->counts[(int64_t)LDP_C_FPT2 * J->ntraj + traj] == 0)
                flags |= LDP_FLAG_CENSORED;
            f_retire(J, S, traj, done, sc1, cell, xp, OVER ? (float)0.0f : rv, state, flags);
            job = -1;
        }
    }
    if (!in_range) return;
    S.job[slot] = job;
    if (job >= 0) {
        S.traj[slot] = traj;
        S.step[slot] = (int64_t)s;
        S.xp[slot] = xp;
        S.rv[slot] = rv;
        S.cell[slot] = cell;
        S.st[slot] = state | (lb << 1);
        S.sc1[slot] = sc1;
    }
}

int fp32_blocks_per_sm(bool dbl, bool over, int block) {
    int n = 0;
    cudaError_t e;
    if (dbl) e = over ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<true, true>, block, 0)
                      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<true, false>, block, 0);
    else e = over ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<false, true>, block, 0)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<false, false>, block, 0);
    return e == cudaSuccess ? n : 0;
}

int launch_fp32_persistent(bool dbl, bool over, const QueueDev& q, const SlotsDev& s, uint64_t pair_budget, int grid,
                           int block, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (dbl) {
        if (over) fp32_persistent_kernel<true, true><<<grid, block, 0, st>>>(q, s, pair_budget);
        else fp32_persistent_kernel<true, false><<<grid, block, 0, st>>>(q, s, pair_budget);
    } else {
        if (over) fp32_persistent_kernel<false, true><<<grid, block, 0, st>>>(q, s, pair_budget);
        else fp32_persistent_kernel<false, false><<<grid, block, 0, st>>>(q, s, pair_budget);
    }
    return (int)cudaGetLastError();
}

}  // namespace ldp
