// ldp_fp64.cu -- plain FP64 trajectory kernels (one trajectory per thread).
//
// Device restatement of LangevinEquationSIMDMultiple and its overdamped
// subclass (src/langevinDynamicsSingleBarrier.h:823-2888) and of the
// double-barrier engine (src/langevinDynamicsDoubleBarrier.h:933-3507): the
// per-lane SIMD loop becomes one CUDA thread per trajectory, the lane's
// __m512d registers become this thread's registers, and the lazily grown
// per-cell barrier table (src/DataLocator.h:100-188) becomes a tagged ring
// of visited cells in HBM whose never-visited entries are a pure function of
// (trajectory, cell).
//
// Compiled with -fmad=false: every a*b+c is two roundings unless written as
// fma(), as in the reference's intrinsics (the only fused step is the
// overdamped drift, _mmSIMD_fmadd_pd at S.h:2868).
#include <cuda_runtime.h>
#include "ldp_device.cuh"
#include "ldp_engine.h"

namespace ldp {

struct T64 {
    double x, v, F, E, rprev, barrier;
    int64_t cell, well;
    int lb, state;
    uint32_t bits;
    double fpt_last, fpt2_last, tpt_last, tpt2_last;
    int64_t init_idx0, init_idx1, idx2_0, idx2_1, tpt2_well, wt_tick;
};

template <bool DBL>
__device__ __forceinline__ int64_t cell_key(int64_t cell, int lb) {
    return DBL ? cell * 2 + lb : cell;
}

// State of a cell never entered: BarrierStatus::Initialize (S.h:78-96),
// drawn from the trajectory's TAG_CELL stream; with UNIFORMINITALSTATES the
// value the reference hands over (S.h:1377-1380, D.h:1576-1578).
template <bool DBL>
__device__ int default_state(const KConst& k, uint32_t g, int64_t ck) {
    if (k.us) {
        if (DBL) return k.init_state;
        const int64_t trial = ((int64_t)g / k.lanes) % k.nruns;
        if (trial == 0) return 0;
        if (!k.rs) return k.init_state;
        const Words w = philox_at(0, g - (uint32_t)k.lanes, TAG_INIT, k.key0, k.key1);
        return ((double)w.w0 * 0x1p-32 <= k.p_first) ? 0 : 1;
    }
    const Words w = philox_at((uint64_t)ck, g, TAG_CELL, k.key0, k.key1);
    return ((double)w.w0 * 0x1p-32 < k.p_cell0) ? 0 : 1;
}

template <bool DBL>
// A cell-table entry: the barrier's state when it was left and its pending
// flip step; *found false for a cell never visited (state as drawn at its
// creation, step 0).
__device__ __forceinline__ void ring_load(const KConst& k, const TrajState& st, int64_t i, uint32_t g, int64_t ck,
                                          int* state, int64_t* nflip, bool* found) {
    const int64_t slot = ck & (int64_t)(k.slots - 1);
    const int64_t o = slot * st.n + i;
    if (st.ring_tag[o] == ck) {
        const int64_t d = st.ring_data[o];
        *state = (int)(d & 1);
        *nflip = d >> 1;
        *found = true;
    } else {
        *state = default_state<DBL>(k, g, ck);
        *nflip = 0;
        *found = false;
    }
}

__device__ __forceinline__ void ring_store(const KConst& k, const TrajState& st, int64_t i, int64_t ck, int state,
                                           int64_t nflip) {
    const int64_t slot = ck & (int64_t)(k.slots - 1);
    const int64_t o = slot * st.n + i;
    const int64_t old = st.ring_tag[o];
    if (old != ck && old != INT64_MIN) st.counts[(int64_t)LDP_C_EVICT * st.n + i] += 1;
    st.ring_tag[o] = ck;
    st.ring_data[o] = (nflip << 1) | (int64_t)state;
}

// EnergyAndForce, S.h:1292-1324 / D.h:1464-1522.
template <bool DBL>
__device__ __forceinline__ void energy_force(const KConst& k, T64& t) {
    const int s = t.state;
    const double xp = t.x - (double)t.cell * k.L;
    if (!DBL) {
        const double sp = k.slope[s], sn = 0.0 - sp, H = k.Hs[s];
        const bool onN = (xp < 0.0) && (xp > -k.w);
        const bool onP = (xp < k.w) && (xp > 0.0);
        double E = 0.0, F = 0.0;
        if (onN) { E = H - xp * sn; F = sn; }
        if (onP) { E = H - xp * sp; F = sp; }
        t.E = E;
        t.F = F;
        t.barrier = H;
    } else {
        const bool onN0 = (xp < k.xb[0]) && (xp > k.lo0);
        const bool onP0 = (xp < k.xc) && (xp > k.xb[0]);
        const bool onN1 = (xp < k.xb[1]) && (xp > k.xc);
        const bool onP1 = (xp < k.hi1) && (xp > k.xb[1]);
        double E = 0.0, f = 0.0, B = 0.0;
        if (onN0) { E = xp * k.sN[0][s] + k.iN[0][s]; f = k.sN[0][s]; B = k.Hd[0][s]; }
        if (onP0) { E = xp * k.sP[0][s] + k.iP[0][s]; f = k.sP[0][s]; B = k.Hd[0][s]; }
        if (onN1) { E = xp * k.sN[1][s] + k.iN[1][s]; f = k.sN[1][s]; B = k.Hd[1][s]; }
        if (onP1) { E = xp * k.sP[1][s] + k.iP[1][s]; f = k.sP[1][s]; B = k.Hd[1][s]; }
        t.E = E;
        t.F = 0.0 - f;
        t.barrier = B;
    }
}

// InitializePeriodicIndices / UpdatePeriodicIndices, S.h:1838-1884,
// D.h:2156-2235: well = floor(x/L), cell = rint(x/L) (ties to even),
// local barrier = (xp < xc) ? 0 : 1.
template <bool DBL>
__device__ __forceinline__ void indices(const KConst& k, T64& t) {
    const double red = t.x * k.invL;
    t.well = (int64_t)floor(red);
    t.cell = (int64_t)rint(red);
    if (DBL) {
        const double xp = t.x - (double)t.cell * k.L;
        t.lb = (xp < k.xc) ? 0 : 1;
    } else {
        t.lb = 0;
    }
}

template <bool DBL>
__device__ __forceinline__ int table_state(const KConst& k, const TrajState& st, int64_t i, uint32_t g,
                                           int64_t cell) {
    int s;
    int64_t nf;
    bool found;
    ring_load<DBL>(k, st, i, g, cell_key<DBL>(cell, 0), &s, &nf, &found);
    return s;
}

// Initial-barrier bookkeeping of the FPT statistic, S.h:2187-2211 and
// S.h:2364-2388; the two recorded states live in bits B_INIT0/B_INIT1.
template <bool DBL>
__device__ __forceinline__ void fpt_set_initial(const KConst& k, const TrajState& st, int64_t i, uint32_t g,
                                                T64& t) {
    int s0, s1;
    if (t.well == t.cell) {
        s0 = t.state;
        t.init_idx0 = t.cell;
        s1 = table_state<DBL>(k, st, i, g, t.cell + 1);
        t.init_idx1 = t.cell + 1;
    } else {
        s0 = table_state<DBL>(k, st, i, g, t.cell - 1);
        t.init_idx0 = t.cell - 1;
        s1 = t.state;
        t.init_idx1 = t.cell;
    }
    t.bits = (t.bits & ~(B_INIT0 | B_INIT1)) | (s0 ? B_INIT0 : 0u) | (s1 ? B_INIT1 : 0u);
}

__device__ __forceinline__ void fpt2_set_idx(T64& t) {
    if (t.well == t.cell) { t.idx2_0 = t.cell; t.idx2_1 = t.cell + 1; }
    else { t.idx2_0 = t.cell - 1; t.idx2_1 = t.cell; }
}

__device__ __forceinline__ bool cg_hit(int64_t well, int size) { return ((int)well % size) == 0; }

// Appends an event duration to list `list` of trajectory i (the reference's
// push_back on its per-lane vectors, S.h:2391, 2447, 2504, 2524, 2580); c is
// the list's count before the event.  A full list flags the trajectory.
__device__ __noinline__ void ev_push(const KConst& k, const TrajState& st, int list, int64_t i, int64_t c, double d,
                                     uint32_t* flags) {
    if (c < k.ev_cap) st.ev[((int64_t)list * st.n + i) * k.ev_cap + c] = d;
    else *flags |= LDP_FLAG_EVENT_OVERFLOW;
}

__device__ __forceinline__ void record(const KConst& k, const TrajState& st, const T64& t, int64_t i,
                                       int64_t frame) {
    if (frame >= k.nframe) return;   // the frame arrays hold nframe rows
    const int64_t o = frame * st.n + i;
    if (st.fx) st.fx[o] = t.x;
    if (k.write_x) {
        if (st.fv) st.fv[o] = t.v;
        if (st.ff) st.ff[o] = t.F;
        if (st.fb) st.fb[o] = t.barrier;
        if (st.fpe) st.fpe[o] = t.E;
        if (st.fke) st.fke[o] = k.mhalf * (t.v * t.v);
        if (st.fst) st.fst[o] = (double)t.state;
    }
}

__device__ __forceinline__ void store_traj(const TrajState& st, const T64& t, int64_t i) {
    st.x[i] = t.x; st.v[i] = t.v; st.F[i] = t.F; st.rprev[i] = t.rprev;
    st.cell[i] = t.cell; st.well[i] = t.well; st.state[i] = t.state; st.lb[i] = t.lb; st.bits[i] = (int32_t)t.bits;
    st.fpt_last[i] = t.fpt_last; st.fpt2_last[i] = t.fpt2_last; st.tpt_last[i] = t.tpt_last;
    st.tpt2_last[i] = t.tpt2_last;
    st.init_idx0[i] = t.init_idx0; st.init_idx1[i] = t.init_idx1; st.idx2_0[i] = t.idx2_0; st.idx2_1[i] = t.idx2_1;
    st.tpt2_well[i] = t.tpt2_well; st.wt_tick[i] = t.wt_tick;
}

__device__ __forceinline__ void load_traj(const TrajState& st, T64& t, int64_t i) {
    t.x = st.x[i]; t.v = st.v[i]; t.F = st.F[i]; t.rprev = st.rprev[i];
    t.cell = st.cell[i]; t.well = st.well[i]; t.state = st.state[i]; t.lb = st.lb[i]; t.bits = (uint32_t)st.bits[i];
    t.fpt_last = st.fpt_last[i]; t.fpt2_last = st.fpt2_last[i]; t.tpt_last = st.tpt_last[i];
    t.tpt2_last = st.tpt2_last[i];
    t.init_idx0 = st.init_idx0[i]; t.init_idx1 = st.init_idx1[i]; t.idx2_0 = st.idx2_0[i]; t.idx2_1 = st.idx2_1[i];
    t.tpt2_well = st.tpt2_well[i]; t.wt_tick = st.wt_tick[i];
    t.E = 0.0; t.barrier = 0.0;
}

// IntegrateStep0 (S.h:1619-1652, overdamped S.h:2825-2832; D.h:1938-1971)
// with InitializeBarrierState (S.h:1885-1915) and InitializeStatistics
// (S.h:2166-2333, D.h:2759-2930).
template <bool DBL, bool OVER>
__global__ void __launch_bounds__(128) fp64_init_kernel(const KConst k, const TrajState st, int64_t g0) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.n) return;
    const uint32_t g = (uint32_t)(g0 + i);
    for (int s = 0; s < k.slots; ++s) {
        st.ring_tag[(int64_t)s * st.n + i] = INT64_MIN;
        st.ring_data[(int64_t)s * st.n + i] = 0;
    }
    for (int f = 0; f < LDP_NCOUNT; ++f) st.counts[(int64_t)f * st.n + i] = 0;
    for (int f = 0; f < LDP_NSUM; ++f) st.sums[(int64_t)f * st.n + i] = 0.0;

    T64 t;
    t.x = k.x0;
    t.v = 0.0; t.F = 0.0; t.E = 0.0; t.rprev = 0.0; t.barrier = 0.0;
    t.bits = 0;
    t.fpt_last = t.fpt2_last = t.tpt_last = t.tpt2_last = 0.0;
    t.init_idx0 = t.init_idx1 = t.idx2_0 = t.idx2_1 = 0;
    t.wt_tick = 0;
    indices<DBL>(k, t);
    const Words w0 = philox_at(0, g, TAG_INIT, k.key0, k.key1);
    t.state = k.rs ? (((double)w0.w0 * 0x1p-32 <= k.p_first) ? 0 : 1) : k.init_state;
    st.state0[i] = t.state;
    st.counts[(int64_t)(t.state ? LDP_C_STATE1 : LDP_C_STATE0) * st.n + i] = 1;
    double zv, zr;
    gauss_pair_f64(w0.w1, w0.w2, &zv, &zr);
    t.v = k.rv ? k.sig_v0 * zv : k.v0;
    st.v0[i] = t.v;
    {
        // waiting time to the initial barrier's first flip
        const Words wf = philox_at(0, g, TAG_FLIP, k.key0, k.key1);
        st.nflip[i] = flip_schedule(0, wf.w0, wf.w1, k.ln1m[t.state]);
    }
    energy_force<DBL>(k, t);
    if (k.at_bottom) {
        if (!DBL && k.fpt) fpt_set_initial<DBL>(k, st, i, g, t);
        fpt2_set_idx(t);
    } else {
        t.bits |= B_FPT_UP | B_FPT2_UP;
    }
    if (!k.at_bottom) t.bits |= B_TPT_UP | B_TPT2_UP;
    t.tpt2_well = t.well;
    for (int j = 0; j < k.n_cg; ++j) {
        st.cg_last[(int64_t)j * st.n + i] = 0.0;
        st.cg_well[(int64_t)j * st.n + i] = t.well;
        if (!(k.at_bottom && cg_hit(t.well, k.cg_size[j]))) t.bits |= (B_CG0 << j);
    }
    if (OVER) t.rprev = k.sig_r * zr;
    if (!k.fp_mode) record(k, st, t, i, 0);
    store_traj(st, t, i);
}

// Where a step's flip schedule comes from.  FlipDraw draws it on the spot
// (the TAG_FLIP words at the flip step, geometric waiting time in FP64) and
// hands the words on, so that a cell entry at the same step reuses them.
struct FlipDraw {
    __device__ __forceinline__ int64_t schedule(const KConst& k, uint32_t g, uint64_t s, int state, Words* wf,
                                                bool* have) const {
        *wf = philox_at(s, g, TAG_FLIP, k.key0, k.key1);
        *have = true;
        return flip_schedule(s, wf->w0, wf->w1, k.ln1m[state]);
    }
};

// One step s of a trajectory (Integrate's loop body, S.h:1403-1511):
// IntegrateStepEta / IntegrateStep (S.h:1654-1706, 2833-2886; D.h:1973-2024,
// 3448-3505) followed by UpdateStatistics (S.h:2334-2592, D.h:2931-3209).
// z is the step's Gaussian; src supplies the flip schedule of a flip at s.
// Returns 0 to continue, 1 when the trajectory stops before completing s
// (non-finite position), 2 when it stops after s (first passage reached).
// The position (and velocity) update of a step, IntegrateStepEta's first
// part (S.h:1680-1695, 2860-2870).
template <bool OVER>
__device__ __forceinline__ void fp64_move(const KConst& k, T64& t, double z) {
    if (OVER) {
        const double rf = k.sig_r * z;
        t.x = fma(t.F, k.c_drift, t.x);
        t.x = t.x + rf;
        t.x = t.x + t.rprev;
        t.rprev = rf;
    } else {
        t.v = t.v + (k.invM * t.F) * k.hdt;
        t.x = t.x + t.v * k.hdt;
        t.v = k.expg * t.v + k.sig_v * z;
        t.x = t.x + t.v * k.hdt;
    }
}

// The rest of step s after fp64_move: indices, barrier flips and cell
// entries, the state count, the force, the statistics and the frame.
// cell_prev, well_prev, lb_prev: the indices before the move.
template <bool DBL, bool OVER, bool ETA, class Src>
__device__ __forceinline__ int fp64_after_move(const KConst& k, const TrajState& st, int64_t i, uint32_t g, T64& t,
                                               uint64_t s, const Src& src, int64_t& nflip, int64_t& sc0,
                                               int64_t& sc1, uint32_t& flags, uint64_t& nxf, int64_t cell_prev,
                                               int64_t well_prev, int lb_prev) {
    const int64_t n = st.n;
    const uint64_t fs = k.freq_save;
    if (!isfinite(t.x)) {
        flags |= LDP_FLAG_NONFINITE;
        t.bits |= B_DONE;
        return 1;
    }
    indices<DBL>(k, t);
    const bool dWell = t.well != well_prev;
    const bool dCell = t.cell != cell_prev;
    const bool dKey = DBL ? (t.lb != lb_prev) : dCell;

    if (ETA) {
        // UpdateBarrierStateEta, S.h:1998-2153 / D.h:2435-2736, with
        // every barrier's flips on a schedule (geometric waiting times of
        // the per-step Bernoulli flips): the current barrier flips at its
        // pending flip step; a barrier left keeps its pending flip in the
        // cell table; one re-entered before that step has not flipped
        // meanwhile (no draw); one whose flip came while it was away (or
        // never visited: created at step 0) is caught up from that step
        // with the two-state transition probability (S.h:2025-2068).
        const bool flip = (int64_t)s == nflip;
        Words wf{};
        bool have_wf = false;
        if (flip) {
            t.state ^= 1;
            nflip = src.schedule(k, g, s, t.state, &wf, &have_wf);
        }
        if (dKey) {
            ring_store(k, st, i, cell_key<DBL>(cell_prev, lb_prev), t.state, nflip);
            int ps;
            int64_t nb;
            bool found;
            ring_load<DBL>(k, st, i, g, cell_key<DBL>(t.cell, t.lb), &ps, &nb, &found);
            if (found && nb > (int64_t)s) {
                t.state = ps;
                nflip = nb;
            } else {
                const int64_t base = found ? nb : 0;
                const int sb = found ? (ps ^ 1) : ps;
                const double lap = (double)((int64_t)s - base);
                const double pl = k.c_lap[k.eq ? 0 : sb] * -expm1_f64(k.a_lap * lap);
                const uint64_t Tl = prob_to_u64(pl);
                const Words wc = philox_at(s, g, TAG_CATCHUP, k.key0, k.key1);
                const uint64_t U = ((uint64_t)wc.w0 << 32) | wc.w1;
                t.state = (U < Tl) ? (sb ^ 1) : sb;
                if (!have_wf) wf = philox_at(s, g, TAG_FLIP, k.key0, k.key1);
                nflip = flip_schedule(s, wf.w2, wf.w3, k.ln1m[t.state]);
            }
        }
    } else {
        // UpdateBarrierState (TAU == 0), S.h:1933-1997 / D.h:2299-2434.
        if (dKey) {
            ring_store(k, st, i, cell_key<DBL>(cell_prev, lb_prev), t.state, nflip);
            int ps;
            int64_t nb;
            bool found;
            ring_load<DBL>(k, st, i, g, cell_key<DBL>(t.cell, t.lb), &ps, &nb, &found);
            t.state = ps;
        }
    }
    if (t.state) ++sc1; else ++sc0;   // UpdateBarrierStateEtaParamter
    energy_force<DBL>(k, t);
    if (!OVER) t.v = t.v + (k.invM * t.F) * k.hdt;

    // UpdateStatistics.
    if (dWell || dCell) {
        const double now = k.dt * (double)s;
        if (!DBL && k.wt && !k.fp_mode) {
            if (dWell) { t.wt_tick = (int64_t)s; t.bits |= B_WT_PASSED; }
            else if (dCell && (t.bits & B_WT_PASSED)) {
                int64_t& nwt = st.counts[(int64_t)LDP_C_WT * n + i];
                if (nwt < k.tick_cap) st.ticks[i * k.tick_cap + nwt] = t.wt_tick;
                else flags |= LDP_FLAG_TICK_OVERFLOW;
                nwt += 1;
                t.bits &= ~B_WT_PASSED;
            }
        }
        if (k.fpt || k.fp_mode) {
            if (!DBL && !k.fp_mode) {
                if ((t.bits & B_FPT_UP) && dCell) {
                    t.bits &= ~B_FPT_UP;
                    t.fpt_last = now;
                    fpt_set_initial<DBL>(k, st, i, g, t);
                }
                if (!(t.bits & B_FPT_UP) && dWell) {
                    t.bits |= B_FPT_UP;
                    const int64_t c = st.counts[(int64_t)LDP_C_FPT * n + i];
                    if (c == 0) st.sums[(int64_t)LDP_S_FIRST_FPT * n + i] = now - t.fpt_last;
                    st.sums[(int64_t)LDP_S_FPT * n + i] += now - t.fpt_last;
                    st.counts[(int64_t)LDP_C_FPT * n + i] = c + 1;
                    const bool ib = ((double)t.cell == (double)t.init_idx0) ? ((t.bits & B_INIT0) != 0)
                                                                            : ((t.bits & B_INIT1) != 0);
                    if (k.ev_cap) {
                        ev_push(k, st, LDP_E_FPT, i, c, now - t.fpt_last, &flags);
                        if (c < k.ev_cap) st.ev_st[i * k.ev_cap + c] = (uint8_t)((t.state ? 1 : 0) | (ib ? 2 : 0));
                    }
                    st.counts[(int64_t)(ib ? LDP_C_INIT1 : LDP_C_INIT0) * n + i] += 1;
                    st.counts[(int64_t)(t.state ? LDP_C_INST1 : LDP_C_INST0) * n + i] += 1;
                }
            }
            if ((t.bits & B_FPT2_UP) && dCell) {
                t.bits &= ~B_FPT2_UP;
                t.fpt2_last = now;
                fpt2_set_idx(t);
            }
            if (dCell && !(t.bits & B_FPT2_UP) && t.idx2_0 != t.cell && t.idx2_1 != t.cell) {
                const int64_t c = st.counts[(int64_t)LDP_C_FPT2 * n + i];
                if (c == 0) st.sums[(int64_t)LDP_S_FIRST_FPT2 * n + i] = now - t.fpt2_last;
                st.sums[(int64_t)LDP_S_FPT2 * n + i] += now - t.fpt2_last;
                st.counts[(int64_t)LDP_C_FPT2 * n + i] = c + 1;
                if (k.ev_cap) ev_push(k, st, LDP_E_FPT2, i, c, now - t.fpt2_last, &flags);
                t.fpt2_last = now;
                fpt2_set_idx(t);
                if (k.fp_mode) t.bits |= B_DONE;   // first passage reached
            }
        }
        if (!DBL && k.tpt && !k.fp_mode) {
            if (dCell) { t.bits &= ~B_TPT_UP; t.tpt_last = now; }
            if (!(t.bits & B_TPT_UP) && dWell) {
                t.bits |= B_TPT_UP;
                const int64_t c = st.counts[(int64_t)LDP_C_TPT * n + i];
                if (c == 0) st.sums[(int64_t)LDP_S_FIRST_TPT * n + i] = now - t.tpt_last;
                st.sums[(int64_t)LDP_S_TPT * n + i] += now - t.tpt_last;
                st.counts[(int64_t)LDP_C_TPT * n + i] = c + 1;
                if (k.ev_cap) ev_push(k, st, LDP_E_TPT, i, c, now - t.tpt_last, &flags);
            }
            if (dCell) {
                if (t.bits & B_TPT2_UP) t.bits &= ~B_TPT2_UP;
                else if (t.well != t.tpt2_well) {
                    const int64_t c = st.counts[(int64_t)LDP_C_TPT2 * n + i];
                    if (c == 0) st.sums[(int64_t)LDP_S_FIRST_TPT2 * n + i] = now - t.tpt2_last;
                    st.sums[(int64_t)LDP_S_TPT2 * n + i] += now - t.tpt2_last;
                    st.counts[(int64_t)LDP_C_TPT2 * n + i] = c + 1;
                    if (k.ev_cap) ev_push(k, st, LDP_E_TPT2, i, c, now - t.tpt2_last, &flags);
                }
                t.tpt2_last = now;
                t.tpt2_well = t.well;
            }
        }
        if (k.cg && !k.fp_mode && dCell) {
            for (int jj = 0; jj < k.n_cg; ++jj) {
                if (cg_hit(t.well, k.cg_size[jj])) {
                    const int64_t o = (int64_t)jj * n + i;
                    if (t.bits & (B_CG0 << jj)) {
                        t.bits &= ~(B_CG0 << jj);
                        st.cg_last[o] = now;
                        st.cg_well[o] = t.well;
                    } else if (t.well != st.cg_well[o]) {
                        st.sums[(int64_t)(LDP_S_CG0 + jj) * n + i] += now - st.cg_last[o];
                        const int64_t c = st.counts[(int64_t)(LDP_C_CG0 + jj) * n + i];
                        st.counts[(int64_t)(LDP_C_CG0 + jj) * n + i] = c + 1;
                        if (k.ev_cap) ev_push(k, st, LDP_E_CG0 + jj, i, c, now - st.cg_last[o], &flags);
                        st.cg_last[o] = now;
                        st.cg_well[o] = t.well;
                    }
                }
            }
        }
    }
    if (!k.fp_mode && s == nxf) {
        record(k, st, t, i, (int64_t)(s / fs));
        nxf += fs;
    }
    if (t.bits & B_DONE) return 2;
    return 0;
}

template <bool DBL, bool OVER, bool ETA, class Src>
__device__ __forceinline__ int fp64_step(const KConst& k, const TrajState& st, int64_t i, uint32_t g, T64& t,
                                         uint64_t s, double z, const Src& src, int64_t& nflip, int64_t& sc0,
                                         int64_t& sc1, uint32_t& flags, uint64_t& nxf) {
    const int64_t cell_prev = t.cell, well_prev = t.well;
    const int lb_prev = t.lb;
    fp64_move<OVER>(k, t, z);
    return fp64_after_move<DBL, OVER, ETA>(k, st, i, g, t, s, src, nflip, sc0, sc1, flags, nxf, cell_prev, well_prev,
                                           lb_prev);
}

// The open interval of positions (absolute x) in which a step cannot change
// the cell, the well, the local barrier or the force: the interval between
// the breakpoints of energy_force (and indices) around the current
// cell-local position -- the cell edges, the barrier top 0, the flanks --
// shrunk at both ends by a margin, 1e-9 (1 + |x|), far above the rounding of
// x * invL and x - cell * L (~2e-16 |x|), so that for x inside it the full
// step would compute the same indices and force.  Empty (lo > hi) when x is
// within the margin of a breakpoint.
template <bool DBL>
__device__ __forceinline__ void quiet_band(const KConst& k, const T64& t, double* lo, double* hi) {
    const double cL = (double)t.cell * k.L;
    const double xp = t.x - cL;
    const double hL = 0.5 * k.L;
    double l = -hL, h = hL;
    auto cut = [&](double b) {
        if (b > -hL && b < hL) {
            if (b <= xp) l = fmax(l, b);
            if (b >= xp) h = fmin(h, b);
        }
    };
    cut(0.0);
    if (!DBL) {
        cut(0.0 - k.w);
        cut(k.w);
    } else {
        cut(k.lo0);
        cut(k.xb[0]);
        cut(k.xc);
        cut(k.xb[1]);
        cut(k.hi1);
    }
    const double m = 1e-9 * (1.0 + fabs(cL) + fabs(t.x));
    *lo = cL + l + m;
    *hi = cL + h - m;
}

// The force energy_force gives at the current position for either barrier
// state (constant over the quiet band).
template <bool DBL>
__device__ __forceinline__ void band_forces(const KConst& k, const T64& t, double* f0, double* f1) {
    T64 a = t;
    a.state = 0;
    energy_force<DBL>(k, a);
    *f0 = a.F;
    a.state = 1;
    energy_force<DBL>(k, a);
    *f1 = a.F;
}

// Steps s_begin .. s_end-1 of the hot loop, one trajectory per thread, each
// drawing its own Gaussians (one Philox block per four steps) and flips.
template <bool DBL, bool OVER, bool ETA>
__global__ void __launch_bounds__(128, 4) fp64_steps_kernel(const KConst k, const TrajState st, int64_t g0,
                                                         uint64_t s_begin, uint64_t s_end) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= st.n) return;
    const uint32_t g = (uint32_t)(g0 + i);
    T64 t;
    load_traj(st, t, i);
    if (t.bits & B_DONE) return;
    const int64_t n = st.n;
    int64_t sc0 = st.counts[(int64_t)LDP_C_STATE0 * n + i];
    int64_t sc1 = st.counts[(int64_t)LDP_C_STATE1 * n + i];
    // Force at the current position (not stored between launches).
    energy_force<DBL>(k, t);
    int64_t nflip = st.nflip[i];
    uint32_t flags = 0;
    uint64_t s = s_begin;
    const uint64_t fs = k.freq_save;
    // Next frame step (a multiple of FREQSAVE), so that no step divides.
    uint64_t nxf = (s_begin + fs - 1) / fs * fs;
    // One Philox block serves steps 4a+1 .. 4a+4: words 0,1 the first
    // Gaussian pair, words 2,3 (kept) the second.
    double za = 0, zb = 0;
    uint32_t wc2 = 0, wc3 = 0;
    const FlipDraw src;
    // quiet band (empty: the first step takes the full path) and the force
    // in it for either barrier state
    double blo = 1.0, bhi = 0.0, bF0 = 0.0, bF1 = 0.0;
    for (; s < s_end; ++s) {
        const int q = (int)((s - 1) & 3);
        if (q == 0 || s == s_begin) {
            const Words w = philox_at((s - 1) >> 2, g, TAG_STEP, k.key0, k.key1);
            wc2 = w.w2;
            wc3 = w.w3;
            if (q < 2) gauss_pair_f64(w.w0, w.w1, &za, &zb);
            else gauss_pair_f64(w.w2, w.w3, &za, &zb);
        } else if (q == 2) {
            gauss_pair_f64(wc2, wc3, &za, &zb);
        }
        const double z = (q & 1) ? zb : za;
        const int64_t cell_prev = t.cell, well_prev = t.well;
        const int lb_prev = t.lb;
        fp64_move<OVER>(k, t, z);
        if (t.x > blo && t.x < bhi && (int64_t)s != (int64_t)nxf) {
            // a quiet step (see quiet_band): same indices, no frame, no
            // event; a flip draws its schedule and takes the band's force
            if (ETA && (int64_t)s == nflip) {
                t.state ^= 1;
                Words wf;
                bool have = false;
                nflip = src.schedule(k, g, s, t.state, &wf, &have);
                t.F = t.state ? bF1 : bF0;
            }
            if (t.state) ++sc1; else ++sc0;
            if (!OVER) t.v = t.v + (k.invM * t.F) * k.hdt;
            continue;
        }
        const int r = fp64_after_move<DBL, OVER, ETA>(k, st, i, g, t, s, src, nflip, sc0, sc1, flags, nxf, cell_prev,
                                                      well_prev, lb_prev);
        if (r == 1) break;
        if (r == 2) { ++s; break; }
        quiet_band<DBL>(k, t, &blo, &bhi);
        band_forces<DBL>(k, t, &bF0, &bF1);
    }
    // s is the first step not integrated.
    st.counts[(int64_t)LDP_C_STATE0 * n + i] = sc0;
    st.counts[(int64_t)LDP_C_STATE1 * n + i] = sc1;
    st.counts[(int64_t)LDP_C_STEPS * n + i] = (int64_t)s - 1;
    if (k.fp_mode && !(t.bits & B_DONE) && s_end > k.step_cap) flags |= LDP_FLAG_CENSORED;
    if (flags) st.counts[(int64_t)LDP_C_FLAGS * n + i] |= (int64_t)flags;
    st.nflip[i] = nflip;
    store_traj(st, t, i);
}

// ---------------------------------------------------------------------------
// Latency mode: few long trajectories (the reference's own sample runs 16-32
// trajectories for 3e9 steps).  One trajectory per thread leaves a step's
// whole dependency chain -- Philox rounds, the FP64 logarithm and sincos of
// Box-Muller, the flip's logarithm and division -- on one thread, ~1800
// cycles per step.  Here a trajectory gets a CTA of two warps:
//  * the producer warp computes, for a block of 32 steps, lane l the inputs
//    of step s0 + l that do not depend on the position: its Gaussian (the
//    same Philox block and Box-Muller pair the thread-per-trajectory kernel
//    uses) and, when barriers flip, the flip schedule a flip at that step
//    would give for either new state (its TAG_FLIP words, one logarithm,
//    the two geometric waiting times);
//  * lane 0 of the consumer warp runs the steps with fp64_step, taking those
//    inputs from shared memory, so its chain is the position update,
//    indices, flip selection and force.
// Two buffers of 32 steps alternate; named barriers 1-2 ("full") and 3-4
// ("empty") hand them over, every arrival matched by one wait (the producer
// waits for the last two buffers' release before it exits).  Every input is
// the same FP64 value, so results equal the thread-per-trajectory kernel's
// (and the oracle's) bit for bit.
// ---------------------------------------------------------------------------
constexpr int kLatBlock = 32;   // steps per buffer

constexpr int kLatSub = 8;       // steps per speculative sub-block (see the consumer)
struct LatBuf {
    double z[2][kLatBlock];
    int64_t cand[2][2][kLatBlock];   // [buffer][new state][step]
};

// The flip schedule of a flip at step s for both new states, from the words
// (hi, lo) of TAG_FLIP at s: flip_schedule of either state, with the
// logarithm evaluated once.
__device__ __forceinline__ void flip_schedule_both(uint64_t s, uint32_t hi, uint32_t lo, const double ln1m[2],
                                                   int64_t* c0, int64_t* c1) {
    const double u = ((double)(((uint64_t)hi << 32) | lo) + 1.0) * 0x1p-64;
    const double lu = log_f64(u);
    int64_t c[2];
#pragma unroll
    for (int st = 0; st < 2; ++st) {
        uint64_t wt = 0xffffffffffffffffull;
        if (ln1m[st] < 0.0) {
            const double q = lu / ln1m[st];
            if (q < 0x1p62) wt = 1ull + (uint64_t)floor(q);
        }
        c[st] = (wt >= (uint64_t)kNeverFlip - s) ? kNeverFlip : (int64_t)(s + wt);
    }
    *c0 = c[0];
    *c1 = c[1];
}

// The consumer's flip schedule source: the producer's candidates for step s.
struct FlipFromBuffer {
    const int64_t* c0;
    const int64_t* c1;
    __device__ __forceinline__ int64_t schedule(const KConst&, uint32_t, uint64_t, int state, Words*, bool*) const {
        return state ? *c1 : *c0;
    }
};

__device__ __forceinline__ void named_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void named_arrive(int id) { asm volatile("bar.arrive %0, 64;" ::"r"(id) : "memory"); }

template <bool DBL, bool OVER, bool ETA>
__global__ void __launch_bounds__(64, 4) fp64_latency_kernel(const KConst k, const TrajState st, int64_t g0,
                                                          uint64_t s_begin, uint64_t s_end) {
    __shared__ LatBuf buf;
    const int64_t i = blockIdx.x;
    if (i >= st.n) return;   // whole CTA: no barrier is reached
    const uint32_t g = (uint32_t)(g0 + i);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t nblk = (s_end > s_begin) ? (s_end - s_begin + kLatBlock - 1) / kLatBlock : 0;
    if (warp == 1) {
        // ---- producer ----
        for (uint64_t b = 0; b < nblk; ++b) {
            const int u = (int)(b & 1);
            if (b >= 2) named_sync(3 + u);   // buffer u released by the consumer
            const uint64_t s = s_begin + b * kLatBlock + (uint64_t)lane;
            if (s < s_end) {
                const int q = (int)((s - 1) & 3);
                const Words w = philox_at((s - 1) >> 2, g, TAG_STEP, k.key0, k.key1);
                double za, zb;
                if (q < 2) gauss_pair_f64(w.w0, w.w1, &za, &zb);
                else gauss_pair_f64(w.w2, w.w3, &za, &zb);
                buf.z[u][lane] = (q & 1) ? zb : za;
                if (ETA) {
                    const Words wf = philox_at(s, g, TAG_FLIP, k.key0, k.key1);
                    flip_schedule_both(s, wf.w0, wf.w1, k.ln1m, &buf.cand[u][0][lane], &buf.cand[u][1][lane]);
                }
            }
            __syncwarp();
            named_arrive(1 + u);             // buffer u full
        }
        // the consumer's release of the last two buffers
        for (uint64_t b = (nblk > 2 ? nblk - 2 : 0); b < nblk; ++b) named_sync(3 + (int)(b & 1));
        return;
    }
    // ---- consumer ----
    T64 t;
    int64_t sc0 = 0, sc1 = 0, nflip = 0;
    uint32_t flags = 0;
    uint64_t s = s_begin, nxf = 0;
    bool run = false, active = false;
    // quiet band (empty: the first step takes the full path) and the force
    // in it for either barrier state
    double blo = 1.0, bhi = 0.0, bF0 = 0.0, bF1 = 0.0;
    if (lane == 0) {
        load_traj(st, t, i);
        active = run = !(t.bits & B_DONE);
        sc0 = st.counts[(int64_t)LDP_C_STATE0 * st.n + i];
        sc1 = st.counts[(int64_t)LDP_C_STATE1 * st.n + i];
        energy_force<DBL>(k, t);
        nflip = st.nflip[i];
        const uint64_t fs = k.freq_save;
        nxf = (s_begin + fs - 1) / fs * fs;
    }
    for (uint64_t b = 0; b < nblk; ++b) {
        const int u = (int)(b & 1);
        named_sync(1 + u);                   // buffer u full
        if (lane == 0 && run) {
            const uint64_t s1 = (s_begin + (b + 1) * kLatBlock < s_end) ? s_begin + (b + 1) * kLatBlock : s_end;
            const int nl = (int)(s1 - s);
            // the next step's Gaussian and flip schedules are loaded one step
            // ahead, so their shared-memory latency is off the chain (zn,
            // cn0, cn1 hold step pf's)
            double zn = buf.z[u][0];
            int64_t cn0 = 0, cn1 = 0;
            if (ETA) {
                cn0 = buf.cand[u][0][0];
                cn1 = buf.cand[u][1][0];
            }
            int pf = 0;
            for (int l = 0; l < nl;) {
                // Speculative sub-block: the next kLatSub steps run as quiet
                // steps without the per-step band test, keeping the lowest
                // and highest position; when every position stayed inside
                // the quiet band (and no frame falls in the sub-block) they
                // were quiet steps and stand, else the state at the
                // sub-block's start is restored and the steps run one by one.
                // x turning NaN stays NaN to the end, which the final test
                // catches.
                if (l + kLatSub <= nl && (l & (kLatSub - 1)) == 0 && (int64_t)nxf >= (int64_t)s + kLatSub &&
                    t.x > blo && t.x < bhi) {
                    double zb[kLatSub];
                    int64_t c0b[kLatSub], c1b[kLatSub];
#pragma unroll
                    for (int m = 0; m < kLatSub; ++m) {
                        zb[m] = buf.z[u][l + m];
                        if (ETA) {
                            c0b[m] = buf.cand[u][0][l + m];
                            c1b[m] = buf.cand[u][1][l + m];
                        }
                    }
                    const double x0 = t.x, v0 = t.v, F0 = t.F, r0 = t.rprev;
                    const int st0 = t.state;
                    const int64_t nflip0 = nflip;
                    int n1 = 0;
                    double xmin = t.x, xmax = t.x;
#pragma unroll
                    for (int m = 0; m < kLatSub; ++m) {
                        fp64_move<OVER>(k, t, zb[m]);
                        xmin = fmin(xmin, t.x);
                        xmax = fmax(xmax, t.x);
                        if (ETA) {
                            // flips by selects (t.F is the band's force of
                            // the state throughout), so the steps form one
                            // chain in x
                            const bool f = (int64_t)s + m == nflip;
                            t.state ^= (int)f;
                            const int64_t cn = t.state ? c1b[m] : c0b[m];
                            nflip = f ? cn : nflip;
                            t.F = t.state ? bF1 : bF0;
                        }
                        n1 += t.state;
                        if (!OVER) t.v = t.v + (k.invM * t.F) * k.hdt;
                    }
                    if (xmin > blo && xmax < bhi && t.x > blo) {
                        sc1 += n1;
                        sc0 += kLatSub - n1;
                        s += kLatSub;
                        l += kLatSub;
                        continue;
                    }
                    t.x = x0;
                    t.v = v0;
                    t.F = F0;
                    t.rprev = r0;
                    t.state = st0;
                    nflip = nflip0;
                }
                double z;
                int64_t ca0 = 0, ca1 = 0;
                if (pf == l) {
                    z = zn;
                    ca0 = cn0;
                    ca1 = cn1;
                } else {
                    z = buf.z[u][l];
                    if (ETA) {
                        ca0 = buf.cand[u][0][l];
                        ca1 = buf.cand[u][1][l];
                    }
                }
                if (l + 1 < nl) {
                    zn = buf.z[u][l + 1];
                    if (ETA) {
                        cn0 = buf.cand[u][0][l + 1];
                        cn1 = buf.cand[u][1][l + 1];
                    }
                    pf = l + 1;
                }
                const int64_t cell_prev = t.cell, well_prev = t.well;
                const int lb_prev = t.lb;
                fp64_move<OVER>(k, t, z);
                if (t.x > blo && t.x < bhi && (int64_t)s != (int64_t)nxf) {
                    // a quiet step: same indices, no frame, no event; a flip
                    // toggles the state, takes its new schedule and the
                    // band's force for that state (the rest of the full step)
                    if (ETA && (int64_t)s == nflip) {
                        t.state ^= 1;
                        nflip = t.state ? ca1 : ca0;
                        t.F = t.state ? bF1 : bF0;
                    }
                    if (t.state) ++sc1; else ++sc0;
                    if (!OVER) t.v = t.v + (k.invM * t.F) * k.hdt;
                    ++s;
                    ++l;
                    continue;
                }
                const FlipFromBuffer src{&buf.cand[u][0][l], &buf.cand[u][1][l]};
                const int r = fp64_after_move<DBL, OVER, ETA>(k, st, i, g, t, s, src, nflip, sc0, sc1, flags, nxf,
                                                              cell_prev, well_prev, lb_prev);
                if (r == 1) { run = false; break; }
                if (r == 2) { ++s; run = false; break; }
                quiet_band<DBL>(k, t, &blo, &bhi);
                band_forces<DBL>(k, t, &bF0, &bF1);
                ++s;
                ++l;
            }
        }
        __syncwarp();
        named_arrive(3 + u);                 // buffer u released
    }
    if (lane != 0 || !active) return;   // a trajectory done before the launch keeps its state
    // s is the first step not integrated
    const int64_t n = st.n;
    st.counts[(int64_t)LDP_C_STATE0 * n + i] = sc0;
    st.counts[(int64_t)LDP_C_STATE1 * n + i] = sc1;
    st.counts[(int64_t)LDP_C_STEPS * n + i] = (int64_t)s - 1;
    if (k.fp_mode && !(t.bits & B_DONE) && s_end > k.step_cap) flags |= LDP_FLAG_CENSORED;
    if (flags) st.counts[(int64_t)LDP_C_FLAGS * n + i] |= (int64_t)flags;
    st.nflip[i] = nflip;
    store_traj(st, t, i);
}

// ---------------------------------------------------------------------------
// Group mode: mid-size runs (a few thousand trajectories).  Latency mode
// gives each trajectory a CTA and saturates near 7e9 particle-steps/s; one
// trajectory per thread leaves a few warps per SM, each waiting on its own
// draws.  Here a CTA runs 32 trajectories: a consumer warp, lane l the
// trajectory 32 blockIdx + l, steps them with latency mode's consumer code
// (quiet steps, speculative sub-blocks, full steps through fp64_after_move),
// and P producer warps draw their Gaussians and flip schedules for the
// next 4 P steps into shared memory (producer lane p: the trajectory p mod
// 32, the four consecutive steps 4 (p / 32) .. 4 (p / 32) + 3 of the block,
// one Philox block and two Box-Muller pairs for them when the block starts
// on a Philox block).  Two buffers alternate, handed over with named
// barriers 5-6 ("full") and 7-8 ("empty") over all the CTA's warps; every
// arrival is matched by one wait, with no spin loop.  Same inputs, same operations:
// results equal the other kernels' and the oracle's bit for bit.
// ---------------------------------------------------------------------------
// P producer warps per CTA, 4 P steps per buffer (four consecutive steps
// per producer lane); P = 4 up to kGrpWideMin trajectories, P = 2 above
// (fewer warps per group, more groups per SM).
constexpr int64_t kGrpWideMin = 8192;
template <int P>
struct GrpBuf {
    double z[2][4 * P][32];          // [buffer][step][trajectory]
    int64_t cand[2][2][4 * P][32];   // [buffer][new state][step][trajectory]
};

template <int P>
__device__ __forceinline__ void grp_sync(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(32 * (1 + P)) : "memory");
}
template <int P>
__device__ __forceinline__ void grp_arrive(int id) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "n"(32 * (1 + P)) : "memory");
}

template <bool DBL, bool OVER, bool ETA, int P>
__global__ void __launch_bounds__(32 * (1 + P), 2) fp64_group_kernel(const KConst k, const TrajState st, int64_t g0,
                                                                     uint64_t s_begin, uint64_t s_end) {
    constexpr int kGrpBlock = 4 * P, kGrpProducers = P;
    __shared__ GrpBuf<P> buf;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t nblk = (s_end > s_begin) ? (s_end - s_begin + kGrpBlock - 1) / kGrpBlock : 0;
    if (warp >= 1) {
        // ---- producers ----
        const int p = (warp - 1) * 32 + lane;
        const int tl = p & 31;               // the trajectory's lane
        const int e0 = (p >> 5) * (kGrpBlock / kGrpProducers);   // its steps e0 .. e0 + 3 of each block
        const int64_t ip = (int64_t)blockIdx.x * 32 + tl;
        const uint32_t g = (uint32_t)(g0 + ip);
        // the last Philox block's four Gaussians (a block serves four steps;
        // a lane's four steps share one when the block start is aligned)
        uint64_t aq = ~0ull;
        double z0 = 0.0, z1 = 0.0, z2 = 0.0, z3 = 0.0;
        for (uint64_t b = 0; b < nblk; ++b) {
            const int u = (int)(b & 1);
            if (b >= 2) grp_sync<P>(7 + u);     // buffer u released by the consumer
            for (int e = e0; e < e0 + kGrpBlock / kGrpProducers; ++e) {
                const uint64_t s = s_begin + b * kGrpBlock + (uint64_t)e;
                if (ip >= st.n || s >= s_end) continue;
                const uint64_t a = (s - 1) >> 2;
                if (a != aq) {
                    const Words w = philox_at(a, g, TAG_STEP, k.key0, k.key1);
                    gauss_pair_f64(w.w0, w.w1, &z0, &z1);
                    gauss_pair_f64(w.w2, w.w3, &z2, &z3);
                    aq = a;
                }
                const int q = (int)((s - 1) & 3);
                buf.z[u][e][tl] = (q == 0) ? z0 : (q == 1) ? z1 : (q == 2) ? z2 : z3;
                if (ETA) {
                    const Words wf = philox_at(s, g, TAG_FLIP, k.key0, k.key1);
                    flip_schedule_both(s, wf.w0, wf.w1, k.ln1m, &buf.cand[u][0][e][tl], &buf.cand[u][1][e][tl]);
                }
            }
            __syncwarp();
            grp_arrive<P>(5 + u);               // buffer u full
        }
        // the consumer's release of the last two buffers
        for (uint64_t b = (nblk > 2 ? nblk - 2 : 0); b < nblk; ++b) grp_sync<P>(7 + (int)(b & 1));
        return;
    }
    // ---- consumer: lane l runs trajectory 32 blockIdx + l ----
    const int64_t i = (int64_t)blockIdx.x * 32 + lane;
    const uint32_t g = (uint32_t)(g0 + i);
    T64 t;
    int64_t sc0 = 0, sc1 = 0, nflip = 0;
    uint32_t flags = 0;
    uint64_t s = s_begin, nxf = 0;
    bool run = false, active = false;
    // quiet band (empty: the first step takes the full path) and the force
    // in it for either barrier state
    double blo = 1.0, bhi = 0.0, bF0 = 0.0, bF1 = 0.0;
    if (i < st.n) {
        load_traj(st, t, i);
        active = run = !(t.bits & B_DONE);
        sc0 = st.counts[(int64_t)LDP_C_STATE0 * st.n + i];
        sc1 = st.counts[(int64_t)LDP_C_STATE1 * st.n + i];
        energy_force<DBL>(k, t);
        nflip = st.nflip[i];
        const uint64_t fs = k.freq_save;
        nxf = (s_begin + fs - 1) / fs * fs;
    }
    for (uint64_t b = 0; b < nblk; ++b) {
        const int u = (int)(b & 1);
        grp_sync<P>(5 + u);                     // buffer u full
        if (run) {
            const uint64_t s1 = (s_begin + (b + 1) * kGrpBlock < s_end) ? s_begin + (b + 1) * kGrpBlock : s_end;
            const int nl = (int)(s1 - s);
            // the next step's Gaussian and flip schedules are loaded one step
            // ahead, so their shared-memory latency is off the chain (zn,
            // cn0, cn1 hold step pf's)
            double zn = buf.z[u][0][lane];
            int64_t cn0 = 0, cn1 = 0;
            if (ETA) {
                cn0 = buf.cand[u][0][0][lane];
                cn1 = buf.cand[u][1][0][lane];
            }
            int pf = 0;
            for (int l = 0; l < nl;) {
                // Speculative sub-block: the next kLatSub steps run as quiet
                // steps without the per-step band test, keeping the lowest
                // and highest position; when every position stayed inside
                // the quiet band (and no frame falls in the sub-block) they
                // were quiet steps and stand, else the state at the
                // sub-block's start is restored and the steps run one by one.
                // x turning NaN stays NaN to the end, which the final test
                // catches.
                if (l + kLatSub <= nl && (l & (kLatSub - 1)) == 0 && (int64_t)nxf >= (int64_t)s + kLatSub &&
                    t.x > blo && t.x < bhi) {
                    double zb[kLatSub];
                    int64_t c0b[kLatSub], c1b[kLatSub];
#pragma unroll
                    for (int m = 0; m < kLatSub; ++m) {
                        zb[m] = buf.z[u][l + m][lane];
                        if (ETA) {
                            c0b[m] = buf.cand[u][0][l + m][lane];
                            c1b[m] = buf.cand[u][1][l + m][lane];
                        }
                    }
                    const double x0 = t.x, v0 = t.v, F0 = t.F, r0 = t.rprev;
                    const int st0 = t.state;
                    const int64_t nflip0 = nflip;
                    int n1 = 0;
                    double xmin = t.x, xmax = t.x;
#pragma unroll
                    for (int m = 0; m < kLatSub; ++m) {
                        fp64_move<OVER>(k, t, zb[m]);
                        xmin = fmin(xmin, t.x);
                        xmax = fmax(xmax, t.x);
                        if (ETA) {
                            // flips by selects (t.F is the band's force of
                            // the state throughout), so the steps form one
                            // chain in x
                            const bool f = (int64_t)s + m == nflip;
                            t.state ^= (int)f;
                            const int64_t cn = t.state ? c1b[m] : c0b[m];
                            nflip = f ? cn : nflip;
                            t.F = t.state ? bF1 : bF0;
                        }
                        n1 += t.state;
                        if (!OVER) t.v = t.v + (k.invM * t.F) * k.hdt;
                    }
                    if (xmin > blo && xmax < bhi && t.x > blo) {
                        sc1 += n1;
                        sc0 += kLatSub - n1;
                        s += kLatSub;
                        l += kLatSub;
                        continue;
                    }
                    t.x = x0;
                    t.v = v0;
                    t.F = F0;
                    t.rprev = r0;
                    t.state = st0;
                    nflip = nflip0;
                }
                double z;
                int64_t ca0 = 0, ca1 = 0;
                if (pf == l) {
                    z = zn;
                    ca0 = cn0;
                    ca1 = cn1;
                } else {
                    z = buf.z[u][l][lane];
                    if (ETA) {
                        ca0 = buf.cand[u][0][l][lane];
                        ca1 = buf.cand[u][1][l][lane];
                    }
                }
                if (l + 1 < nl) {
                    zn = buf.z[u][l + 1][lane];
                    if (ETA) {
                        cn0 = buf.cand[u][0][l + 1][lane];
                        cn1 = buf.cand[u][1][l + 1][lane];
                    }
                    pf = l + 1;
                }
                const int64_t cell_prev = t.cell, well_prev = t.well;
                const int lb_prev = t.lb;
                fp64_move<OVER>(k, t, z);
                if (t.x > blo && t.x < bhi && (int64_t)s != (int64_t)nxf) {
                    // a quiet step: same indices, no frame, no event; a flip
                    // toggles the state, takes its new schedule and the
                    // band's force for that state (the rest of the full step)
                    if (ETA && (int64_t)s == nflip) {
                        t.state ^= 1;
                        nflip = t.state ? ca1 : ca0;
                        t.F = t.state ? bF1 : bF0;
                    }
                    if (t.state) ++sc1; else ++sc0;
                    if (!OVER) t.v = t.v + (k.invM * t.F) * k.hdt;
                    ++s;
                    ++l;
                    continue;
                }
                const FlipFromBuffer src{&buf.cand[u][0][l][lane], &buf.cand[u][1][l][lane]};
                const int r = fp64_after_move<DBL, OVER, ETA>(k, st, i, g, t, s, src, nflip, sc0, sc1, flags, nxf,
                                                              cell_prev, well_prev, lb_prev);
                if (r == 1) { run = false; break; }
                if (r == 2) { ++s; run = false; break; }
                quiet_band<DBL>(k, t, &blo, &bhi);
                band_forces<DBL>(k, t, &bF0, &bF1);
                ++s;
                ++l;
            }
        }
        __syncwarp();
        grp_arrive<P>(7 + u);                   // buffer u released
    }
    if (!active) return;   // a trajectory done before the launch keeps its state
    // s is the first step not integrated
    const int64_t n = st.n;
    st.counts[(int64_t)LDP_C_STATE0 * n + i] = sc0;
    st.counts[(int64_t)LDP_C_STATE1 * n + i] = sc1;
    st.counts[(int64_t)LDP_C_STEPS * n + i] = (int64_t)s - 1;
    if (k.fp_mode && !(t.bits & B_DONE) && s_end > k.step_cap) flags |= LDP_FLAG_CENSORED;
    if (flags) st.counts[(int64_t)LDP_C_FLAGS * n + i] |= (int64_t)flags;
    st.nflip[i] = nflip;
    store_traj(st, t, i);
}

template <bool DBL, bool OVER>
static int launch_init_t(const KConst& k, const TrajState& st, int64_t g0, int block, cudaStream_t stream) {
    const int64_t grid = (st.n + block - 1) / block;
    fp64_init_kernel<DBL, OVER><<<(unsigned)grid, block, 0, stream>>>(k, st, g0);
    return (int)cudaGetLastError();
}

int launch_fp64_init(const KConst& k, const TrajState& st, int64_t g0, int block, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    block = 128;
    if (k.dbl) return k.over ? launch_init_t<true, true>(k, st, g0, block, s) : launch_init_t<true, false>(k, st, g0, block, s);
    return k.over ? launch_init_t<false, true>(k, st, g0, block, s) : launch_init_t<false, false>(k, st, g0, block, s);
}

template <bool DBL, bool OVER, bool ETA>
static int launch_steps_t(const KConst& k, const TrajState& st, int64_t g0, uint64_t s0, uint64_t s1, int block,
                          cudaStream_t stream) {
    const int64_t grid = (st.n + block - 1) / block;
    fp64_steps_kernel<DBL, OVER, ETA><<<(unsigned)grid, block, 0, stream>>>(k, st, g0, s0, s1);
    return (int)cudaGetLastError();
}

template <bool DBL, bool OVER, bool ETA>
static int launch_latency_t(const KConst& k, const TrajState& st, int64_t g0, uint64_t s0, uint64_t s1,
                            cudaStream_t stream) {
    fp64_latency_kernel<DBL, OVER, ETA><<<(unsigned)st.n, 64, 0, stream>>>(k, st, g0, s0, s1);
    return (int)cudaGetLastError();
}

int launch_fp64_latency(const KConst& k, const TrajState& st, int64_t g0, uint64_t s_begin, uint64_t s_end,
                        void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (st.n <= 0) return 0;
    const int sel = (k.dbl ? 4 : 0) | (k.over ? 2 : 0) | (k.eta ? 1 : 0);
    switch (sel) {
        case 0: return launch_latency_t<false, false, false>(k, st, g0, s_begin, s_end, s);
        case 1: return launch_latency_t<false, false, true>(k, st, g0, s_begin, s_end, s);
        case 2: return launch_latency_t<false, true, false>(k, st, g0, s_begin, s_end, s);
        case 3: return launch_latency_t<false, true, true>(k, st, g0, s_begin, s_end, s);
        case 4: return launch_latency_t<true, false, false>(k, st, g0, s_begin, s_end, s);
        case 5: return launch_latency_t<true, false, true>(k, st, g0, s_begin, s_end, s);
        case 6: return launch_latency_t<true, true, false>(k, st, g0, s_begin, s_end, s);
        default: return launch_latency_t<true, true, true>(k, st, g0, s_begin, s_end, s);
    }
}

template <bool DBL, bool OVER, bool ETA>
static int launch_group_t(const KConst& k, const TrajState& st, int64_t g0, uint64_t s0, uint64_t s1,
                          cudaStream_t stream) {
    const int64_t grid = (st.n + 31) / 32;
    if (st.n > kGrpWideMin) fp64_group_kernel<DBL, OVER, ETA, 2><<<(unsigned)grid, 96, 0, stream>>>(k, st, g0, s0, s1);
    else fp64_group_kernel<DBL, OVER, ETA, 4><<<(unsigned)grid, 160, 0, stream>>>(k, st, g0, s0, s1);
    return (int)cudaGetLastError();
}

int launch_fp64_group(const KConst& k, const TrajState& st, int64_t g0, uint64_t s_begin, uint64_t s_end,
                      void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (st.n <= 0) return 0;
    const int sel = (k.dbl ? 4 : 0) | (k.over ? 2 : 0) | (k.eta ? 1 : 0);
    switch (sel) {
        case 0: return launch_group_t<false, false, false>(k, st, g0, s_begin, s_end, s);
        case 1: return launch_group_t<false, false, true>(k, st, g0, s_begin, s_end, s);
        case 2: return launch_group_t<false, true, false>(k, st, g0, s_begin, s_end, s);
        case 3: return launch_group_t<false, true, true>(k, st, g0, s_begin, s_end, s);
        case 4: return launch_group_t<true, false, false>(k, st, g0, s_begin, s_end, s);
        case 5: return launch_group_t<true, false, true>(k, st, g0, s_begin, s_end, s);
        case 6: return launch_group_t<true, true, false>(k, st, g0, s_begin, s_end, s);
        default: return launch_group_t<true, true, true>(k, st, g0, s_begin, s_end, s);
    }
}

int launch_fp64_steps(const KConst& k, const TrajState& st, int64_t g0, uint64_t s_begin, uint64_t s_end, int block,
                      void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    block = 128;
    const int sel = (k.dbl ? 4 : 0) | (k.over ? 2 : 0) | (k.eta ? 1 : 0);
    switch (sel) {
        case 0: return launch_steps_t<false, false, false>(k, st, g0, s_begin, s_end, block, s);
        case 1: return launch_steps_t<false, false, true>(k, st, g0, s_begin, s_end, block, s);
        case 2: return launch_steps_t<false, true, false>(k, st, g0, s_begin, s_end, block, s);
        case 3: return launch_steps_t<false, true, true>(k, st, g0, s_begin, s_end, block, s);
        case 4: return launch_steps_t<true, false, false>(k, st, g0, s_begin, s_end, block, s);
        case 5: return launch_steps_t<true, false, true>(k, st, g0, s_begin, s_end, block, s);
        case 6: return launch_steps_t<true, true, false>(k, st, g0, s_begin, s_end, block, s);
        default: return launch_steps_t<true, true, true>(k, st, g0, s_begin, s_end, block, s);
    }
}

}  // namespace ldp
