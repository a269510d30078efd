// ldp_fp32.cu -- FP32 batched persistent trajectory kernel.
//
// Same model as the FP64 plain path (src/langevinDynamicsSingleBarrier.h:
// 1292-1324, 1680-1706, 1861-1884, 1998-2165, 2334-2592, 2860-2886 and the
// double-barrier counterparts in src/langevinDynamicsDoubleBarrier.h), with
// the step in FP32:
//  * position = cell * L + xp with an int cell index and an FP32 cell-local
//    coordinate xp in [-L/2, L/2) (no FP32 absolute position);
//  * Box-Muller noise on the special-function units (lg2/sqrt/sin/cos
//    approximations) from the same Philox words the FP64 path uses, the
//    uniforms built from the words' high bits by exponent splicing;
//  * an exact integer step counter as the clock; event durations are summed
//    as integer step counts (exact), frames are saved as FP64 cell*L + xp.
//
// Hot loop.  The force of both models is piecewise constant in xp: between
// consecutive "breakpoints" (cell edges, barrier flanks, the barrier top and,
// for the double model, the flank meeting point) neither the force, the
// cell, the well nor the local barrier changes.  Each thread keeps the open
// band (lo, hi) around its position, the force of its current barrier state
// and the high word of its flip threshold in registers, so a step is the
// Philox/Box-Muller draw, the position update and three compares.  Every
// step that leaves the band, draws a flip (or a threshold tie), or reaches a
// frame or the last step takes the general step below, which follows the
// FP64 step exactly (wrap, indices, flip, cell-table entry with lazy
// catch-up, force, renewal statistics, frame, end).
//
// Rare state lives in shared memory (statistics clocks and flags, the cached
// state of the cell left last, the state-1 step count), counts and duration
// sums go out as fire-and-forget atomics, and the cell-table ring is written
// through on every cell exit, so re-crossing back into the cell just left
// needs no memory read.
//
// Batching: each thread is a slot that owns one trajectory; when it retires
// (fixed step count reached, or first passage in FIRST_PASSAGE mode) the
// warp's idle lanes claim new trajectories from the device work queue with
// one fetch-and-add per warp and a ballot/popc prefix.
#include <cuda_runtime.h>

#include "ldp_device.cuh"
#include "ldp_fp32.h"

namespace ldp {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxBlock = 256;
constexpr int kLeftMax = 1 << 30;      // countdown clamp; a clamped zero is a no-op general step

// Statistics flags used only by this path (bits 0..23 are the shared B_*).
enum : uint32_t { B_HAS_FPT = 1u << 24, B_HAS_FPT2 = 1u << 25, B_HAS_TPT = 1u << 26, B_HAS_TPT2 = 1u << 27 };
// Slot word: local barrier, eviction pending for the current cell, cache of
// the cell left last (valid, its state).
enum : int32_t { W_LB = 1, W_EVICT = 2, W_CVALID = 4, W_CSTATE = 8 };

// Per-thread rare state, structure of arrays (conflict-free by thread).
struct RareSm {
    uint32_t bits[kMaxBlock];
    int32_t init0[kMaxBlock];     // first cell of the FPT initial-barrier pair
    int32_t idx2[kMaxBlock];      // first cell of the FPT2 reference pair
    int32_t tpt2w[kMaxBlock];     // well of the last TPT2 renewal
    int32_t ckey[kMaxBlock];      // key of the cell left last
    int32_t cgw[kMaxBlock];       // well of the last FPTCG evaluation
    int32_t fidx[kMaxBlock];      // index of the next frame
    long long nxf[kMaxBlock];     // step of the next frame
    long long fpt[kMaxBlock], fpt2[kMaxBlock], tpt[kMaxBlock], tpt2[kMaxBlock];
    long long cflip[kMaxBlock];   // pending flip step of the cached cell
    long long sc1[kMaxBlock];     // completed state-1 steps
    long long since[kMaxBlock];   // first step of the current state-1 run
    // Lane state the hot loop hands to the general step and takes back, and
    // the lane state only the general step uses.
    float xp[kMaxBlock], rv[kMaxBlock], F[kMaxBlock], lo[kMaxBlock], hi[kMaxBlock], c1[kMaxBlock];
    uint32_t traj[kMaxBlock];
    uint32_t gtraj[kMaxBlock];    // the trajectory's random-stream index (traj + the job's g0)
    uint32_t key0[kMaxBlock], key1[kMaxBlock];
    float kn[kMaxBlock];
    long long nflip[kMaxBlock];   // step of the current barrier's next flip
    int32_t left[kMaxBlock], job[kMaxBlock], cell[kMaxBlock], state[kMaxBlock], sw[kMaxBlock];
};

__device__ __forceinline__ void red_add(int64_t* p, int64_t v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

__device__ __forceinline__ int fkey(bool dbl, int cell, int lb) { return dbl ? cell * 2 + lb : cell; }

// Step of the next flip of a barrier now in state st, scheduled at step s
// (words w0:w1 of TAG_FLIP at a = s; geometric waiting time, FP64 as in the
// FP64 path, so both precisions schedule the same flips from the same
// history).
__device__ __forceinline__ long long next_flip(const JobF& J, uint32_t traj, uint64_t s, int st) {
    const Words w = philox_at(s, traj, TAG_FLIP, J.key0, J.key1);
    return flip_schedule(s, w.w0, w.w1, J.ln1m[st]);
}

// Uniform in (0, 1): the high 23 bits of w as a mantissa, offset by 2^-24.
__device__ __forceinline__ float unit_open(uint32_t w) {
    return __int_as_float((int)__funnelshift_r(w, 0x7fu, 9)) - 0.99999994039535522461f;
}
// w * 2^-32 folded into [-1/2, 1/2) (same angle mod 1), 23 high bits.
__device__ __forceinline__ float unit_centered(uint32_t w) {
    return __int_as_float((int)(__funnelshift_r(w, 0x7fu, 9) ^ 0x00400000u)) - 1.5f;
}

// Box-Muller pair scaled by sigma: k = -2 ln 2 sigma^2 (log2 is the native
// logarithm of the special-function unit).  Flush-to-zero forms: the
// uniforms are normal numbers in (2^-24, 1) and the angle in [-pi, pi).
__device__ __forceinline__ void noise_pair(uint32_t wa, uint32_t wb, float k, float* n0, float* n1) {
    float lg, r, sn, cs;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(lg) : "f"(unit_open(wa)));
    const float t = fmaxf(lg * k, 0.0f);
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(t));
    const float a = 6.28318530717958647692f * unit_centered(wb);
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(sn) : "f"(a));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(cs) : "f"(a));
    *n0 = r * cs;
    *n1 = r * sn;
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

__device__ __forceinline__ int f_ring_state(const JobF& J, const SlotsDev& S, int64_t slot, bool dbl, uint32_t g,
                                            int key) {
    const longlong2 e = S.ring[(int64_t)(key & (S.ring_slots - 1)) * S.nslots + slot];
    return (e.x == (long long)key) ? (int)(e.y & 1) : f_default_state(J, dbl, g, key);
}

// FP32 force of state st at xp (EnergyAndForce, S.h:1292-1324 /
// D.h:1464-1522).
template <bool DBL>
__device__ __forceinline__ float force_of(const JobF& J, float xp, int st) {
    if (!DBL) {
        const float a = fabsf(xp);
        return (a < J.w && a > 0.0f) ? copysignf(J.slope[st], xp) : 0.0f;
    } else {
        float f = 0.0f;
        if (xp < J.xb[0] && xp > J.lo0) f = J.sN[0][st];
        if (xp < J.xc && xp > J.xb[0]) f = J.sP[0][st];
        if (xp < J.xb[1] && xp > J.xc) f = J.sN[1][st];
        if (xp < J.hi1 && xp > J.xb[1]) f = J.sP[1][st];
        return -f;
    }
}

// Open band (lo, hi) of consecutive breakpoints around xp; lo = hi = xp when
// xp sits on a breakpoint, so that the next step takes the general path.
// Single barrier: the breakpoints are -L/2, -w, 0, w (clamped to the cell).
template <bool DBL>
__device__ __forceinline__ void band_of(const JobF& J, float xp, float* lo, float* hi) {
    if (!DBL) {
        const float w = J.w, hL = J.halfL, a = fabsf(xp);
        float l, h;
        if (a < w) { l = (xp > 0.0f) ? 0.0f : -w; h = (xp > 0.0f) ? w : 0.0f; }
        else { l = (xp > 0.0f) ? w : -hL; h = (xp > 0.0f) ? hL : -w; }
        l = fmaxf(l, -hL);
        h = fminf(h, hL);
        if (a == w || xp == 0.0f || xp == -hL) l = h = xp;
        *lo = l;
        *hi = h;
        return;
    }
    float l = -__int_as_float(0x7f800000), h = __int_as_float(0x7f800000);
    for (int i = 0; i < J.nbp; ++i) {
        const float b = J.bp[i];
        if (b < xp) { l = b; continue; }
        if (b == xp) l = h = xp; else h = b;
        break;
    }
    *lo = l;
    *hi = h;
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

// WRITEX frame fields (velocity, force, barrier, energies, state).
template <bool DBL>
__device__ __noinline__ void f_record_extra(const JobF* Jp, int64_t o, float xp, float v, float F, int state) {
    const JobF& J = *Jp;
    double E, B;
    f_energy<DBL>(J, (double)xp, state, &E, &B);
    if (J.fv) J.fv[o] = (double)v;
    if (J.ff) J.ff[o] = (double)F;
    if (J.fb) J.fb[o] = B;
    if (J.fpe) J.fpe[o] = E;
    if (J.fke) J.fke[o] = J.mhalf * ((double)v * (double)v);
    if (J.fst) J.fst[o] = (double)state;
}

template <bool DBL>
__device__ __forceinline__ void f_record(const JobF& J, uint32_t traj, int64_t frame, int cell, float xp, float v,
                                         float F, int state) {
    if (frame >= J.nframe) return;   // the frame arrays hold nframe rows
    const int64_t o = frame * J.ntraj + traj;
    if (J.fx) J.fx[o] = (double)cell * J.Ld + (double)xp;
    if (J.write_x) f_record_extra<DBL>(&J, o, xp, v, F, state);
}

__device__ __forceinline__ bool cg_hit32(int well, int size) { return (well % size) == 0; }

// Step 0 of a trajectory (IntegrateStep0 + InitializeBarrierState +
// InitializeStatistics), FP64 where it is cheap and exact, then the hot
// state is rounded to FP32.  Writes the thread's rare state.
template <bool DBL, bool OVER>
__device__ __noinline__ void f_start(const JobF* Jp, longlong2* ring, int64_t nslots, int ring_slots, int64_t slot,
                                     uint32_t traj, RareSm* sm, int t, float* xp, float* rv, int* cell, int* state,
                                     int* sw) {
    const JobF& J = *Jp;
    const uint32_t g = traj + J.g0;   // the trajectory's random streams
    if (J.resume) {
        // Continue from the state kept at step S = step0 - 1: the ring, the
        // hot state, the statistics clocks; the state-1 steps counted so far
        // complete, a state-1 run going on restarting at S + 1 (the same
        // total); frames continue after frame S / FREQSAVE.
        const int64_t n = J.ntraj;
        for (int r = 0; r < ring_slots; ++r) ring[(int64_t)r * nslots + slot] = J.ck_ring[(int64_t)r * n + traj];
        // a trajectory frozen as non-finite stays so (its first step retires it)
        *xp = (J.counts[(int64_t)LDP_C_FLAGS * n + traj] & LDP_FLAG_NONFINITE) ? __int_as_float(0x7fc00000)
                                                                                : J.ck_xp[traj];
        *rv = J.ck_rv[traj];
        *cell = J.ck_cell[traj];
        *sw = J.ck_sw[traj];
        *state = J.state_final[traj];
        sm->bits[t] = (uint32_t)J.bits[traj];
        sm->init0[t] = J.init_idx0[traj];
        sm->idx2[t] = J.idx2_0[traj];
        sm->tpt2w[t] = J.tpt2_well[traj];
        sm->ckey[t] = J.ck_ckey[traj];
        sm->cflip[t] = J.ck_cflip[traj];
        sm->nflip[t] = J.ck_nflip[traj];
        sm->fpt[t] = J.fpt_last[traj];
        sm->fpt2[t] = J.fpt2_last[traj];
        sm->tpt[t] = J.tpt_last[traj];
        sm->tpt2[t] = J.tpt2_last[traj];
        sm->cgw[t] = INT32_MIN;
        const uint64_t S0 = J.step0 - 1, fs = J.freq_save;
        sm->fidx[t] = (int)(S0 / fs) + 1;
        sm->nxf[t] = (long long)((S0 / fs + 1) * fs);
        sm->sc1[t] = J.counts[(int64_t)LDP_C_STATE1 * n + traj];
        sm->since[t] = (long long)J.step0;
        return;
    }
    for (int r = 0; r < ring_slots; ++r) ring[(int64_t)r * nslots + slot] = make_longlong2((long long)INT64_MIN, 0);
    const double red = J.x0 * J.invL;
    const int c = (int)rint(red);
    const int well = (int)floor(red);
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
    int init0 = 0, idx2 = 0;
    if (J.at_bottom) {
        if (!DBL && J.fpt && !J.fp_mode) {
            // FPT initial barrier pair (S.h:2187-2211); the ring is empty, so
            // the neighbour has its default state.
            int s0, s1;
            if (well == c) { s0 = st; s1 = f_default_state(J, false, g, c + 1); init0 = c; }
            else { s0 = f_default_state(J, false, g, c - 1); s1 = st; init0 = c - 1; }
            bits |= (s0 ? B_INIT0 : 0u) | (s1 ? B_INIT1 : 0u);
        }
        idx2 = (well == c) ? c : c - 1;
    } else {
        bits |= B_FPT_UP | B_FPT2_UP | B_TPT_UP | B_TPT2_UP;
    }
    for (int j = 0; j < J.n_cg; ++j) {
        J.cg_last[(int64_t)j * J.ntraj + traj] = 0;
        J.cg_well[(int64_t)j * J.ntraj + traj] = well;
        if (!(J.at_bottom && cg_hit32(well, J.cg_size[j]))) bits |= (B_CG0 << j);
    }
    if (!DBL && J.wt) J.wt_tick[traj] = 0;
    sm->bits[t] = bits;
    sm->init0[t] = init0;
    sm->idx2[t] = idx2;
    sm->tpt2w[t] = well;
    sm->ckey[t] = 0;
    sm->cgw[t] = INT32_MIN;
    sm->fidx[t] = 1;
    sm->nxf[t] = (!J.fp_mode && J.freq_save) ? (long long)J.freq_save : INT64_MAX;
    sm->nflip[t] = next_flip(J, g, 0, st);
    sm->fpt[t] = sm->fpt2[t] = sm->tpt[t] = sm->tpt2[t] = 0;
    sm->cflip[t] = 0;
    sm->sc1[t] = 0;
    sm->since[t] = 0;
    *xp = (float)xpd;
    *cell = c;
    *state = st;
    *sw = l ? W_LB : 0;
    *rv = OVER ? (float)(J.sig_r_d * zr) : (float)v;
    if (!J.fp_mode) {
        const float F = force_of<DBL>(J, *xp, st);
        f_record<DBL>(J, traj, 0, c, *xp, OVER ? 0.0f : (float)v, F, st);
    }
}

__device__ __noinline__ void f_retire(const JobF* Jp, unsigned long long* retired, uint32_t traj, uint64_t steps_done,
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
    atomicAdd(retired, 1ull);
}

// Resolves a claimed queue index to (job, trajectory).
__device__ __noinline__ int64_t f_resolve(const int64_t* range_end, const int32_t* range_job,
                                          const int64_t* range_first, const int32_t* nranges, int64_t idx, int* job) {
    int lo = 0, hi = *(volatile const int32_t*)nranges - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (range_end[mid] > idx) hi = mid; else lo = mid + 1;
    }
    const int64_t begin = lo ? range_end[lo - 1] : 0;
    *job = range_job[lo];
    return range_first[lo] + (idx - begin);
}

// Steps from step s to the next frame (step nxf), flip (step nf) or the
// last step.
__device__ __forceinline__ int steps_to_special(const JobF& J, uint64_t s, long long nxf, long long nf) {
    uint64_t e = (uint64_t)nxf < J.nsteps ? (uint64_t)nxf : J.nsteps;
    e = (uint64_t)nf < e ? (uint64_t)nf : e;
    const uint64_t d = e - s;
    return (int)(d < (uint64_t)kLeftMax ? d : (uint64_t)kLeftMax);
}

// 1 - e^x for x <= 0 in FP32: a degree-5 Taylor polynomial of -expm1 on
// (-1/32, 0] (truncation below 1e-10 relative), 1 - expf(x) below.
__device__ __forceinline__ float one_minus_exp(float x) {
    if (x > -0.03125f)
        return -x * fmaf(x, fmaf(x, fmaf(x, fmaf(x, 1.0f / 120.0f, 1.0f / 24.0f), 1.0f / 6.0f), 0.5f), 1.0f);
    return 1.0f - expf(x);
}

// End of a trajectory after step `done` (v: velocity after that step).
template <bool OVER>
__device__ __forceinline__ void retire_lane(const JobF& J, unsigned long long* retired, RareSm& sm, int t,
                                            uint64_t done, float xp, float v, uint32_t flags) {
    const int state = sm.state[t];
    const int64_t sc1 = sm.sc1[t] + (state ? (int64_t)done + 1 - sm.since[t] : 0);
    if (J.fp_mode && !(flags & LDP_FLAG_NONFINITE) && !(sm.bits[t] & B_HAS_FPT2)) flags |= LDP_FLAG_CENSORED;
    f_retire(&J, retired, sm.traj[t], done, sc1, sm.cell[t], xp, OVER ? 0.0f : v, state, flags);
}

// Keeps the continuation state of a trajectory that completed its last
// step (see JobF::ck_*); rv: the velocity after the step (underdamped) or
// the step's random force (overdamped).
__device__ __noinline__ void f_keep_state(const JobF* Jp, const SlotsDev* Sp, const RareSm* smp, int t, int64_t slot,
                                          uint32_t traj, float xp, float rv, int cell, int sw) {
    const JobF& J = *Jp;
    const SlotsDev& S = *Sp;
    const RareSm& sm = *smp;
    const int64_t n = J.ntraj;
    J.ck_xp[traj] = xp;
    J.ck_rv[traj] = rv;
    J.ck_cell[traj] = cell;
    J.ck_sw[traj] = sw;
    J.ck_ckey[traj] = sm.ckey[t];
    J.ck_cflip[traj] = sm.cflip[t];
    J.ck_nflip[traj] = sm.nflip[t];
    for (int r = 0; r < S.ring_slots; ++r) J.ck_ring[(int64_t)r * n + traj] = S.ring[(int64_t)r * S.nslots + slot];
    J.bits[traj] = (int32_t)sm.bits[t];
    J.init_idx0[traj] = sm.init0[t];
    J.idx2_0[traj] = sm.idx2[t];
    J.tpt2_well[traj] = sm.tpt2w[t];
    J.fpt_last[traj] = sm.fpt[t];
    J.fpt2_last[traj] = sm.fpt2[t];
    J.tpt_last[traj] = sm.tpt[t];
    J.tpt2_last[traj] = sm.tpt2[t];
}

// Ends a lane's trajectory after step `done` (general step): keeps its
// continuation state when the job asks for it and the trajectory completed,
// then retires it.  The lane's cell, state and slot word in sm are current.
template <bool OVER>
__device__ __noinline__ void f_end_lane(const JobF* Jp, const SlotsDev* Sp, RareSm* smp, int t, int64_t slot,
                                        uint64_t done, float xp, float v, float rv, uint32_t flags) {
    const JobF& J = *Jp;
    RareSm& sm = *smp;
    if (J.ck_xp && !flags && done == J.nsteps)
        f_keep_state(Jp, Sp, smp, t, slot, sm.traj[t], xp, OVER ? rv : v, sm.cell[t], sm.sw[t]);
    retire_lane<OVER>(J, Sp->retired, sm, t, done, xp, v, flags);
}

// The general step s of one lane (position already advanced):
// the FP64 step order of ldp_fp64.cu from the index update on.  Out of line,
// on the lane state in shared memory, so that the hot loop's registers do
// not carry its working set.
template <bool DBL, bool OVER>
__device__ __noinline__ void general_step(const JobF* jobs, const SlotsDev* Sp, RareSm* smp, int t, int64_t slot,
                                          uint64_t s) {
    RareSm& sm = *smp;
    const SlotsDev& S = *Sp;
    const float kInf = __int_as_float(0x7f800000);
    int job = sm.job[t];
    if (job < 0) return;
    const JobF& J = jobs[job];
    const uint32_t traj = sm.traj[t];
    const uint32_t gp = traj + J.g0;   // the trajectory's random streams
    float xp = sm.xp[t];
    const float rv = sm.rv[t];
    float lo = sm.lo[t], hi = sm.hi[t];
    int cell = sm.cell[t], state = sm.state[t], sw = sm.sw[t];
    int left = sm.left[t];

    auto retire = [&](uint64_t done, float v, uint32_t flags) {
        sm.cell[t] = cell;
        sm.state[t] = state;
        sm.sw[t] = sw;
        f_end_lane<OVER>(&J, &S, &sm, t, slot, done, xp, v, rv, flags);
        sm.job[t] = -1;
        sm.lo[t] = -kInf;
        sm.hi[t] = kInf;
        sm.F[t] = 0.f;
        sm.left[t] = kLeftMax;
    };

    // Cell (double model: local barrier) entry (UpdateBarrierStateEta,
    // S.h:2025-2068 / D.h:2468-2517): write the state and pending flip step
    // of the key left (*nf) through to the ring and the one-entry cache, take
    // the entered key's from the cache or the ring.  A barrier re-entered
    // before its pending flip has not flipped meanwhile; one whose flip came
    // while it was away (or never visited: created at step 0) is caught up
    // from that step and gets a new schedule (words w2:w3 of TAG_FLIP at s,
    // *wf when the flip of this step already drew them).
    auto enter = [&](int key_prev, int st, int key_cur, long long* nf, Words* wf, bool have_wf) -> int {
        const int64_t n = J.ntraj;
        const int rmask = S.ring_slots - 1;
        if (sw & W_EVICT) red_add(&J.counts[(int64_t)LDP_C_EVICT * n + traj], 1);
        S.ring[(int64_t)(key_prev & rmask) * S.nslots + slot] =
            make_longlong2((long long)key_prev, (*nf << 1) | (long long)st);
        int ps;
        long long nb;
        bool found = true, ev = false;
        if ((sw & W_CVALID) && sm.ckey[t] == key_cur) {
            ps = (sw & W_CSTATE) ? 1 : 0;
            nb = sm.cflip[t];
        } else {
            const longlong2 e = S.ring[(int64_t)(key_cur & rmask) * S.nslots + slot];
            if (e.x == (long long)key_cur) {
                ps = (int)(e.y & 1);
                nb = e.y >> 1;
            } else {
                ps = f_default_state(J, DBL, gp, key_cur);
                nb = 0;
                found = false;
                ev = e.x != (long long)INT64_MIN;
            }
        }
        sm.ckey[t] = key_prev;
        sm.cflip[t] = *nf;
        sw = (sw & W_LB) | W_CVALID | (st ? W_CSTATE : 0) | (ev ? W_EVICT : 0);
        if (!J.eta) return ps;
        if (found && nb > (long long)s) {
            *nf = nb;
            return ps;
        }
        // Flip with probability c (1 - e^{a lap}) over the steps since the
        // missed flip, FP32, against the high word of the same catch-up
        // uniform the FP64 path draws.
        const int sb = found ? (ps ^ 1) : ps;
        const float pl = J.c_lapf[J.eq ? 0 : sb] * one_minus_exp(J.a_lapf * (float)((long long)s - nb));
        const uint32_t w0 = philox_at(s, gp, TAG_CATCHUP, J.key0, J.key1).w0;
        const int sn = ((pl >= 1.0f) || (w0 < (uint32_t)(pl * 4294967296.0f))) ? (sb ^ 1) : sb;
        if (!have_wf) *wf = philox_at(s, gp, TAG_FLIP, J.key0, J.key1);
        *nf = flip_schedule(s, wf->w2, wf->w3, J.ln1m[sn]);
        return sn;
    };

    // Renewal statistics (UpdateStatistics, S.h:2334-2592 / D.h:2931-3209)
    // with integer step clocks.  Returns true when a FIRST_PASSAGE
    // trajectory ends.
    auto events = [&](int64_t now, bool dWell, bool dCell, int well) -> bool {
        const int64_t n = J.ntraj;
        int64_t* C = J.counts;
        int64_t* U = J.ssum;
        uint32_t bits = sm.bits[t];
        bool done = false;
        const int evm = J.evm;
        if (!DBL && (evm & EV_WT)) {
            if (dWell) { J.wt_tick[traj] = now; bits |= B_WT_PASSED; }
            else if (dCell && (bits & B_WT_PASSED)) {
                int64_t& nwt = C[(int64_t)LDP_C_WT * n + traj];
                if (nwt < J.tick_cap) J.ticks[(int64_t)traj * J.tick_cap + nwt] = J.wt_tick[traj];
                else C[(int64_t)LDP_C_FLAGS * n + traj] |= LDP_FLAG_TICK_OVERFLOW;
                nwt += 1;
                bits &= ~B_WT_PASSED;
            }
        }
        if (evm & EV_FPT2) {
            if (!DBL && (evm & EV_FPT)) {
                if ((bits & B_FPT_UP) && dCell) {
                    // initial barrier pair (S.h:2364-2388)
                    bits &= ~(B_FPT_UP | B_INIT0 | B_INIT1);
                    sm.fpt[t] = now;
                    int s0, s1, i0;
                    if (well == cell) { s0 = state; s1 = f_ring_state(J, S, slot, false, gp, cell + 1); i0 = cell; }
                    else { s0 = f_ring_state(J, S, slot, false, gp, cell - 1); s1 = state; i0 = cell - 1; }
                    sm.init0[t] = i0;
                    bits |= (s0 ? B_INIT0 : 0u) | (s1 ? B_INIT1 : 0u);
                }
                if (!(bits & B_FPT_UP) && dWell) {
                    bits |= B_FPT_UP;
                    const int64_t d = now - sm.fpt[t];
                    if (!(bits & B_HAS_FPT)) { bits |= B_HAS_FPT; U[(int64_t)LDP_S_FIRST_FPT * n + traj] = d; }
                    red_add(&U[(int64_t)LDP_S_FPT * n + traj], d);
                    red_add(&C[(int64_t)LDP_C_FPT * n + traj], 1);
                    const bool ib = (cell == sm.init0[t]) ? ((bits & B_INIT0) != 0) : ((bits & B_INIT1) != 0);
                    red_add(&C[(int64_t)(ib ? LDP_C_INIT1 : LDP_C_INIT0) * n + traj], 1);
                    red_add(&C[(int64_t)(state ? LDP_C_INST1 : LDP_C_INST0) * n + traj], 1);
                }
            }
            if ((bits & B_FPT2_UP) && dCell) {
                bits &= ~B_FPT2_UP;
                sm.fpt2[t] = now;
                sm.idx2[t] = (well == cell) ? cell : cell - 1;
            }
            const int i2 = sm.idx2[t];
            if (dCell && !(bits & B_FPT2_UP) && i2 != cell && i2 + 1 != cell) {
                const int64_t d = now - sm.fpt2[t];
                if (!(bits & B_HAS_FPT2)) { bits |= B_HAS_FPT2; U[(int64_t)LDP_S_FIRST_FPT2 * n + traj] = d; }
                red_add(&U[(int64_t)LDP_S_FPT2 * n + traj], d);
                red_add(&C[(int64_t)LDP_C_FPT2 * n + traj], 1);
                sm.fpt2[t] = now;
                sm.idx2[t] = (well == cell) ? cell : cell - 1;
                if (evm & EV_FP) done = true;
            }
        }
        if (!DBL && (evm & EV_TPT)) {
            if (dCell) { bits &= ~B_TPT_UP; sm.tpt[t] = now; }
            if (!(bits & B_TPT_UP) && dWell) {
                bits |= B_TPT_UP;
                const int64_t d = now - sm.tpt[t];
                if (!(bits & B_HAS_TPT)) { bits |= B_HAS_TPT; U[(int64_t)LDP_S_FIRST_TPT * n + traj] = d; }
                red_add(&U[(int64_t)LDP_S_TPT * n + traj], d);
                red_add(&C[(int64_t)LDP_C_TPT * n + traj], 1);
            }
            if (dCell) {
                if (bits & B_TPT2_UP) bits &= ~B_TPT2_UP;
                else if (well != sm.tpt2w[t]) {
                    const int64_t d = now - sm.tpt2[t];
                    if (!(bits & B_HAS_TPT2)) { bits |= B_HAS_TPT2; U[(int64_t)LDP_S_FIRST_TPT2 * n + traj] = d; }
                    red_add(&U[(int64_t)LDP_S_TPT2 * n + traj], d);
                    red_add(&C[(int64_t)LDP_C_TPT2 * n + traj], 1);
                }
                sm.tpt2[t] = now;
                sm.tpt2w[t] = well;
            }
        }
        // An FPTCG evaluation at the well of the previous one changes nothing
        // (every entry it hits already holds that well), so it is skipped.
        if ((evm & EV_CG) && dCell && well != sm.cgw[t]) {
            sm.cgw[t] = well;
            for (int jj = 0; jj < J.n_cg; ++jj) {
                if (cg_hit32(well, J.cg_size[jj])) {
                    const int64_t o = (int64_t)jj * n + traj;
                    if (bits & (B_CG0 << jj)) {
                        bits &= ~(B_CG0 << jj);
                        J.cg_last[o] = now;
                        J.cg_well[o] = well;
                    } else if (well != J.cg_well[o]) {
                        red_add(&U[(int64_t)(LDP_S_CG0 + jj) * n + traj], now - J.cg_last[o]);
                        red_add(&C[(int64_t)(LDP_C_CG0 + jj) * n + traj], 1);
                        J.cg_last[o] = now;
                        J.cg_well[o] = well;
                    }
                }
            }
        }
        sm.bits[t] = bits;
        return done;
    };

    if (J.eta && xp > lo && xp < hi && (long long)s == sm.nflip[t] && (long long)s != sm.nxf[t] &&
        s != J.nsteps && (xp < 0.0f) == (lo < 0.0f) && (!DBL || (xp < J.xc ? 0 : W_LB) == (sw & W_LB))) {
        // Only the current barrier's flip (no band exit, so the same cell,
        // well and local barrier; no frame; not the last step): the path
        // below with flip alone -- the new state and its schedule, the
        // state-1 run, the state's force, the countdown.
        const int st = state ^ 1;
        const Words w = philox_at(s, gp, TAG_FLIP, J.key0, J.key1);
        const long long nf = flip_schedule(s, w.w0, w.w1, J.ln1m[st]);
        if (st) sm.since[t] = (long long)s;
        else sm.sc1[t] += (long long)s - sm.since[t];
        sm.state[t] = st;
        sm.nflip[t] = nf;
        sm.F[t] = force_of<DBL>(J, xp, st);
        sm.left[t] = steps_to_special(J, s, sm.nxf[t], nf);
        return;
    }
    if (xp > lo && xp < hi && (long long)s != sm.nflip[t]) {
        // Only the countdown ran out: a frame and/or the last step.
        const float F = sm.F[t];
        const float vk = OVER ? 0.0f : fmaf(F, sm.c1[t], rv);
        if ((long long)s == sm.nxf[t]) {
            f_record<DBL>(J, traj, sm.fidx[t], cell, xp, vk, F, state);
            sm.fidx[t] += 1;
            sm.nxf[t] += (long long)J.freq_save;
        }
        sm.left[t] = steps_to_special(J, s, sm.nxf[t], sm.nflip[t]);
        if (s == J.nsteps) retire(s, vk, 0);
        return;
    }
    if (!(fabsf(xp) < kInf)) {
        retire(s - 1, rv, LDP_FLAG_NONFINITE);
        return;
    }
    const int cell_prev = cell;
    const int lb_prev = sw & W_LB;
    const int well_prev = cell_prev - (lo < 0.0f ? 1 : 0);
    const bool moved = !(xp > lo && xp < hi);
    if (moved) {
        if (xp >= J.halfL) { xp -= J.L; ++cell; }
        else if (xp < -J.halfL) { xp += J.L; --cell; }
        if (!(xp >= -J.halfL && xp < J.halfL)) {
            // more than one cell in one step
            const float k = floorf(xp * J.invLf + 0.5f);
            xp = fmaf(-k, J.L, xp);
            cell += (int)k;
            if (xp >= J.halfL) { xp -= J.L; ++cell; }
            else if (xp < -J.halfL) { xp += J.L; --cell; }
        }
    }
    const int well = cell - (xp < 0.0f ? 1 : 0);
    const int lb = DBL ? (xp < J.xc ? 0 : 1) : 0;
    const bool dCell = cell != cell_prev;
    const bool dWell = well != well_prev;
    const bool dKey = DBL ? (lb != lb_prev) : dCell;
    // the current barrier flips at its pending flip step and draws the next
    // one; a barrier change takes the entered barrier's schedule
    const bool flip = (long long)s == sm.nflip[t];
    int st = state ^ (int)flip;
    long long nf = sm.nflip[t];
    Words wf{};
    if (flip) {
        wf = philox_at(s, gp, TAG_FLIP, J.key0, J.key1);
        nf = flip_schedule(s, wf.w0, wf.w1, J.ln1m[st]);
    }
    if (dKey) st = enter(fkey(DBL, cell_prev, lb_prev), st, fkey(DBL, cell, lb), &nf, &wf, flip);
    if (DBL) sw = (sw & ~W_LB) | (lb ? W_LB : 0);
    if (st != state) {
        if (st) sm.since[t] = (long long)s;
        else sm.sc1[t] += (long long)s - sm.since[t];
        state = st;
    }
    if (J.eta && (flip || dKey)) {
        sm.nflip[t] = nf;
        left = 0;   // recompute the countdown below
    }
    band_of<DBL>(J, xp, &lo, &hi);
    const float F = force_of<DBL>(J, xp, state);
    bool finish = false;
    if (dCell || dWell) finish = events((int64_t)s, dWell, dCell, well);
    const float vk = OVER ? 0.0f : fmaf(F, sm.c1[t], rv);
    if (left == 0) {
        if ((long long)s == sm.nxf[t]) {
            f_record<DBL>(J, traj, sm.fidx[t], cell, xp, vk, F, state);
            sm.fidx[t] += 1;
            sm.nxf[t] += (long long)J.freq_save;
        }
        if (s == J.nsteps) finish = true;
        left = steps_to_special(J, s, sm.nxf[t], sm.nflip[t]);
    }
    sm.xp[t] = xp;
    sm.cell[t] = cell;
    sm.state[t] = state;
    sm.sw[t] = sw;
    sm.lo[t] = lo;
    sm.hi[t] = hi;
    sm.F[t] = F;
    sm.left[t] = left;
    if (finish) retire(s, vk, 0);
}

// The light step: the commonest special steps, handled in the hot loop
// with the same result the general step gives them, so that the warp does
// not pay for the out-of-line call.  Returns 0 when the step needs the
// general step; 1 when it was handled and the countdown is unchanged; 2 when
// it was handled and *lrel holds the steps from s to the next special step.
//  * A frame step (the countdown ends at a frame, not at a flip or the last
//    step), the position inside its band, no WRITEX series: the frame is
//    written (FP64 cell * L + xp) and the countdown restarts.
//  * A band exit inside the cell (a barrier flank entered or left), with no
//    change of well (barrier top) or local barrier: new band and force.
//  * A crossing of the cell edge into the flat band of the neighbour cell
//    whose barrier is the cached one (the cell left last) and has not passed
//    its pending flip, with no flip at this step and no renewal statistic
//    firing (every statistic already holds this well): the barrier state,
//    pending flip and state-1 run change as in the general step's cell
//    entry, the ring is written through, the transition-path clocks restart.
template <bool DBL>
__device__ __forceinline__ int light_step(const JobF* jobs, const SlotsDev& S, RareSm& sm, int t, int64_t slot,
                                          int job, uint32_t traj, uint64_t s, bool countdown, float& xp, float& lo,
                                          float& hi, float& F, int& lrel) {
    const JobF& J = jobs[job];
    const long long nflip = sm.nflip[t];
    if (countdown) {
        const long long nxf = sm.nxf[t];
        if (!(xp > lo && xp < hi) || (long long)s != nxf || (long long)s == nflip || s == J.nsteps || J.write_x)
            return 0;
        const int fidx = sm.fidx[t];
        if (fidx < J.nframe && J.fx) J.fx[(int64_t)fidx * J.ntraj + traj] = (double)sm.cell[t] * J.Ld + (double)xp;
        sm.fidx[t] = fidx + 1;
        const long long nx2 = nxf + (long long)J.freq_save;
        sm.nxf[t] = nx2;
        lrel = steps_to_special(J, s, nx2, nflip);
        return 2;
    }
    if ((long long)s == nflip) return 0;
    const float hL = J.halfL;
    int sw = sm.sw[t];
    if (xp >= -hL && xp < hL) {
        // inside the cell: a band change unless the well or the local
        // barrier changes, or xp sits on a breakpoint
        float l2, h2;
        band_of<DBL>(J, xp, &l2, &h2);
        if (!(xp > l2 && xp < h2)) return 0;
        if ((xp < 0.0f) != (lo < 0.0f)) return 0;
        if (DBL && ((xp < J.xc ? 0 : W_LB) != (sw & W_LB))) return 0;
        lo = l2;
        hi = h2;
        F = force_of<DBL>(J, xp, sm.state[t]);
        return 1;
    }
    if (!J.edge_flat || !J.eta) return 0;
    float xn;
    int dc;
    if (xp >= hL) {
        xn = xp - J.L;
        dc = 1;
        if (!(xn > -hL && xn < J.edge_lo)) return 0;
    } else if (xp < -hL) {
        xn = xp + J.L;
        dc = -1;
        if (!(xn > J.edge_hi && xn < hL)) return 0;
    } else {
        return 0;   // not finite
    }
    const int cell_prev = sm.cell[t], cell = cell_prev + dc;
    const int well = cell - (xn < 0.0f ? 1 : 0);
    if (well != cell_prev - (lo < 0.0f ? 1 : 0)) return 0;
    const int lb = DBL ? (xn < J.xc ? 0 : 1) : 0;
    if (DBL && lb == (sw & W_LB)) return 0;   // the general step enters a key only when lb changes
    const int key_prev = fkey(DBL, cell_prev, sw & W_LB), key = fkey(DBL, cell, lb);
    if (!(sw & W_CVALID) || sm.ckey[t] != key || sm.cflip[t] <= (long long)s) return 0;
    const uint32_t bits = sm.bits[t];
    const int evm = J.evm;
    if ((evm & EV_FPT) && (bits & B_FPT_UP)) return 0;
    if ((evm & EV_FPT2) && ((bits & B_FPT2_UP) || sm.idx2[t] != well)) return 0;
    if ((evm & EV_TPT) && !(bits & B_TPT2_UP) && sm.tpt2w[t] != well) return 0;
    if ((evm & EV_CG) && sm.cgw[t] != well) return 0;
    if ((evm & EV_WT) && (bits & B_WT_PASSED)) return 0;
    // leave key_prev (its eviction, if its entry displaced another cell's,
    // is counted now), enter the cached key
    const int st_prev = sm.state[t];
    if (sw & W_EVICT) red_add(&J.counts[(int64_t)LDP_C_EVICT * J.ntraj + traj], 1);
    S.ring[(int64_t)(key_prev & (S.ring_slots - 1)) * S.nslots + slot] =
        make_longlong2((long long)key_prev, (nflip << 1) | (long long)st_prev);
    const int ps = (sw & W_CSTATE) ? 1 : 0;
    const long long nb = sm.cflip[t];
    sm.ckey[t] = key_prev;
    sm.cflip[t] = nflip;
    sm.nflip[t] = nb;
    sw = (DBL ? (lb ? W_LB : 0) : (sw & W_LB)) | W_CVALID | (st_prev ? W_CSTATE : 0);
    sm.sw[t] = sw;
    if (ps != st_prev) {
        if (ps) sm.since[t] = (long long)s;
        else sm.sc1[t] += (long long)s - sm.since[t];
        sm.state[t] = ps;
    }
    sm.cell[t] = cell;
    if (evm & EV_TPT) {
        sm.bits[t] = bits & ~(B_TPT_UP | B_TPT2_UP);
        sm.tpt[t] = (long long)s;
        sm.tpt2[t] = (long long)s;
        sm.tpt2w[t] = well;
    }
    xp = xn;
    if (dc > 0) { lo = -hL; hi = J.edge_lo; }
    else { lo = J.edge_hi; hi = hL; }
    F = 0.0f;
    lrel = steps_to_special(J, s, sm.nxf[t], nb);
    return 2;
}

}  // namespace

#ifndef LDP_FP32_MIN_BLOCKS
// Resident 256-thread blocks per SM the register budget is sized for: 3
// gives the hot loop 80 registers without spills (measured faster than 4
// blocks at 64 registers, which spill in the loop).
#define LDP_FP32_MIN_BLOCKS 3
#endif

// The persistent loop of one model type for the calling warp: its slots'
// trajectories (and new ones claimed from queue q) for up to quad_budget
// blocks of four steps.  Returns the blocks run; *drained is set when it
// stopped early because every lane of the warp was idle and the queue had
// nothing left for it.  Slot state is loaded at entry and saved at exit.
template <bool DBL, bool OVER>
__device__ __forceinline__ uint32_t persistent_run(const QueueDev& q, const SlotsDev& S, RareSm& sm,
                                                   uint32_t quad_budget, bool* drained) {
    const int t = threadIdx.x;
    const int64_t slot = (int64_t)blockIdx.x * blockDim.x + t;
    const unsigned lane = t & 31u;
    const float kInf = __int_as_float(0x7f800000);

    // ---- hot lane state (registers); the rest lives in sm ----
    int job = (slot < S.nslots) ? S.job[slot] : -1;
    uint64_t j = 0;                 // next block of four steps: 4j+1 .. 4j+4
    float xp = 0.f, rv = 0.f, F = 0.f, lo = -kInf, hi = kInf;
    int left = kLeftMax;
    float c1 = 0.f, c2 = 0.f, c3 = 0.f;
    sm.job[t] = job;

    // Per-job constants into registers; band, force and countdown from the
    // position.  s = next step.
    auto bind = [&](uint32_t traj, uint64_t s) {
        const JobF& J = q.jobs[job];
        if (OVER) c1 = J.c_drift;
        else { c1 = J.hdt_invM; c2 = J.hdt; c3 = J.expg; }
        sm.c1[t] = c1;
        sm.traj[t] = traj;
        sm.kn[t] = J.bm_k;
        sm.key0[t] = J.key0;
        sm.key1[t] = J.key1;
        sm.gtraj[t] = traj + J.g0;
        const int state = sm.state[t];
        band_of<DBL>(J, xp, &lo, &hi);
        F = force_of<DBL>(J, xp, state);
        left = steps_to_special(J, s - 1, sm.nxf[t], sm.nflip[t]);
        j = (s - 1) >> 2;
    };

    if (job >= 0) {
        const JobF& J = q.jobs[job];
        const uint32_t traj = (uint32_t)S.traj[slot];
        const uint64_t s = (uint64_t)S.step[slot];
        xp = S.xp[slot];
        rv = S.rv[slot];
        sm.cell[t] = S.cell[slot];
        const int st = S.st[slot];
        sm.state[t] = st & 1;
        sm.sw[t] = st >> 1;
        sm.bits[t] = (uint32_t)J.bits[traj];
        sm.init0[t] = J.init_idx0[traj];
        sm.idx2[t] = J.idx2_0[traj];
        sm.tpt2w[t] = J.tpt2_well[traj];
        sm.fpt[t] = J.fpt_last[traj];
        sm.fpt2[t] = J.fpt2_last[traj];
        sm.tpt[t] = J.tpt_last[traj];
        sm.tpt2[t] = J.tpt2_last[traj];
        sm.ckey[t] = S.ckey[slot];
        sm.cflip[t] = S.cflip[slot];
        sm.sc1[t] = S.sc1[slot];
        sm.since[t] = S.since[slot];
        sm.cgw[t] = S.cgw[slot];
        sm.fidx[t] = S.fidx[slot];
        sm.nxf[t] = S.nxf[slot];
        sm.nflip[t] = S.nflip[slot];
        bind(traj, s);
    }

    bool dry = false;   // the queue had nothing left for this warp
    uint32_t it = 0;
    for (; it < quad_budget; ++it) {
        // ---- warp-aggregated refill of idle lanes ----
        const unsigned idle = __ballot_sync(kFull, job < 0);
        if (__builtin_expect(idle != 0, 0)) {
            const bool need = job < 0 && !dry && slot < S.nslots;
            const unsigned m = __ballot_sync(kFull, need);
            if (m) {
                const int leader = __ffs(m) - 1;
                unsigned long long base = 0, got = 0;
                if ((int)lane == leader) {
                    // One fetch-and-add per warp.  A claim that runs past the
                    // tail gets the part below it; the overshoot of head is
                    // clamped back to the tail when more work is published
                    // (fp32_publish_kernel, stream-ordered between launches).
                    const unsigned long long tail = *(volatile unsigned long long*)q.tail;
                    if (*(volatile unsigned long long*)q.head < tail) {
                        const unsigned long long want = (unsigned long long)__popc(m);
                        const unsigned long long old = atomicAdd(q.head, want);
                        if (old < tail) {
                            base = old;
                            got = min(want, tail - old);
                        }
                    }
                }
                base = __shfl_sync(kFull, base, leader);
                got = __shfl_sync(kFull, got, leader);
                if (got < (unsigned long long)__popc(m)) dry = true;
                if (need) {
                    const unsigned rank = __popc(m & ((1u << lane) - 1u));
                    if (rank < got) {
                        const uint32_t traj = (uint32_t)f_resolve(q.range_end, q.range_job, q.range_first, q.nranges,
                                                   (int64_t)(base + rank), &job);
                        const JobF* Jn = &q.jobs[job];
                        f_start<DBL, OVER>(Jn, S.ring, S.nslots, S.ring_slots, slot, traj, &sm, t, &xp, &rv,
                                           &sm.cell[t], &sm.state[t], &sm.sw[t]);
                        sm.job[t] = job;
                        bind(traj, Jn->step0);
                        if (Jn->nsteps == 0) {
                            retire_lane<OVER>(*Jn, S.retired, sm, t, 0, xp, rv, 0);
                            job = -1;
                            sm.job[t] = -1;
                            lo = -kInf;
                            hi = kInf;
                            F = 0.f;
                            left = kLeftMax;
                        }
                    }
                }
            }
            if (__all_sync(kFull, job < 0)) {
                if (dry || m == 0) {
                    *drained = true;
                    break;
                }
                continue;
            }
            if (job < 0) continue;
        }

        // ---- one Philox block, four steps ----
        const Words w = philox_wide((uint32_t)j, (uint32_t)(j >> 32), sm.gtraj[t], TAG_STEP, sm.key0[t], sm.key1[t]);
        const float kn = sm.kn[t];
        float nq[4];
        noise_pair(w.w0, w.w1, kn, &nq[0], &nq[1]);
        noise_pair(w.w2, w.w3, kn, &nq[2], &nq[3]);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const float nz = nq[h];
            if (OVER) {
                xp = fmaf(F, c1, xp);
                xp = xp + nz;
                xp = xp + rv;
                rv = nz;
            } else {
                rv = fmaf(F, c1, rv);
                xp = fmaf(rv, c2, xp);
                rv = fmaf(c3, rv, nz);
                xp = fmaf(rv, c2, xp);
            }
            // left counts from the quad's start: the countdown ends at this
            // sub-step when it equals h + 1 (one decrement per quad)
            if (__builtin_expect(!(xp > lo && xp < hi) || left == h + 1, 0)) {
                const uint64_t s = 4 * j + 1 + h;
                int lrel = 0;
                const int lt = light_step<DBL>(q.jobs, S, sm, t, slot, job, sm.traj[t], s, left == h + 1, xp, lo, hi, F,
                                               lrel);
                if (lt == 2) {
                    left = lrel + (h + 1);
                } else if (lt == 0) {
                    sm.xp[t] = xp;
                    sm.rv[t] = rv;
                    sm.F[t] = F;
                    sm.left[t] = left - (h + 1);
                    sm.lo[t] = lo;
                    sm.hi[t] = hi;
                    general_step<DBL, OVER>(q.jobs, &S, &sm, t, slot, s);
                    xp = sm.xp[t];
                    F = sm.F[t];
                    lo = sm.lo[t];
                    hi = sm.hi[t];
                    left = sm.left[t] + (h + 1);
                    job = sm.job[t];
                }
            }
            if (!OVER) rv = fmaf(F, c1, rv);
        }
        left -= 4;
        ++j;
    }

    if (slot >= S.nslots) return it;
    S.job[slot] = job;
    if (job >= 0) {
        const JobF& J = q.jobs[job];
        const uint32_t traj = sm.traj[t];
        S.traj[slot] = traj;
        S.step[slot] = (int64_t)(4 * j + 1);
        S.xp[slot] = xp;
        S.rv[slot] = rv;
        S.cell[slot] = sm.cell[t];
        S.st[slot] = sm.state[t] | (sm.sw[t] << 1);
        S.ckey[slot] = sm.ckey[t];
        S.cflip[slot] = sm.cflip[t];
        S.sc1[slot] = sm.sc1[t];
        S.since[slot] = sm.since[t];
        S.cgw[slot] = sm.cgw[t];
        S.fidx[slot] = sm.fidx[t];
        S.nxf[slot] = sm.nxf[t];
        S.nflip[slot] = sm.nflip[t];
        J.bits[traj] = (int32_t)sm.bits[t];
        J.init_idx0[traj] = sm.init0[t];
        J.idx2_0[traj] = sm.idx2[t];
        J.tpt2_well[traj] = sm.tpt2w[t];
        J.fpt_last[traj] = sm.fpt[t];
        J.fpt2_last[traj] = sm.fpt2[t];
        J.tpt_last[traj] = sm.tpt[t];
        J.tpt2_last[traj] = sm.tpt2[t];
    }
    return it;
}

template <bool DBL, bool OVER>
__global__ void __launch_bounds__(256, LDP_FP32_MIN_BLOCKS) fp32_persistent_kernel(
    const __grid_constant__ QueueDev q, const __grid_constant__ SlotsDev S, uint32_t quad_budget) {
    __shared__ RareSm sm;
    bool drained = false;
    persistent_run<DBL, OVER>(q, S, sm, quad_budget, &drained);
}

// All four model types in one persistent launch (the serving loop's).  A
// warp serves one type at a time -- a warp-uniform switch over the four
// instantiated loops -- with every lane's trajectory from that type's queue;
// when all its lanes are idle and that queue is dry it takes another type
// with unclaimed items, so no type's work waits for another type's launch.
// Its pick is the type its SM serves (sm_type) while that queue has work,
// else the first type with work round robin from the SM's index, which then
// becomes the SM's type: the warps of an SM converge on one type, whose code
// alone then fills the SM's instruction caches (warps of different types on
// one SM measured as stalls on instruction fetch).  The warp's type is kept
// across launches in wtype (-1: none).  A warp ends its launch when the
// budget is spent, no queue has work, or eight type changes in a row found
// nothing to claim (claims raced away by other warps).
template <int kUnused>
__global__ void __launch_bounds__(256, LDP_FP32_MIN_BLOCKS) fp32_mixed_kernel(const __grid_constant__ MixedDev m,
                                                                               uint32_t quad_budget) {
    __shared__ RareSm sm;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int type = m.wtype[w];
    uint32_t left = quad_budget;
    int empty_picks = 0;
    while (left > 0) {
        if (type < 0) {
            int pick = -1;
            if ((threadIdx.x & 31) == 0) {
                unsigned smid;
                asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
                volatile int32_t* home = m.sm_type + (smid & (unsigned)(kMixedSmTypes - 1));
                auto has_work = [&](int tt) {
                    const unsigned long long h = *(volatile const unsigned long long*)m.q[tt].head;
                    const unsigned long long tl = *(volatile const unsigned long long*)m.q[tt].tail;
                    return h < tl;
                };
                const int pref = *home;
                if (pref >= 0 && pref < 4 && has_work(pref)) {
                    pick = pref;
                } else {
                    for (int k = 0; k < 4; ++k) {
                        const int tt = (int)((smid + (unsigned)k) & 3u);
                        if (has_work(tt)) {
                            pick = tt;
                            break;
                        }
                    }
                    if (pick >= 0) *home = pick;
                }
            }
            pick = __shfl_sync(kFull, pick, 0);
            if (pick < 0) break;
            type = pick;
        }
        bool drained = false;
        uint32_t used;
        switch (type) {
            case 0: used = persistent_run<false, false>(m.q[0], m.S, sm, left, &drained); break;
            case 1: used = persistent_run<false, true>(m.q[1], m.S, sm, left, &drained); break;
            case 2: used = persistent_run<true, false>(m.q[2], m.S, sm, left, &drained); break;
            default: used = persistent_run<true, true>(m.q[3], m.S, sm, left, &drained); break;
        }
        left -= (used < left) ? used : left;
        if (drained) {
            type = -1;
            if (used == 0) {
                if (++empty_picks >= 8) break;
            } else {
                empty_picks = 0;
            }
        }
    }
    if ((threadIdx.x & 31) == 0 && w < m.nwarps) m.wtype[w] = type;
}

// Publishes item ranges [.., new_tail): clamps the head (claims may have run
// past the old tail) and moves the tail; one thread, between launches.
__global__ void fp32_publish_kernel(unsigned long long* head, unsigned long long* tail, int32_t* nranges,
                                    unsigned long long new_tail, int32_t new_nranges) {
    const unsigned long long t = *tail;
    if (*head > t) *head = t;
    *tail = new_tail;
    *nranges = new_nranges;
}

int launch_fp32_publish(const QueueDev& q, unsigned long long new_tail, int32_t new_nranges, void* stream) {
    fp32_publish_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(q.head, q.tail, q.nranges, new_tail, new_nranges);
    return (int)cudaGetLastError();
}

template <bool DBL, bool OVER>
static cudaError_t fp32_kernel_attrs() {
    // The kernel reads little global memory: give shared memory the whole
    // carveout so that the occupancy the grid is sized for is resident.
    return cudaFuncSetAttribute(fp32_persistent_kernel<DBL, OVER>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
}

int fp32_blocks_per_sm(bool dbl, bool over, int block) {
    int n = 0;
    cudaError_t e;
    if (dbl) e = over ? fp32_kernel_attrs<true, true>() : fp32_kernel_attrs<true, false>();
    else e = over ? fp32_kernel_attrs<false, true>() : fp32_kernel_attrs<false, false>();
    if (e != cudaSuccess) return 0;
    if (dbl) e = over ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<true, true>, block, 0)
                      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<true, false>, block, 0);
    else e = over ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<false, true>, block, 0)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_persistent_kernel<false, false>, block, 0);
    return e == cudaSuccess ? n : 0;
}

int fp32_mixed_blocks_per_sm(int block) {
    int n = 0;
    cudaError_t e = cudaFuncSetAttribute(fp32_mixed_kernel<0>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp32_mixed_kernel<0>, block, 0);
    return e == cudaSuccess ? n : 0;
}

int launch_fp32_mixed(const MixedDev& m, uint32_t pair_budget, int grid, int block, void* stream) {
    const uint32_t quad_budget = pair_budget > 1 ? pair_budget / 2 : 1;
    if (block != 256 || (int64_t)grid * block > m.S.nslots) return (int)cudaErrorInvalidValue;
    fp32_mixed_kernel<0><<<grid, block, 0, (cudaStream_t)stream>>>(m, quad_budget);
    return (int)cudaGetLastError();
}

int launch_fp32_persistent(bool dbl, bool over, const QueueDev& q, const SlotsDev& s, uint32_t pair_budget, int grid,
                           int block, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t quad_budget = pair_budget > 1 ? pair_budget / 2 : 1;   // blocks of four steps
    if (block > kMaxBlock) return (int)cudaErrorInvalidValue;
    if (dbl) {
        if (over) fp32_persistent_kernel<true, true><<<grid, block, 0, st>>>(q, s, quad_budget);
        else fp32_persistent_kernel<true, false><<<grid, block, 0, st>>>(q, s, quad_budget);
    } else {
        if (over) fp32_persistent_kernel<false, true><<<grid, block, 0, st>>>(q, s, quad_budget);
        else fp32_persistent_kernel<false, false><<<grid, block, 0, st>>>(q, s, quad_budget);
    }
    return (int)cudaGetLastError();
}

}  // namespace ldp
