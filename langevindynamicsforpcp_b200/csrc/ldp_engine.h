// ldp_engine.h -- per-job constants and device-resident trajectory state.
//
// KConst is the restatement of the reference's per-trial constants
// (IntegrateInitializeVariables, src/langevinDynamicsSingleBarrier.h:1520-1618
// and 2812-2824; src/langevinDynamicsDoubleBarrier.h:1733-1937 and
// 3427-3439).  It is computed once on the host (prepare_kconst) and passed by
// value to every kernel.
//
// TrajState holds one structure-of-arrays per trajectory field in HBM.  The
// trajectory kernels load a trajectory into registers at the start of a
// launch and store it back at the end, so HBM is touched only at launch
// boundaries, on the rare cell-table events, and for saved frames.
#pragma once
#include <cstdint>
#include "../../include/ldp.h"

namespace ldp {

// bits of TrajState::bits
enum : uint32_t {
    B_FPT_UP = 1u << 0, B_FPT2_UP = 1u << 1, B_TPT_UP = 1u << 2, B_TPT2_UP = 1u << 3,
    B_WT_PASSED = 1u << 4, B_DONE = 1u << 5, B_INIT0 = 1u << 6, B_INIT1 = 1u << 7,
    B_CG0 = 1u << 8  // B_CG0 << j: FPTCG entry j still waits for its first bottom
};

struct KConst {
    int32_t dbl, over, eta, eq, rv, rs, us, init_state;
    int32_t wt, fpt, tpt, cg, n_cg;
    int32_t cg_size[LDP_MAX_CG];
    int32_t write_x, fp_mode, lanes, nruns, slots, at_bottom;
    uint32_t key0, key1;
    uint32_t g0;             // stream index of the job's trajectory 0 (first_rank * runs * lanes)
    double x0, v0, dt, L, invL;
    double w, Hs[2], slope[2];
    double xb[2], lo0, hi1, xc;
    double Hd[2][2], sN[2][2], sP[2][2], iN[2][2], iP[2][2];
    double c_drift, sig_r, invM, hdt, expg, sig_v, mhalf, sig_v0;
    uint64_t T_eq, T_as[2];
    double ln1m[2];          // log(1 - per-step flip probability) by state; 0: never flips
    double a_lap, c_lap[2], p_first, p_cell0;
    uint64_t nsteps, freq_save, step_cap;
    int64_t nframe, tick_cap, ev_cap;
    // FP32 cell-local copies (FP32 batched path)
    float fL, fhalfL, fw, fslope[2], fxb[2], flo0, fhi1, fxc;
    float fsN[2][2], fsP[2][2];
    float fc_drift, fsig_r, fhdt_invM, fhdt, fexpg, fsig_v;
};

struct TrajState {
    int64_t n;
    double *x, *v, *F, *rprev;
    int64_t *cell, *well;
    int32_t *state, *lb, *bits;
    double *fpt_last, *fpt2_last, *tpt_last, *tpt2_last;
    int64_t *init_idx0, *init_idx1, *idx2_0, *idx2_1, *tpt2_well, *wt_tick;
    int64_t* nflip;     // step of the current barrier's next flip
    double *cg_last;    // [LDP_MAX_CG][n]
    int64_t *cg_well;   // [LDP_MAX_CG][n]
    int64_t *counts;    // [LDP_NCOUNT][n]
    double *sums;       // [LDP_NSUM][n]
    int32_t *state0;
    double *v0;
    int64_t *ring_tag, *ring_data;  // [slots][n]
    int64_t *ticks;     // [n][tick_cap]
    double *ev;         // per-event lists [LDP_E_CG0 + n_cg][n][ev_cap]
    uint8_t *ev_st;     // FPT event barrier states [n][ev_cap]
    double *fx, *fv, *ff, *fb, *fpe, *fke, *fst;  // frames [nframe][n]
};

// Host side (ldp_prepare.cpp).
void prepare_kconst(const ldp_params& p, const ldp_job_opts& o, uint32_t seed, KConst* k);
uint64_t effective_steps(const ldp_params& p);
int64_t frame_count(const ldp_params& p);

// Launchers (ldp_fp64.cu); return cudaError_t as int.
int launch_fp64_init(const KConst& k, const TrajState& st, int64_t g0, int block, void* stream);
int launch_fp64_steps(const KConst& k, const TrajState& st, int64_t g0, uint64_t s_begin, uint64_t s_end,
                      int block, void* stream);
// Latency mode (few long trajectories): one CTA of a producer and a consumer
// warp per trajectory, the same results bit for bit.
int launch_fp64_latency(const KConst& k, const TrajState& st, int64_t g0, uint64_t s_begin, uint64_t s_end,
                        void* stream);
// Group mode: a CTA of 32 trajectories, producer warps drawing ahead of a
// consumer warp (same results bit for bit).
int launch_fp64_group(const KConst& k, const TrajState& st, int64_t g0, uint64_t s_begin, uint64_t s_end,
                        void* stream);

}  // namespace ldp
