/*
 * ldp_oracle.c -- CPU oracle for the trajectory hot path (test
 * infrastructure only; see ldp_oracle.h).
 *
 * Each function restates a piece of the reference; the citation names the
 * reference lines it follows (S.h = src/langevinDynamicsSingleBarrier.h,
 * D.h = src/langevinDynamicsDoubleBarrier.h).  Where the reference draws
 * from MKL VSL banks, this oracle draws from the per-trajectory Philox
 * streams the product defines (ctr = {a, b, trajectory, tag},
 * key = {seed, job}); the draw points stay where the reference has them.
 *
 * Build with -ffp-contract=off: every a*b+c below is two roundings unless it
 * is written as fma(), exactly as in the device FP64 path.
 */
#include "ldp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TAG_STEP 0u
#define TAG_INIT 1u
#define TAG_CATCHUP 2u
#define TAG_CELL 3u
#define TAG_FLIP 4u

/* ---------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11, "Parallel random
 * numbers: as easy as 1, 2, 3").  Replaces the MKL VSL MT19937 banks of
 * src/RANDOMNUMBER.cpp:70-340.                                            */
/* ---------------------------------------------------------------------- */
void ldpo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void philox_at(uint64_t a, uint32_t g, uint32_t tag, const uint32_t key[2], uint32_t w[4]) {
    uint32_t ctr[4] = {(uint32_t)a, (uint32_t)(a >> 32), g, tag};
    ldpo_philox4x32_10(ctr, key, w);
}

/* ---------------------------------------------------------------------- */
/* Deterministic FP64 elementary functions (written from textbook methods;
 * the device FP64 path evaluates the same operation sequence).            */
/* ---------------------------------------------------------------------- */
static const double LN2_HI = 6.93147180559945286227e-01;   /* nearest double to ln 2 */
static const double LN2_LO = 2.31904681384629955842e-17;   /* ln 2 - LN2_HI          */
static const double TWO_PI_HI = 6.28318530717958623200e+00;
static const double TWO_PI_LO = 2.44929359829470635445e-16;

static uint64_t as_u64(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
static double as_f64(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }

/* log(u), u positive normal: u = m 2^e, m in [sqrt(1/2), sqrt(2)),
 * log m = 2 atanh(f), f = (m-1)/(m+1), atanh by its odd power series. */
double ldpo_log(double u) {
    uint64_t b = as_u64(u);
    int64_t e = (int64_t)((b >> 52) & 0x7ff) - 1023;
    double m = as_f64((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if (m > 1.41421356237309504880) { m = m * 0.5; e += 1; }
    double f = (m - 1.0) / (m + 1.0);
    double f2 = f * f;
    double s = 1.0 / 23.0;
    s = fma(s, f2, 1.0 / 21.0);
    s = fma(s, f2, 1.0 / 19.0);
    s = fma(s, f2, 1.0 / 17.0);
    s = fma(s, f2, 1.0 / 15.0);
    s = fma(s, f2, 1.0 / 13.0);
    s = fma(s, f2, 1.0 / 11.0);
    s = fma(s, f2, 1.0 / 9.0);
    s = fma(s, f2, 1.0 / 7.0);
    s = fma(s, f2, 1.0 / 5.0);
    s = fma(s, f2, 1.0 / 3.0);
    double logm = fma(2.0 * f * f2, s, 2.0 * f);
    double de = (double)e;
    return fma(de, LN2_HI, fma(de, LN2_LO, logm));
}

/* sin(2 pi t), cos(2 pi t) for t in [0, 1): quadrant from rint(4t), the
 * rest by Taylor series on [-pi/4, pi/4]. */
void ldpo_sincos2pi(double t, double *sn, double *cs) {
    double q = rint(t * 4.0);
    double f = t - q * 0.25;
    double x = fma(f, TWO_PI_HI, f * TWO_PI_LO);
    double x2 = x * x;
    double ps = -1.0 / 121645100408832000.0;         /* -1/19! */
    ps = fma(ps, x2, 1.0 / 355687428096000.0);       /*  1/17! */
    ps = fma(ps, x2, -1.0 / 1307674368000.0);        /* -1/15! */
    ps = fma(ps, x2, 1.0 / 6227020800.0);            /*  1/13! */
    ps = fma(ps, x2, -1.0 / 39916800.0);             /* -1/11! */
    ps = fma(ps, x2, 1.0 / 362880.0);                /*  1/9!  */
    ps = fma(ps, x2, -1.0 / 5040.0);                 /* -1/7!  */
    ps = fma(ps, x2, 1.0 / 120.0);                   /*  1/5!  */
    ps = fma(ps, x2, -1.0 / 6.0);                    /* -1/3!  */
    double s = fma(x * x2, ps, x);
    double pc = 1.0 / 2432902008176640000.0;         /*  1/20! */
    pc = fma(pc, x2, -1.0 / 6402373705728000.0);     /* -1/18! */
    pc = fma(pc, x2, 1.0 / 20922789888000.0);        /*  1/16! */
    pc = fma(pc, x2, -1.0 / 87178291200.0);          /* -1/14! */
    pc = fma(pc, x2, 1.0 / 479001600.0);             /*  1/12! */
    pc = fma(pc, x2, -1.0 / 3628800.0);              /* -1/10! */
    pc = fma(pc, x2, 1.0 / 40320.0);                 /*  1/8!  */
    pc = fma(pc, x2, -1.0 / 720.0);                  /* -1/6!  */
    pc = fma(pc, x2, 1.0 / 24.0);                    /*  1/4!  */
    pc = fma(pc, x2, -0.5);                          /* -1/2!  */
    double c = fma(x2, pc, 1.0);
    int qi = ((int)q) & 3;
    switch (qi) {
        case 0: *sn = s; *cs = c; break;
        case 1: *sn = c; *cs = -s; break;
        case 2: *sn = -s; *cs = -c; break;
        default: *sn = -c; *cs = s; break;
    }
}

/* expm1(x) for x <= 0: x = k ln2 + r (Cody-Waite, |r| <= ln2/2), Taylor
 * series for expm1(r), then 2^k (expm1(r) + 1) - 1. */
double ldpo_expm1(double x) {
    if (x < -60.0) return -1.0;
    double k = rint(x * 1.44269504088896340736);
    double r = fma(-k, LN2_HI, x);
    r = fma(-k, LN2_LO, r);
    double p = 1.0 / 6227020800.0;                   /* 1/13! */
    p = fma(p, r, 1.0 / 479001600.0);
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    double e = fma(r * r, p, r);
    if (k == 0.0) return e;
    double s = ldexp(1.0, (int)k);
    return fma(s, e, s - 1.0);
}

/* Steps to the next flip of a barrier flipping with probability p per step
 * (ln1m = log(1 - p)): W = 1 + floor(ln U / ln(1 - p)), U in (0, 1] from the
 * 64-bit word pair -- the geometric waiting time of the reference's per-step
 * Bernoulli flips (S.h:2010-2015); UINT64_MAX when the barrier never flips. */
uint64_t ldpo_flip_wait(uint32_t hi, uint32_t lo, double ln1m) {
    if (!(ln1m < 0.0)) return UINT64_MAX;
    const double u = ((double)(((uint64_t)hi << 32) | lo) + 1.0) * 0x1p-64;
    const double q = ldpo_log(u) / ln1m;
    if (!(q < 0x1p62)) return UINT64_MAX;
    return 1ull + (uint64_t)floor(q);
}

/* Step of the next flip drawn at step s: s + W, clamped to LDPO_NEVER. */
int64_t ldpo_schedule(uint64_t s, uint32_t hi, uint32_t lo, double ln1m) {
    const uint64_t wt = ldpo_flip_wait(hi, lo, ln1m);
    return (wt >= (uint64_t)LDPO_NEVER - s) ? LDPO_NEVER : (int64_t)(s + wt);
}

uint64_t ldpo_prob_to_u64(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return UINT64_MAX;
    return (uint64_t)ldexp(p, 64);
}

/* Box-Muller pair from two 32-bit words. */
static void gauss_pair(uint32_t wa, uint32_t wb, double *z0, double *z1) {
    double u1 = ((double)wa + 1.0) * 0x1p-32;
    double u2 = (double)wb * 0x1p-32;
    double r = sqrt(-2.0 * ldpo_log(u1));
    double sn, cs;
    ldpo_sincos2pi(u2, &sn, &cs);
    *z0 = r * cs;
    *z1 = r * sn;
}

/* ---------------------------------------------------------------------- */
/* Per-job constants: IntegrateInitializeVariables, S.h:1520-1618 and
 * S.h:2812-2824; D.h:1733-1937 and D.h:3427-3439.                         */
/* ---------------------------------------------------------------------- */
typedef struct {
    int dbl, over, eta, eq, rv, rs, us, init_state;
    int wt, fpt, tpt, cg, n_cg, cg_size[LDP_MAX_CG];
    double x0, v0, dt, L, invL, halfL;
    double w, Hs[2], slope[2];
    double xb[2], lo0, hi1, xc, Hd[2][2], sN[2][2], sP[2][2], iN[2][2], iP[2][2];
    double c_drift, sig_r, invM, hdt, expg, sig_v, mhalf, sig_v0;
    uint64_t T_eq, T_as[2];
    double ln1m[2];    /* log(1 - per-step flip probability) by state; 0: never */
    double a_lap, c_lap[2];
    double p_first, p_cell0;
    int at_bottom;
    uint64_t nsteps, freq_save;
    int64_t nframe;
    int write_x;
} ocst;

uint64_t ldpo_effective_steps(const ldp_params *p) {
    if (p->freq_save >= 10) return (p->number_of_steps / p->freq_save) * p->freq_save;
    return p->number_of_steps;
}

int64_t ldpo_nframe(const ldp_params *p) {
    /* CalculateNumberOfFrame(numberOfStep + numberOfStepPrevious), S.h:3220 */
    return (int64_t)((p->number_of_steps + p->number_of_previous_steps) / p->freq_save + 1);
}

static void prepare(const ldp_params *p, ocst *k) {
    memset(k, 0, sizeof(*k));
    k->dbl = p->model == LDP_MODEL_DOUBLE;
    k->over = p->overdamped != 0;
    k->eta = p->tau != 0.0;
    k->eq = p->eq != 0;
    k->rv = p->randomize_v != 0;
    k->rs = p->randomize_states != 0;
    k->us = p->uniform_initial_states != 0;
    k->init_state = p->initial_state;
    k->wt = p->waiting_time != 0 && !k->dbl;
    k->fpt = p->fpt != 0;
    k->tpt = p->tpt != 0 && !k->dbl;
    k->cg = p->fptcg != 0;
    k->n_cg = p->n_cg;
    for (int j = 0; j < p->n_cg && j < LDP_MAX_CG; ++j) k->cg_size[j] = p->cg_sizes[j];
    k->x0 = p->x0;
    k->v0 = p->v0;
    k->dt = p->timestep;
    k->L = p->periodic_length;
    k->invL = 1.0 / k->L;
    k->halfL = k->L * 0.5;
    k->write_x = p->write_x != 0;
    if (!k->dbl) {
        k->w = p->barrier_half_width[0];
        k->Hs[0] = p->barrier_heights[0][0];
        k->Hs[1] = p->barrier_heights[0][1];
        k->slope[0] = k->Hs[0] / k->w;
        k->slope[1] = k->Hs[1] / k->w;
    } else {
        double x1b = p->barrier_position[0], w1 = p->barrier_half_width[0];
        double x2b = p->barrier_position[1], w2 = p->barrier_half_width[1];
        double y1 = p->barrier_heights[0][0], y2 = p->barrier_heights[1][0];
        /* GetXc, D.h:1722-1732 */
        double x1h = x1b + w1, x2l = x2b - w2;
        double xc = (x1h * y1 * (x2b - x2l) + x2l * y2 * (x1h - x1b)) /
                    (y1 * (x2b - x2l) + y2 * (x1h - x1b));
        double yc = (x1h - xc) / (x1h - x1b) * y1;
        k->xc = xc;
        k->xb[0] = x1b;
        k->xb[1] = x2b;
        double lo[2] = {x1b - w1, x2b - w2}, hi[2] = {x1b + w1, x2b + w2};
        k->lo0 = lo[0];
        k->hi1 = hi[1];
        double xb_xl[2] = {k->xb[0] - lo[0], k->xb[1] - lo[1]};
        double xh_xb[2] = {hi[0] - k->xb[0], hi[1] - k->xb[1]};
        for (int s = 0; s < 2; ++s) {
            double h0 = p->barrier_heights[0][s], h1 = p->barrier_heights[1][s];
            k->Hd[0][s] = h0;
            k->Hd[1][s] = h1;
            /* D.h:1863-1899 */
            k->sN[0][s] = h0 / xb_xl[0];
            k->sP[0][s] = (yc - h0) / (xc - k->xb[0]);
            k->sN[1][s] = (h1 - yc) / (k->xb[1] - xc);
            k->sP[1][s] = 0.0 - h1 / xh_xb[1];
            k->iN[0][s] = 0.0 - h0 * (lo[0] / xb_xl[0]);
            k->iP[0][s] = (xc * h0 - yc * k->xb[0]) / (xc - k->xb[0]);
            k->iN[1][s] = (yc * k->xb[1] - xc * h1) / (k->xb[1] - xc);
            k->iP[1][s] = h1 * (hi[1] / xh_xb[1]);
        }
    }
    double m = p->mass, g = p->gamma, kT = p->kb * p->temperature;
    k->invM = 1.0 / m;
    k->hdt = k->dt * 0.5;
    k->mhalf = m * 0.5;
    k->expg = exp(-g * k->dt);
    k->sig_v = sqrt(p->kb * p->temperature / m * (1.0 - exp(-2.0 * g * k->dt)));
    double mgi = 1.0 / (m * g);
    k->c_drift = k->dt * mgi;
    k->sig_r = sqrt(p->kb * p->temperature * mgi * k->dt * 0.5);
    k->sig_v0 = sqrt(p->kb * p->temperature / m);
    (void)kT;
    double K = p->eq_constant;
    if (k->eq) {
        k->a_lap = -2.0 * k->dt / p->tau;
        k->T_eq = k->eta ? ldpo_prob_to_u64(0.5 * -expm1(-2.0 * k->dt / p->tau)) : 0;
        k->c_lap[0] = k->c_lap[1] = 0.5;
        k->p_first = 0.5;
    } else {
        k->a_lap = -(K + 1.0) * k->dt / p->tau;
        double e = -expm1(k->a_lap);
        k->T_as[0] = k->eta ? ldpo_prob_to_u64(K / (1.0 + K) * e) : 0;
        k->T_as[1] = k->eta ? ldpo_prob_to_u64(1.0 / (1.0 + K) * e) : 0;
        k->c_lap[0] = K / (1.0 + K);
        k->c_lap[1] = 1.0 / (1.0 + K);
        k->p_first = 1.0 / (1.0 + K);
    }
    /* Waiting times between flips: geometric in the per-step probability. */
    for (int s = 0; s < 2; ++s) {
        double pf = 0.0;
        if (k->eta) pf = k->eq ? 0.5 * -expm1(-2.0 * k->dt / p->tau) : k->c_lap[s] * -expm1(k->a_lap);
        k->ln1m[s] = (pf > 0.0) ? log1p(-pf) : 0.0;
    }
    k->p_cell0 = 1.0 / (1.0 + K);   /* BarrierStatus::Initialize, S.h:90 */
    /* Math::Modulo(X0, L) == L/2, S.h:2184, src/mathdef.h:20 */
    k->at_bottom = fmod(fmod(k->x0, k->L) + k->L, k->L) == k->halfL;
    k->nsteps = ldpo_effective_steps(p);
    k->freq_save = p->freq_save;
    k->nframe = ldpo_nframe(p);
}

/* GenerateLog10Scale, src/MOLUTILITY.cpp:59-73 (with the frame count of
 * S.h:3220 that includes NUMBEROFPREVIOUSSTEPS). */
int64_t ldpo_lags(const ldp_params *p, int64_t *lags, int64_t cap) {
    uint64_t nf = (p->number_of_steps + p->number_of_previous_steps) / p->freq_save + 1;
    double ts = p->timestep * (double)p->freq_save;
    double step = 1.0 / (double)p->number_of_log_samples;
    double maxTime = ts * (double)(nf - 1000);
    double t0 = log10(ts), t1 = log10(maxTime);
    int64_t n = 0;
    if (cap > 0) lags[0] = 0;
    n = 1;
    for (double t = t0; t <= t1; t += step) {
        int64_t iv = (int64_t)(uint64_t)round(pow(10.0, t) / ts);
        if (lags[n - 1] != iv) {
            if (n < cap) lags[n] = iv;
            ++n;
            if (n > cap) return -1;
        }
    }
    return n;
}

/* ---------------------------------------------------------------------- */
/* Per-trajectory state                                                    */
/* ---------------------------------------------------------------------- */
typedef struct {
    int64_t *tag;   /* ring of visited cells: key, or INT64_MIN if empty */
    int64_t *data;  /* stamp << 1 | state                                */
    int slots;
} ring;

typedef struct {
    double x, v, F, E, rprev, barrier;
    int64_t cell, well;
    int lb, state;
    /* statistics state (InitializeStatistics, S.h:2166-2333) */
    int wt_passed;
    int64_t wt_tick;
    int fpt_up, fpt2_up, tpt_up, tpt2_up;
    double fpt_last, fpt2_last, tpt_last, tpt2_last;
    double init_state[2];
    int64_t init_idx[2], idx2[2], tpt2_well;
    int cg_up[LDP_MAX_CG];
    double cg_last[LDP_MAX_CG];
    int64_t cg_well[LDP_MAX_CG];
} tstate;

/* Appends an event duration to list `list` of trajectory i (the reference's
 * push_back on its per-lane vectors, S.h:2391, 2447, 2504, 2524, 2580); a
 * full list flags the trajectory. */
static void ev_push(const ldpo_cfg *c, ldp_traj_results *out, int64_t n, int64_t i, int list, int64_t cnt, double d,
                    uint32_t *flags) {
    if (c->event_cap <= 0) return;
    if (cnt < c->event_cap) {
        if (out->events) out->events[((int64_t)list * n + i) * c->event_cap + cnt] = d;
    } else {
        *flags |= LDP_FLAG_EVENT_OVERFLOW;
    }
}

static int64_t cell_key(const ocst *k, int64_t cell, int lb) {
    return k->dbl ? cell * 2 + lb : cell;
}

static int default_state(const ocst *k, const ldpo_cfg *c, const ldp_params *p, const uint32_t key[2],
                         uint32_t g, int64_t ck) {
    if (k->us) {
        /* UNIFORMINITALSTATES: S.h:1377-1380 hands BarrierStatus the state
         * array as it stood before this trial's draw (the previous trial's
         * initial state, 0 for trial 0); D.h:1576-1578 hands INITIALSTATE. */
        if (k->dbl) return k->init_state;
        int64_t lanes = c->lanes;
        int64_t trial = ((int64_t)g / lanes) % p->number_of_runs;
        if (trial == 0) return 0;
        uint32_t gp = g - (uint32_t)lanes;
        if (!k->rs) return k->init_state;
        uint32_t w[4];
        philox_at(0, gp, TAG_INIT, key, w);
        return ((double)w[0] * 0x1p-32 <= k->p_first) ? 0 : 1;
    }
    uint32_t w[4];
    philox_at((uint64_t)ck, g, TAG_CELL, key, w);
    return ((double)w[0] * 0x1p-32 < k->p_cell0) ? 0 : 1;   /* S.h:90-94 */
}

/* A cell-table entry: the barrier's state when it was left and its pending
 * flip step (the first flip after it was left); *found = 0 for a cell never
 * visited (state drawn as at creation, step 0: m_UserData.m_iStep stays 0,
 * S.h:1375). */
static void ring_load(const ocst *k, const ldpo_cfg *c, const ldp_params *p, const uint32_t key[2], uint32_t g,
                      ring *r, int64_t ck, int *state, int64_t *nflip, int *found) {
    int slot = (int)(ck & (r->slots - 1));
    if (r->tag[slot] == ck) {
        *state = (int)(r->data[slot] & 1);
        *nflip = r->data[slot] >> 1;
        *found = 1;
    } else {
        *state = default_state(k, c, p, key, g, ck);
        *nflip = 0;
        *found = 0;
    }
}

static void ring_store(ring *r, int64_t ck, int state, int64_t nflip, int64_t *evict) {
    int slot = (int)(ck & (r->slots - 1));
    if (r->tag[slot] != ck && r->tag[slot] != INT64_MIN) ++*evict;
    r->tag[slot] = ck;
    r->data[slot] = (nflip << 1) | state;
}

static int table_state(const ocst *k, const ldpo_cfg *c, const ldp_params *p, const uint32_t key[2], uint32_t g,
                       ring *r, int64_t cell) {
    int st, found;
    int64_t nf;
    ring_load(k, c, p, key, g, r, cell_key(k, cell, 0), &st, &nf, &found);
    return st;
}

/* EnergyAndForce: S.h:1292-1324 (single), D.h:1464-1522 (double). */
static void energy_force(const ocst *k, tstate *t) {
    int s = t->state;
    if (!k->dbl) {
        double xp = t->x - (double)t->cell * k->L;
        double sp = k->slope[s], sn = 0.0 - sp, H = k->Hs[s];
        int onN = (xp < 0.0) && (xp > -k->w);
        int onP = (xp < k->w) && (xp > 0.0);
        double E = 0.0, F = 0.0;
        if (onN) { E = H - xp * sn; F = sn; }
        if (onP) { E = H - xp * sp; F = sp; }
        t->E = E;
        t->F = F;
        t->barrier = H;
    } else {
        double xp = t->x - (double)t->cell * k->L;
        int onN0 = (xp < k->xb[0]) && (xp > k->lo0);
        int onP0 = (xp < k->xc) && (xp > k->xb[0]);
        int onN1 = (xp < k->xb[1]) && (xp > k->xc);
        int onP1 = (xp < k->hi1) && (xp > k->xb[1]);
        double E = 0.0, f = 0.0, B = 0.0;
        if (onN0) { E = xp * k->sN[0][s] + k->iN[0][s]; f = k->sN[0][s]; B = k->Hd[0][s]; }
        if (onP0) { E = xp * k->sP[0][s] + k->iP[0][s]; f = k->sP[0][s]; B = k->Hd[0][s]; }
        if (onN1) { E = xp * k->sN[1][s] + k->iN[1][s]; f = k->sN[1][s]; B = k->Hd[1][s]; }
        if (onP1) { E = xp * k->sP[1][s] + k->iP[1][s]; f = k->sP[1][s]; B = k->Hd[1][s]; }
        t->E = E;
        t->F = 0.0 - f;
        t->barrier = B;
    }
}

/* Index helpers: InitializePeriodicIndices / UpdatePeriodicIndices,
 * S.h:1838-1884, D.h:2156-2235. */
static void indices(const ocst *k, double x, int64_t *well, int64_t *cell, int *lb) {
    double red = x * k->invL;
    *well = (int64_t)floor(red);
    *cell = (int64_t)rint(red);
    if (k->dbl) {
        double xp = x - (double)(*cell) * k->L;
        *lb = (xp < k->xc) ? 0 : 1;
    } else {
        *lb = 0;
    }
}

typedef struct {
    int64_t *counts; /* local column pointers: counts[f] for this trajectory */
} dummy_t;

#define CNT(f) out->counts[(int64_t)(f) * n + i]
#define SUM(f) out->sums[(int64_t)(f) * n + i]

static void record(const ocst *k, const tstate *t, ldp_traj_results *out, int64_t n, int64_t i, int64_t frame) {
    if (frame >= k->nframe) return;
    int64_t o = frame * n + i;
    if (out->frames_x) out->frames_x[o] = t->x;
    if (k->write_x) {
        if (out->frames_v) out->frames_v[o] = t->v;
        if (out->frames_f) out->frames_f[o] = t->F;
        if (out->frames_barrier) out->frames_barrier[o] = t->barrier;
        if (out->frames_pe) out->frames_pe[o] = t->E;
        if (out->frames_ke) out->frames_ke[o] = k->mhalf * (t->v * t->v);
        if (out->frames_state) out->frames_state[o] = (double)t->state;
    }
}

/* FPT initial-barrier bookkeeping shared by InitializeStatistics and the
 * renew branch of UpdateStatistics (S.h:2187-2211, S.h:2364-2388). */
static void fpt_set_initial(const ocst *k, const ldpo_cfg *c, const ldp_params *p, const uint32_t key[2], uint32_t g,
                            ring *r, tstate *t) {
    if (t->well == t->cell) {
        t->init_state[0] = (double)t->state;
        t->init_idx[0] = t->cell;
        t->init_state[1] = (double)table_state(k, c, p, key, g, r, t->cell + 1);
        t->init_idx[1] = t->cell + 1;
    } else {
        t->init_state[0] = (double)table_state(k, c, p, key, g, r, t->cell - 1);
        t->init_idx[0] = t->cell - 1;
        t->init_state[1] = (double)t->state;
        t->init_idx[1] = t->cell;
    }
}

static void fpt2_set_idx(tstate *t) {
    if (t->well == t->cell) { t->idx2[0] = t->cell; t->idx2[1] = t->cell + 1; }
    else { t->idx2[0] = t->cell - 1; t->idx2[1] = t->cell; }
}

static int cg_hit(int64_t well, int size) {
    return ((int)well % size) == 0;   /* (int)round(well) % size == 0, S.h:2564 */
}

int ldpo_run(const ldp_params *p, const ldpo_cfg *c, ldp_traj_results *out) {
    ocst K;
    prepare(p, &K);
    const ocst *k = &K;
    const int64_t n = c->traj_end - c->traj_begin;
    const uint32_t key[2] = {c->seed, c->job_id};
    const int fp_mode = c->mode == LDP_MODE_FIRST_PASSAGE;
    const uint64_t nsteps = fp_mode ? c->step_cap : k->nsteps;
    ring r;
    r.slots = c->table_slots;
    r.tag = (int64_t *)malloc(sizeof(int64_t) * (size_t)r.slots);
    r.data = (int64_t *)malloc(sizeof(int64_t) * (size_t)r.slots);
    if (!r.tag || !r.data) { free(r.tag); free(r.data); return 1; }
    if (out->counts) memset(out->counts, 0, sizeof(int64_t) * LDP_NCOUNT * (size_t)n);
    if (out->sums) memset(out->sums, 0, sizeof(double) * LDP_NSUM * (size_t)n);

    for (int64_t i = 0; i < n; ++i) {
        const int64_t gg = c->traj_begin + i;
        const uint32_t g = (uint32_t)gg;
        for (int s = 0; s < r.slots; ++s) { r.tag[s] = INT64_MIN; r.data[s] = 0; }
        int64_t evict = 0, wt_n = 0;
        uint32_t flags = 0;
        int64_t cnt[LDP_NCOUNT];
        double sum[LDP_NSUM];
        memset(cnt, 0, sizeof(cnt));
        memset(sum, 0, sizeof(sum));
        tstate t;
        memset(&t, 0, sizeof(t));

        /* ---- IntegrateStep0, S.h:1619-1652 (+ S.h:2825-2832) ---- */
        t.x = k->x0;
        indices(k, t.x, &t.well, &t.cell, &t.lb);
        uint32_t w0[4];
        philox_at(0, g, TAG_INIT, key, w0);
        /* InitializeBarrierState, S.h:1885-1915 */
        if (k->rs) t.state = ((double)w0[0] * 0x1p-32 <= k->p_first) ? 0 : 1;
        else t.state = k->init_state;
        int state0 = t.state;
        /* UpdateBarrierStateEtaParamter at step 0 counts the state. */
        cnt[t.state ? LDP_C_STATE1 : LDP_C_STATE0]++;
        double zv, zr;
        gauss_pair(w0[1], w0[2], &zv, &zr);
        t.v = k->rv ? k->sig_v0 * zv : k->v0;
        double v0inst = t.v;
        int64_t nflip;
        {
            uint32_t wf[4];
            philox_at(0, g, TAG_FLIP, key, wf);
            nflip = ldpo_schedule(0, wf[0], wf[1], k->ln1m[t.state]);
        }
        energy_force(k, &t);
        /* InitializeStatistics, S.h:2166-2333 */
        t.wt_tick = 0;
        t.wt_passed = 0;
        if (k->at_bottom) {
            t.fpt_up = 0;
            t.fpt_last = 0.0;
            if (!k->dbl) fpt_set_initial(k, c, p, key, g, &r, &t);
            t.fpt2_up = 0;
            t.fpt2_last = 0.0;
            fpt2_set_idx(&t);
        } else {
            t.fpt_up = 1;
            t.fpt_last = 0.0;
            t.init_state[0] = 0.0;
            t.fpt2_up = 1;
            t.fpt2_last = 0.0;
        }
        t.tpt_up = !k->at_bottom;
        t.tpt_last = 0.0;
        t.tpt2_up = !k->at_bottom;
        t.tpt2_last = 0.0;
        t.tpt2_well = t.well;
        for (int j = 0; j < k->n_cg; ++j) {
            t.cg_last[j] = 0.0;
            t.cg_well[j] = t.well;
            t.cg_up[j] = !(k->at_bottom && cg_hit(t.well, k->cg_size[j]));
        }
        if (k->over) t.rprev = k->sig_r * zr;
        if (!fp_mode) record(k, &t, out, n, i, 0);

        /* ---- hot loop: Integrate, S.h:1403-1511 ---- */
        uint64_t s;
        uint64_t done_steps = 0;
        int stop = 0;
        double zq[4];
        for (s = 1; s <= nsteps && !stop; ++s) {
            /* one Philox block: the Gaussians of steps 4a+1 .. 4a+4 */
            const int qi = (int)((s - 1) & 3);
            if (qi == 0) {
                uint32_t w[4];
                philox_at((s - 1) >> 2, g, TAG_STEP, key, w);
                gauss_pair(w[0], w[1], &zq[0], &zq[1]);
                gauss_pair(w[2], w[3], &zq[2], &zq[3]);
            }
            const double z = zq[qi];

            const int64_t cell_prev = t.cell, well_prev = t.well;
            const int lb_prev = t.lb;
            if (k->over) {
                /* IntegrateStepEta overdamped, S.h:2860-2886 */
                double rf = k->sig_r * z;
                t.x = fma(t.F, k->c_drift, t.x);
                t.x = t.x + rf;
                t.x = t.x + t.rprev;
                t.rprev = rf;
            } else {
                /* IntegrateStepEta underdamped, S.h:1680-1695 */
                t.v = t.v + (k->invM * t.F) * k->hdt;
                t.x = t.x + t.v * k->hdt;
                t.v = k->expg * t.v + k->sig_v * z;
                t.x = t.x + t.v * k->hdt;
            }
            if (!isfinite(t.x)) { flags |= LDP_FLAG_NONFINITE; done_steps = s - 1; break; }
            indices(k, t.x, &t.well, &t.cell, &t.lb);
            const int dWell = t.well != well_prev;
            const int dCell = t.cell != cell_prev;
            const int dKey = k->dbl ? (t.lb != lb_prev) : dCell;

            if (k->eta) {
                /* UpdateBarrierStateEta, S.h:1998-2153 / D.h:2435-2736, with
                 * every barrier's flips on a schedule: the current barrier
                 * flips at its pending flip step; a barrier left keeps its
                 * pending flip in the cell table; one re-entered before that
                 * step has not flipped meanwhile (no draw), one whose flip
                 * came while it was away (or never visited: created at step
                 * 0) is caught up from that step with the two-state
                 * transition probability (S.h:2025-2068). */
                const int flip = (int64_t)s == nflip;
                uint32_t wf[4];
                int have_wf = 0;
                if (flip) {
                    t.state ^= 1;
                    philox_at(s, g, TAG_FLIP, key, wf);
                    have_wf = 1;
                    nflip = ldpo_schedule(s, wf[0], wf[1], k->ln1m[t.state]);
                }
                if (dKey) {
                    ring_store(&r, cell_key(k, cell_prev, lb_prev), t.state, nflip, &evict);
                    int ps, found;
                    int64_t nb;
                    ring_load(k, c, p, key, g, &r, cell_key(k, t.cell, t.lb), &ps, &nb, &found);
                    if (found && nb > (int64_t)s) {
                        t.state = ps;
                        nflip = nb;
                    } else {
                        const int64_t base = found ? nb : 0;
                        const int sb = found ? (ps ^ 1) : ps;
                        double lap = (double)((int64_t)s - base);
                        double pl = k->c_lap[k->eq ? 0 : sb] * -ldpo_expm1(k->a_lap * lap);
                        uint64_t Tl = ldpo_prob_to_u64(pl);
                        uint32_t wc[4];
                        philox_at(s, g, TAG_CATCHUP, key, wc);
                        uint64_t U = ((uint64_t)wc[0] << 32) | wc[1];
                        t.state = (U < Tl) ? (sb ^ 1) : sb;
                        if (!have_wf) philox_at(s, g, TAG_FLIP, key, wf);
                        nflip = ldpo_schedule(s, wf[2], wf[3], k->ln1m[t.state]);
                    }
                }
            } else {
                /* UpdateBarrierState (TAU == 0), S.h:1933-1997 / D.h:2299-2434 */
                if (dKey) {
                    ring_store(&r, cell_key(k, cell_prev, lb_prev), t.state, nflip, &evict);
                    int ps, found;
                    int64_t nb;
                    ring_load(k, c, p, key, g, &r, cell_key(k, t.cell, t.lb), &ps, &nb, &found);
                    t.state = ps;
                }
            }
            cnt[t.state ? LDP_C_STATE1 : LDP_C_STATE0]++;
            energy_force(k, &t);
            if (!k->over) t.v = t.v + (k->invM * t.F) * k->hdt;

            /* ---- UpdateStatistics, S.h:2334-2592 / D.h:2931-3209 ---- */
            const double now = k->dt * (double)s;
            if (k->wt && !fp_mode) {
                if (dWell) { t.wt_tick = (int64_t)s; t.wt_passed = 1; }
                else if (dCell && t.wt_passed) {
                    if (wt_n < c->tick_cap && out->ticks) out->ticks[i * c->tick_cap + wt_n] = t.wt_tick;
                    else if (wt_n >= c->tick_cap) flags |= LDP_FLAG_TICK_OVERFLOW;
                    ++wt_n;
                    t.wt_passed = 0;
                }
            }
            if (k->fpt || fp_mode) {
                if (!k->dbl && !fp_mode) {
                    if (t.fpt_up && dCell) {
                        t.fpt_up = 0;
                        t.fpt_last = now;
                        fpt_set_initial(k, c, p, key, g, &r, &t);
                    }
                    if (!t.fpt_up && dWell) {
                        t.fpt_up = 1;
                        if (cnt[LDP_C_FPT] == 0) sum[LDP_S_FIRST_FPT] = now - t.fpt_last;
                        sum[LDP_S_FPT] += now - t.fpt_last;
                        double ib = ((double)t.cell == (double)t.init_idx[0]) ? t.init_state[0] : t.init_state[1];
                        ev_push(c, out, n, i, LDP_E_FPT, cnt[LDP_C_FPT], now - t.fpt_last, &flags);
                        if (cnt[LDP_C_FPT] < c->event_cap && out->event_states)
                            out->event_states[i * c->event_cap + cnt[LDP_C_FPT]] =
                                (uint8_t)((t.state ? 1 : 0) | (ib != 0.0 ? 2 : 0));
                        cnt[LDP_C_FPT]++;
                        cnt[ib == 0.0 ? LDP_C_INIT0 : LDP_C_INIT1]++;
                        cnt[t.state == 0 ? LDP_C_INST0 : LDP_C_INST1]++;
                    }
                }
                if (t.fpt2_up && dCell) {
                    t.fpt2_up = 0;
                    t.fpt2_last = now;
                    fpt2_set_idx(&t);
                }
                if (dCell && !t.fpt2_up && t.idx2[0] != t.cell && t.idx2[1] != t.cell) {
                    if (cnt[LDP_C_FPT2] == 0) sum[LDP_S_FIRST_FPT2] = now - t.fpt2_last;
                    sum[LDP_S_FPT2] += now - t.fpt2_last;
                    ev_push(c, out, n, i, LDP_E_FPT2, cnt[LDP_C_FPT2], now - t.fpt2_last, &flags);
                    cnt[LDP_C_FPT2]++;
                    t.fpt2_last = now;
                    fpt2_set_idx(&t);
                    if (fp_mode) stop = 1;
                }
            }
            if (k->tpt && !fp_mode) {
                if (dCell) { t.tpt_up = 0; t.tpt_last = now; }
                if (!t.tpt_up && dWell) {
                    t.tpt_up = 1;
                    if (cnt[LDP_C_TPT] == 0) sum[LDP_S_FIRST_TPT] = now - t.tpt_last;
                    sum[LDP_S_TPT] += now - t.tpt_last;
                    ev_push(c, out, n, i, LDP_E_TPT, cnt[LDP_C_TPT], now - t.tpt_last, &flags);
                    cnt[LDP_C_TPT]++;
                }
                if (dCell) {
                    if (t.tpt2_up) t.tpt2_up = 0;
                    else if (t.well != t.tpt2_well) {
                        if (cnt[LDP_C_TPT2] == 0) sum[LDP_S_FIRST_TPT2] = now - t.tpt2_last;
                        sum[LDP_S_TPT2] += now - t.tpt2_last;
                        ev_push(c, out, n, i, LDP_E_TPT2, cnt[LDP_C_TPT2], now - t.tpt2_last, &flags);
                        cnt[LDP_C_TPT2]++;
                    }
                    t.tpt2_last = now;
                    t.tpt2_well = t.well;
                }
            }
            if (k->cg && !fp_mode) {
                for (int jj = 0; jj < k->n_cg; ++jj) {
                    if (dCell && cg_hit(t.well, k->cg_size[jj])) {
                        if (t.cg_up[jj]) {
                            t.cg_up[jj] = 0;
                            t.cg_last[jj] = now;
                            t.cg_well[jj] = t.well;
                        } else if (t.well != t.cg_well[jj]) {
                            sum[LDP_S_CG0 + jj] += now - t.cg_last[jj];
                            ev_push(c, out, n, i, LDP_E_CG0 + jj, cnt[LDP_C_CG0 + jj], now - t.cg_last[jj], &flags);
                            cnt[LDP_C_CG0 + jj]++;
                            t.cg_last[jj] = now;
                            t.cg_well[jj] = t.well;
                        }
                    }
                }
            }
            /* Record every FREQSAVE steps, S.h:1424-1447 / 1475 */
            if (!fp_mode && (s % k->freq_save) == 0) record(k, &t, out, n, i, (int64_t)(s / k->freq_save));
            done_steps = s;
        }
        if (fp_mode && !stop && !(flags & LDP_FLAG_NONFINITE)) flags |= LDP_FLAG_CENSORED;
        cnt[LDP_C_WT] = wt_n;
        cnt[LDP_C_EVICT] = evict;
        cnt[LDP_C_FLAGS] = flags;
        cnt[LDP_C_STEPS] = (int64_t)done_steps;
        if (out->counts)
            for (int f = 0; f < LDP_NCOUNT; ++f) CNT(f) = cnt[f];
        if (out->sums)
            for (int f = 0; f < LDP_NSUM; ++f) SUM(f) = sum[f];
        if (out->state0) out->state0[i] = state0;
        if (out->v0) out->v0[i] = v0inst;
        if (out->x_final) out->x_final[i] = t.x;
        if (out->v_final) out->v_final[i] = t.v;
        if (out->state_final) out->state_final[i] = t.state;
    }
    free(r.tag);
    free(r.data);
    return 0;
}

/* Per-trajectory mean-square displacement at each lag
 * (MeanSquareDisplacementBruteForce, src/langevinDynamicsSingleBarrier.h:24-45):
 * msd0 = sum over origins k < nframe - lag of (x[k + lag] - x[k])^2, divided
 * by the origin count.  The sum is taken in a fixed order that a warp of 32
 * lanes evaluates without shared-memory bank conflicts: 32 partial sums
 * p[l] over the origins k = l, l + 32, l + 64, ... (each in increasing k),
 * then the tree p[l] += p[l + h] for l < h, h = 16, 8, 4, 2, 1, whose result
 * is p[0].  It differs from the reference's single running sum only in
 * rounding. */
void ldpo_msd_traj(const double *frames, int64_t nframe, int64_t ntraj, const int64_t *lags, int64_t nlag,
                   double *msd0) {
    for (int64_t g = 0; g < ntraj; ++g) {
        for (int64_t ii = 0; ii < nlag; ++ii) {
            const int64_t lag = lags[ii];
            const int64_t cnt = nframe - lag;
            double acc = 0.0;
            if (cnt > 0) {
                double p[32];
                for (int l = 0; l < 32; ++l) {
                    double a = 0.0;
                    for (int64_t kk = l; kk < cnt; kk += 32) {
                        const double d = frames[(kk + lag) * ntraj + g] - frames[kk * ntraj + g];
                        a = a + d * d;
                    }
                    p[l] = a;
                }
                for (int h = 16; h >= 1; h >>= 1)
                    for (int l = 0; l < h; ++l) p[l] = p[l] + p[l + h];
                acc = p[0] / (double)cnt;
            }
            msd0[ii * ntraj + g] = acc;
        }
    }
}
