// ldp_device.cuh -- device random streams and FP64 elementary functions.
//
// Random numbers: one Philox4x32-10 stream per trajectory (Salmon et al.,
// SC'11).  Counter = {a_lo, a_hi, trajectory, tag}, key = {seed, job}.  This
// replaces the MKL VSL MT19937 banks of the reference
// (src/RANDOMNUMBER.cpp:70-340; streams created at
// src/langevinDynamicsSingleBarrier.h:1288-1290); the draw points stay where
// the reference has them:
//   TAG_STEP    a = (step-1)>>2: words 0,1 -> Box-Muller pair of steps 4a+1
//               (cosine branch) and 4a+2 (sine branch); words 2,3 -> pair of
//               steps 4a+3 and 4a+4.
//   TAG_INIT    a = 0: word 0 -> initial barrier state, words 1,2 ->
//               Box-Muller pair (v0, R0).
//   TAG_CATCHUP a = step: words 0,1 -> 64-bit uniform of the lazy catch-up
//               flip on entering a cell (S.h:2025-2068).
//   TAG_CELL    a = cell key: word 0 -> state of a never-visited cell
//               (BarrierStatus::Initialize, S.h:78-96).
//   TAG_FLIP    a = step: words 0,1 -> 64-bit uniform of the waiting time to
//               the current barrier's next flip, drawn at step 0, after every
//               flip, and on a barrier change that changes the flip
//               probability.
//
// The reference flips the current barrier with probability p each step
// (S.h:2010-2015); those flips form a Bernoulli process, so the steps
// between them are geometric, and drawing the waiting time once per flip
// gives the same process while each step needs only its Gaussian.  The
// process is memoryless: across a change of barrier with the same flip
// probability the pending waiting time stays valid, with a different one a
// new one is drawn.
//
// The FP64 functions below evaluate a fixed operation sequence with explicit
// fma() so that the FP64 device path is bit-identical to a host evaluation
// of the same sequence.
#pragma once
#include <cstdint>

namespace ldp {

enum : uint32_t { TAG_STEP = 0, TAG_INIT = 1, TAG_CATCHUP = 2, TAG_CELL = 3, TAG_FLIP = 4 };

struct Words { uint32_t w0, w1, w2, w3; };

__device__ __forceinline__ Words philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                        uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return Words{c0, c1, c2, c3};
}

// The same function written with 32 x 32 -> 64-bit products (one wide
// multiply per product gives both halves); identical output.
__device__ __forceinline__ Words philox_wide(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                             uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)c0 * 0xD2511F53u;
        const uint64_t p1 = (uint64_t)c2 * 0xCD9E8D57u;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
    }
    return Words{c0, c1, c2, c3};
}

__device__ __forceinline__ Words philox_at(uint64_t a, uint32_t g, uint32_t tag, uint32_t k0, uint32_t k1) {
    return philox((uint32_t)a, (uint32_t)(a >> 32), g, tag, k0, k1);
}

// ----- FP64 elementary functions (deterministic operation sequences) -----
constexpr double kLn2Hi = 6.93147180559945286227e-01;    // nearest double to ln 2
constexpr double kLn2Lo = 2.31904681384629955842e-17;    // ln 2 - kLn2Hi
constexpr double kTwoPiHi = 6.28318530717958623200e+00;  // nearest double to 2 pi
constexpr double kTwoPiLo = 2.44929359829470635445e-16;  // 2 pi - kTwoPiHi

// log(u) for positive normal u: u = m 2^e with m in [sqrt(1/2), sqrt(2)),
// log m = 2 atanh((m-1)/(m+1)) by the odd power series of atanh.
__device__ __forceinline__ double log_f64(double u) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(u);
    long long e = (long long)((b >> 52) & 0x7ff) - 1023;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull));
    if (m > 1.41421356237309504880) { m = m * 0.5; e += 1; }
    const double f = (m - 1.0) / (m + 1.0);
    const double f2 = f * f;
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
    const double logm = fma(2.0 * f * f2, s, 2.0 * f);
    const double de = (double)e;
    return fma(de, kLn2Hi, fma(de, kLn2Lo, logm));
}

// sin(2 pi t), cos(2 pi t), t in [0, 1): quadrant from rint(4t), Taylor
// series of sin and cos on [-pi/4, pi/4].
__device__ __forceinline__ void sincos2pi_f64(double t, double* sn, double* cs) {
    const double q = rint(t * 4.0);
    const double f = t - q * 0.25;
    const double x = fma(f, kTwoPiHi, f * kTwoPiLo);
    const double x2 = x * x;
    double ps = -1.0 / 121645100408832000.0;
    ps = fma(ps, x2, 1.0 / 355687428096000.0);
    ps = fma(ps, x2, -1.0 / 1307674368000.0);
    ps = fma(ps, x2, 1.0 / 6227020800.0);
    ps = fma(ps, x2, -1.0 / 39916800.0);
    ps = fma(ps, x2, 1.0 / 362880.0);
    ps = fma(ps, x2, -1.0 / 5040.0);
    ps = fma(ps, x2, 1.0 / 120.0);
    ps = fma(ps, x2, -1.0 / 6.0);
    const double s = fma(x * x2, ps, x);
    double pc = 1.0 / 2432902008176640000.0;
    pc = fma(pc, x2, -1.0 / 6402373705728000.0);
    pc = fma(pc, x2, 1.0 / 20922789888000.0);
    pc = fma(pc, x2, -1.0 / 87178291200.0);
    pc = fma(pc, x2, 1.0 / 479001600.0);
    pc = fma(pc, x2, -1.0 / 3628800.0);
    pc = fma(pc, x2, 1.0 / 40320.0);
    pc = fma(pc, x2, -1.0 / 720.0);
    pc = fma(pc, x2, 1.0 / 24.0);
    pc = fma(pc, x2, -0.5);
    const double c = fma(x2, pc, 1.0);
    const int qi = ((int)q) & 3;
    double so, co;
    if (qi == 0) { so = s; co = c; }
    else if (qi == 1) { so = c; co = -s; }
    else if (qi == 2) { so = -s; co = -c; }
    else { so = -c; co = s; }
    *sn = so;
    *cs = co;
}

// expm1(x), x <= 0: Cody-Waite reduction x = k ln2 + r, Taylor series for
// expm1(r), then 2^k (expm1(r) + 1) - 1.
__device__ __forceinline__ double expm1_f64(double x) {
    if (x < -60.0) return -1.0;
    const double k = rint(x * 1.44269504088896340736);
    double r = fma(-k, kLn2Hi, x);
    r = fma(-k, kLn2Lo, r);
    double p = 1.0 / 6227020800.0;
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
    const double e = fma(r * r, p, r);
    if (k == 0.0) return e;
    const double s = ldexp(1.0, (int)k);
    return fma(s, e, s - 1.0);
}

// Steps from the current one to the next flip of a barrier that flips with
// probability p per step, ln1m = log(1 - p): W = 1 + floor(ln U / ln(1-p))
// for U in (0, 1] from the 64-bit word pair (geometric, P(W = k) =
// (1-p)^(k-1) p); UINT64_MAX when the barrier never flips.
__device__ __forceinline__ uint64_t flip_wait(uint32_t hi, uint32_t lo, double ln1m) {
    if (!(ln1m < 0.0)) return 0xffffffffffffffffull;
    const double u = ((double)(((uint64_t)hi << 32) | lo) + 1.0) * 0x1p-64;
    const double q = log_f64(u) / ln1m;
    if (!(q < 0x1p62)) return 0xffffffffffffffffull;
    return 1ull + (uint64_t)floor(q);
}

// "Never" for a flip step; fits the cell table's (step << 1 | state).
constexpr int64_t kNeverFlip = (int64_t)((1ull << 62) - 1);

// Step of the next flip drawn at step s: s + W, clamped to kNeverFlip.
__device__ __forceinline__ int64_t flip_schedule(uint64_t s, uint32_t hi, uint32_t lo, double ln1m) {
    const uint64_t wt = flip_wait(hi, lo, ln1m);
    return (wt >= (uint64_t)kNeverFlip - s) ? kNeverFlip : (int64_t)(s + wt);
}

__device__ __forceinline__ uint64_t prob_to_u64(double p) {
    if (!(p > 0.0)) return 0ull;
    if (p >= 1.0) return 0xffffffffffffffffull;
    return (uint64_t)ldexp(p, 64);
}

// Box-Muller pair from two 32-bit words, FP64.
__device__ __forceinline__ void gauss_pair_f64(uint32_t wa, uint32_t wb, double* z0, double* z1) {
    const double u1 = ((double)wa + 1.0) * 0x1p-32;
    const double u2 = (double)wb * 0x1p-32;
    const double r = sqrt(-2.0 * log_f64(u1));
    double sn, cs;
    sincos2pi_f64(u2, &sn, &cs);
    *z0 = r * cs;
    *z1 = r * sn;
}

// Box-Muller pair from the same two words on the FP32 special-function units.
__device__ __forceinline__ void gauss_pair_f32(uint32_t wa, uint32_t wb, float* z0, float* z1) {
    const float u1 = __fmul_rn((float)(wa >> 8) + 1.0f, 0x1p-24f);
    float u2 = __fmul_rn((float)(wb >> 8), 0x1p-24f);
    u2 = (u2 >= 0.5f) ? u2 - 1.0f : u2;   // same angle, kept in [-pi, pi)
    const float r = sqrtf(-2.0f * __logf(u1));
    float sn, cs;
    __sincosf(6.28318530717958647692f * u2, &sn, &cs);
    *z0 = r * cs;
    *z1 = r * sn;
}

}  // namespace ldp
