// vsl_standin.cpp -- the VSL calls of mkl.h, for the CPU-baseline build of
// the reference's own code (test infrastructure; never part of the
// product).  Published algorithms, restated:
//   * MT19937 (Matsumoto and Nishimura, ACM TOMACS 8(1), 1998): 624-word
//     state, seeding by the recurrence x_i = 1812433253 (x_{i-1} ^
//     (x_{i-1} >> 30)) + i, tempered 32-bit outputs;
//   * uniform doubles on [0, 1) with 53 random bits from two outputs (the
//     authors' genrand_res53 construction), mapped to [a, b);
//   * Gaussian doubles by inversion (the reference asks for
//     VSL_RNG_METHOD_GAUSSIAN_ICDF): the uniform, shifted off 0 by half a
//     unit of the last bit, through P. J. Acklam's rational approximation
//     of the normal quantile (relative error below 1.2e-9, no refinement
//     step), then mean + sigma x.
// One number of either kind takes two 32-bit outputs; vslSkipAheadStream
// skips that many numbers.
#include <cmath>
#include <cstdint>
#include <cstdlib>

#include "mkl.h"

namespace {

struct Mt19937 {
    uint32_t s[624];
    int i;
    void seed(uint32_t v) {
        s[0] = v;
        for (int k = 1; k < 624; ++k) s[k] = 1812433253u * (s[k - 1] ^ (s[k - 1] >> 30)) + (uint32_t)k;
        i = 624;
    }
    void twist() {
        for (int k = 0; k < 624; ++k) {
            const uint32_t y = (s[k] & 0x80000000u) | (s[(k + 1) % 624] & 0x7fffffffu);
            s[k] = s[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        i = 0;
    }
    uint32_t next() {
        if (i >= 624) twist();
        uint32_t y = s[i++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }
    // 53-bit integer from two outputs (27 + 26 high bits).
    uint64_t bits53() {
        const uint64_t a = next() >> 5, b = next() >> 6;
        return a * 67108864ull + b;
    }
};

// Acklam's normal quantile, p in (0, 1).
double quantile(double p) {
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    const double plow = 0.02425;
    if (p < plow || p > 1.0 - plow) {
        const double q = std::sqrt(-2.0 * std::log(p < plow ? p : 1.0 - p));
        const double x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
                         ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
        return p < plow ? x : -x;
    }
    const double q = p - 0.5, r = q * q;
    return (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
           (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
}

}  // namespace

extern "C" {

int vslNewStream(VSLStreamStatePtr* stream, MKL_INT, MKL_UINT seed) {
    Mt19937* m = new Mt19937;
    m->seed((uint32_t)seed);
    *stream = m;
    return VSL_STATUS_OK;
}

int vslDeleteStream(VSLStreamStatePtr* stream) {
    delete static_cast<Mt19937*>(*stream);
    *stream = nullptr;
    return VSL_STATUS_OK;
}

int vslSkipAheadStream(VSLStreamStatePtr stream, long long nskip) {
    Mt19937* m = static_cast<Mt19937*>(stream);
    for (long long k = 0; k < 2 * nskip; ++k) m->next();
    return VSL_STATUS_OK;
}

int vdRngUniform(MKL_INT, VSLStreamStatePtr stream, MKL_INT n, double* r, double a, double b) {
    Mt19937* m = static_cast<Mt19937*>(stream);
    const double w = b - a;
    for (MKL_INT k = 0; k < n; ++k) {
        double v = a + w * ((double)m->bits53() * 0x1p-53);
        r[k] = (v < b) ? v : std::nextafter(b, a);   // [a, b)
    }
    return VSL_STATUS_OK;
}

int vdRngGaussian(MKL_INT, VSLStreamStatePtr stream, MKL_INT n, double* r, double mean, double sigma) {
    Mt19937* m = static_cast<Mt19937*>(stream);
    for (MKL_INT k = 0; k < n; ++k) r[k] = mean + sigma * quantile(((double)m->bits53() + 0.5) * 0x1p-53);
    return VSL_STATUS_OK;
}

}  // extern "C"
