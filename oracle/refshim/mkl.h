/*
 * mkl.h -- stand-in for the part of Intel MKL's VSL the reference calls
 * (src/RANDOMNUMBER.cpp:84, 91, 109-121, 175, 182, 268, 274): MT19937
 * streams, skip-ahead, uniform and Gaussian doubles.  Test infrastructure
 * for building the reference's own code as a CPU baseline and statistical
 * checker; MKL itself is closed and absent here, so the numbers differ from
 * MKL's (the generators are the published algorithms named in
 * vsl_standin.cpp).
 */
#ifndef LDP_REFSHIM_MKL_H
#define LDP_REFSHIM_MKL_H

typedef void* VSLStreamStatePtr;
typedef int MKL_INT;
typedef unsigned int MKL_UINT;

#define VSL_BRNG_MT19937 0x00200000
#define VSL_RNG_METHOD_UNIFORM_STD_ACCURATE 0x40000000
#define VSL_RNG_METHOD_GAUSSIAN_ICDF 3
#define VSL_STATUS_OK 0

#ifdef __cplusplus
extern "C" {
#endif
int vslNewStream(VSLStreamStatePtr* stream, MKL_INT brng, MKL_UINT seed);
int vslDeleteStream(VSLStreamStatePtr* stream);
int vslSkipAheadStream(VSLStreamStatePtr stream, long long nskip);
int vdRngUniform(MKL_INT method, VSLStreamStatePtr stream, MKL_INT n, double* r, double a, double b);
int vdRngGaussian(MKL_INT method, VSLStreamStatePtr stream, MKL_INT n, double* r, double mean, double sigma);
#ifdef __cplusplus
}
#endif

#endif
