/*
 * simd_unaligned.h -- force-included (-include) before every reference
 * source file of the CPU-baseline build.  The reference aliases the aligned
 * AVX load/store intrinsics (src/simd.h:105-108, 140-143) and applies them
 * to std::vector-backed random-number banks, which GCC does not align to
 * 64 bytes, so an aligned vmovapd faults.  After <immintrin.h> is in, the
 * aligned names are mapped to the unaligned forms (same values; alignment
 * is the only difference).
 */
#ifndef LDP_REFSHIM_SIMD_UNALIGNED_H
#define LDP_REFSHIM_SIMD_UNALIGNED_H
#include <immintrin.h>
#define _mm256_load_pd _mm256_loadu_pd
#define _mm256_store_pd _mm256_storeu_pd
#define _mm512_load_pd _mm512_loadu_pd
#define _mm512_store_pd _mm512_storeu_pd
#endif
