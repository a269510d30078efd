// ldp_msd.cu -- mean-square displacement over saved frames.
//
// Device restatement of MeanSquareDisplacementBruteForce
// (src/langevinDynamicsSingleBarrier.h:24-45) for every trajectory, and of
// the run-level sum msd[t] += msd0[t] / nrun (S.h:3452-3461, 3893-3902).
//
// msd_smem_kernel: a block owns G trajectories.  It stages their whole frame
// series in shared memory (one pass over HBM, rows of G doubles).  A warp
// then takes (trajectory, group of kMsdLags lags) work items; its 32 lanes
// take the origins k = lane, lane + 32, ... of every lag of the group, so
// both x[k] (loaded once for the group) and x[k + lag] are 32 consecutive
// words (no bank conflicts).  Each lane keeps one partial sum per lag in
// increasing k, and the 32 partials meet in a fixed shuffle tree
// (h = 16, 8, 4, 2, 1): the summation order of the oracle's msd_traj, so
// msd0 is bit-identical to it (compiled with -fmad=false).  HBM traffic is
// the frames once; the O(frames x lags) work runs from shared memory at
// 1 + 1/kMsdLags conflict-free shared loads and 3 FP64 operations per term.
// msd_traj_kernel is the same computation from global memory, used only when
// one trajectory's frames do not fit in shared memory.
//
// msd_smem_f32_kernel: the same for jobs of the FP32 batched path: a
// trajectory's frames are staged in shared memory as offsets from its first
// frame, rounded to FP32 (an error of at most 2^-24 of the offset), the
// displacement x[k + lag] - x[k] is taken in FP32, its square is summed in
// FP32 over groups of 8 origins per lane, and the groups' sums are
// accumulated in FP64 (32-way interleaved partials of ~nframe/32 terms
// each), so the moment sums are FP64 as on the FP64 path.  Half the shared-memory bytes per term, which
// bound the FP64 kernel; with 6 lags per item, a loop without per-term
// tests over the origins all of them have, and four blocks per SM (54 KiB
// each) to hide the shared-load latency.  The FP64 plain path keeps the
// FP64 kernel (bit-identical to the oracle).
//
// msd_reduce_kernel: one block per lag sums msd0 over trajectories with
// Kahan compensation in a fixed order (per-thread strided partials, then a
// fixed shared-memory tree), so the result does not depend on scheduling.
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/ldp.h"
#include "ldp_msd.h"

namespace ldp {

constexpr int kMsdSmemBytes = 100 * 1024;   // two blocks per SM
constexpr int kMsdBlock = 256;
constexpr int kMsdLags = 4;                  // lags per work item (x[k] reuse)
constexpr int kMsdF32SmemBytes = 54 * 1024;  // FP32 kernel: four blocks per SM
constexpr int kMsdF32Group = 8;              // FP32 kernel: origins per FP32 partial sum
// Lean FP32 instance (msd_smem_f32_kernel<128, 2, 16, true>), for
// post-processing that runs beside the persistent FP32 kernel: one warp per
// SMSP at 32 registers is what three persistent blocks leave of an SM's
// register file, and one staged trajectory (12 KB at 3001 frames) fits in
// its spare shared memory.  Every lag is summed in the same order, so its
// results equal the full instance's bit for bit.

__global__ void __launch_bounds__(kMsdBlock) msd_smem_kernel(const double* __restrict__ frames, int nframe,
                                                             int64_t ntraj, int G, const int64_t* __restrict__ lags,
                                                             int nlag, double* __restrict__ msd0) {
    extern __shared__ double fs[];   // [G][nframe]
    const int64_t t0 = (int64_t)blockIdx.x * G;
    const int gh = (int)((ntraj - t0) < G ? (ntraj - t0) : G);
    // Stage: element (k, j) -> fs[j * nframe + k]; consecutive threads read
    // consecutive trajectories of one frame row.
    const int total = nframe * G;
    for (int e = threadIdx.x; e < total; e += kMsdBlock) {
        const int k = e / G;
        const int j = e - k * G;
        fs[j * nframe + k] = (j < gh) ? frames[(int64_t)k * ntraj + t0 + j] : 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ngroup = (nlag + kMsdLags - 1) / kMsdLags;
    const int items = gh * ngroup;
    for (int it = warp; it < items; it += kMsdBlock / 32) {
        const int j = it / ngroup;
        const int g0 = (it - j * ngroup) * kMsdLags;
        const double* x = fs + j * nframe;
        int lag[kMsdLags], cnt[kMsdLags];
        double acc[kMsdLags];
        int kmax = 0;
#pragma unroll
        for (int r = 0; r < kMsdLags; ++r) {
            const int i = g0 + r;
            lag[r] = (i < nlag) ? (int)lags[i] : 0;
            cnt[r] = (i < nlag) ? nframe - lag[r] : 0;
            if (cnt[r] < 0) cnt[r] = 0;
            kmax = cnt[r] > kmax ? cnt[r] : kmax;
            acc[r] = 0.0;
        }
        for (int k = lane; k < kmax; k += 32) {
            const double xk = x[k];
#pragma unroll
            for (int r = 0; r < kMsdLags; ++r) {
                if (k < cnt[r]) {
                    const double d = x[k + lag[r]] - xk;
                    acc[r] = acc[r] + d * d;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kMsdLags; ++r) {
            double v = acc[r];
#pragma unroll
            for (int h = 16; h >= 1; h >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, h);
            const int i = g0 + r;
            if (lane == 0 && i < nlag) msd0[(int64_t)i * ntraj + t0 + j] = cnt[r] > 0 ? v / (double)cnt[r] : 0.0;
        }
    }
}

template <int kBlk, int kNL, int kMinB, bool kOne>
__global__ void __launch_bounds__(kBlk, kMinB) msd_smem_f32_kernel(const double* __restrict__ frames, int nframe,
                                                                    int64_t ntraj, int G_,
                                                                    const int64_t* __restrict__ lags, int nlag,
                                                                    double* __restrict__ msd0) {
    extern __shared__ float fs32[];   // [G][nframe]
    const int G = kOne ? 1 : G_;      // kOne: one trajectory per block
    const int64_t t0 = (int64_t)blockIdx.x * G;
    const int gh = (int)((ntraj - t0) < G ? (ntraj - t0) : G);
    const int total = nframe * G;
    for (int e = threadIdx.x; e < total; e += kBlk) {
        const int k = e / G;
        const int j = e - k * G;
        fs32[j * nframe + k] = (j < gh) ? (float)(frames[(int64_t)k * ntraj + t0 + j] - frames[t0 + j]) : 0.0f;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ngroup = (nlag + kNL - 1) / kNL;
    const int items = gh * ngroup;
    for (int it = warp; it < items; it += kBlk / 32) {
        const int j = it / ngroup;
        const int g0 = (it - j * ngroup) * kNL;
        const float* x = fs32 + j * nframe;
        int lag[kNL], cnt[kNL];
        double acc[kNL];
        // Slots past the last lag repeat the group's first lag (results not
        // written), so that kmin is the shortest origin count of real lags.
        const int lag0 = (int)lags[g0];
        int kmin = 1 << 30, kmax = 0;
#pragma unroll
        for (int r = 0; r < kNL; ++r) {
            const int i = g0 + r;
            lag[r] = (i < nlag) ? (int)lags[i] : lag0;
            cnt[r] = nframe - lag[r];
            if (cnt[r] < 0) cnt[r] = 0;
            kmin = cnt[r] < kmin ? cnt[r] : kmin;
            kmax = cnt[r] > kmax ? cnt[r] : kmax;
            acc[r] = 0.0;
        }
        // A lag's origins k = lane + 32 i are taken in groups of kMsdF32Group
        // (consecutive i): the squares of a group that lies wholly below the
        // lag's origin count are summed in FP32 (at most kMsdF32Group terms,
        // relative error below kMsdF32Group * 2^-24) and the group's sum is
        // added to the lag's FP64 sum, one widening and one FP64 add per
        // group instead of per term; the origins after its last whole group
        // are added one by one in FP64.  That order depends only on the lane
        // and the lag, not on which lags share the item, so every instance
        // gives the same sums.
        constexpr int kG = kMsdF32Group;
        int k = lane;
        // groups whole for every lag of the item: no per-term test
        for (; k + 32 * (kG - 1) < kmin; k += 32 * kG) {
            float part[kNL];
#pragma unroll
            for (int r = 0; r < kNL; ++r) part[r] = 0.0f;
#pragma unroll
            for (int g = 0; g < kG; ++g) {
                const float xk = x[k + 32 * g];
#pragma unroll
                for (int r = 0; r < kNL; ++r) {
                    const float d = x[k + 32 * g + lag[r]] - xk;
                    part[r] = fmaf(d, d, part[r]);
                }
            }
#pragma unroll
            for (int r = 0; r < kNL; ++r) acc[r] += (double)part[r];
        }
        // groups whole for some lags of the item
        for (; k + 32 * (kG - 1) < kmax; k += 32 * kG) {
#pragma unroll
            for (int r = 0; r < kNL; ++r) {
                if (k + 32 * (kG - 1) < cnt[r]) {
                    float part = 0.0f;
#pragma unroll
                    for (int g = 0; g < kG; ++g) {
                        const float d = x[k + 32 * g + lag[r]] - x[k + 32 * g];
                        part = fmaf(d, d, part);
                    }
                    acc[r] += (double)part;
                } else {
                    for (int g = 0; g < kG && k + 32 * g < cnt[r]; ++g) {
                        const double d = (double)(x[k + 32 * g + lag[r]] - x[k + 32 * g]);
                        acc[r] = fma(d, d, acc[r]);
                    }
                }
            }
        }
        // the origins after the last group, one by one
        for (; k < kmax; k += 32) {
            const float xk = x[k];
#pragma unroll
            for (int r = 0; r < kNL; ++r) {
                if (k < cnt[r]) {
                    const double d = (double)(x[k + lag[r]] - xk);
                    acc[r] = fma(d, d, acc[r]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kNL; ++r) {
            double v = acc[r];
#pragma unroll
            for (int h = 16; h >= 1; h >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, h);
            const int i = g0 + r;
            if (lane == 0 && i < nlag) msd0[(int64_t)i * ntraj + t0 + j] = cnt[r] > 0 ? v / (double)cnt[r] : 0.0;
        }
    }
}

// One warp per (trajectory, lag), frames read from global memory, same
// summation order as msd_smem_kernel.
__global__ void msd_traj_kernel(const double* __restrict__ frames, int64_t nframe, int64_t ntraj,
                                const int64_t* __restrict__ lags, int64_t nlag, double* __restrict__ msd0) {
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t ii = blockIdx.y;
    if (t >= ntraj || ii >= nlag) return;
    const int64_t lag = lags[ii];
    const int64_t cnt = nframe - lag;
    double v = 0.0;
    for (int64_t k = lane; k < cnt; k += 32) {
        const double d = frames[(k + lag) * ntraj + t] - frames[k * ntraj + t];
        v = v + d * d;
    }
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, h);
    if (lane == 0) msd0[ii * ntraj + t] = cnt > 0 ? v / (double)cnt : 0.0;
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) msd_reduce_kernel(const double* __restrict__ msd0, int64_t ntraj,
                                                           double* __restrict__ out) {
    __shared__ double ss[BLOCK], sc[BLOCK];
    const int64_t ii = blockIdx.x;
    const double* row = msd0 + ii * ntraj;
    double s = 0.0, c = 0.0;
    for (int64_t t = threadIdx.x; t < ntraj; t += BLOCK) {
        const double y = row[t] - c;
        const double u = s + y;
        c = (u - s) - y;
        s = u;
    }
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int w = BLOCK / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            // Kahan-style merge of two compensated partial sums.
            const double a = ss[threadIdx.x], b = ss[threadIdx.x + w];
            const double u = a + b;
            const double bp = u - a;
            const double err = (a - (u - bp)) + (b - bp);
            ss[threadIdx.x] = u;
            sc[threadIdx.x] = sc[threadIdx.x] + sc[threadIdx.x + w] - err;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[ii] = ss[0] - sc[0];
}

// Per-trajectory mean event times, [list][traj]: the reference's
// STATISTICS::AVERAGE of each per-lane event list (GetFirstPassageTimeAverage
// {,2}, GetTransitionPathTimeAverage{,2}, GetFirstPassageTimeCGAverage2,
// S.h:2722-2763; src/STATISTICS.cpp:100-106): sum / count, 0 for no event.
// List L reads count field L and sum field L for L < 4 (FPT, FPT2, TPT,
// TPT2) and the FPTCG fields for the rest.
__global__ void traj_means_kernel(const int64_t* __restrict__ counts, const double* __restrict__ sums,
                                  double* __restrict__ means, int64_t n, int nlists) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)nlists * n) return;
    const int L = (int)(idx / n);
    const int64_t i = idx - (int64_t)L * n;
    const int cf = L < LDP_E_CG0 ? L : LDP_C_CG0 + (L - LDP_E_CG0);
    const int sf = L < LDP_E_CG0 ? L : LDP_S_CG0 + (L - LDP_E_CG0);
    const int64_t c = counts[(int64_t)cf * n + i];
    means[idx] = c ? sums[(int64_t)sf * n + i] / (double)c : 0.0;
}

int launch_traj_means(const int64_t* counts, const double* sums, double* means, int64_t n, int ncg, void* stream) {
    const int nlists = LDP_E_CG0 + ncg;
    const int64_t total = (int64_t)nlists * n;
    if (total == 0) return 0;
    const int block = 128;   // one warp per SMSP: fits beside persistent FP32 blocks
    traj_means_kernel<<<(unsigned)((total + block - 1) / block), block, 0, (cudaStream_t)stream>>>(counts, sums, means,
                                                                                               n, nlists);
    return (int)cudaGetLastError();
}

int launch_msd(const double* frames, int64_t nframe, int64_t ntraj, const int64_t* lags, int64_t nlag,
               double* msd0, double* msd_sum, void* stream, int mode) {
    cudaStream_t s = (cudaStream_t)stream;
    const bool f32 = mode != LDP_MSD_FP64;
    const bool lean = mode == LDP_MSD_FP32_LEAN;
    const int64_t per_traj = nframe * (int64_t)(f32 ? sizeof(float) : sizeof(double));
    int G;
    if (lean) {
        // one trajectory per block (kOne), or the global-memory kernel
        G = per_traj <= kMsdSmemBytes ? 1 : 0;
    } else {
        G = (int)((f32 ? kMsdF32SmemBytes : kMsdSmemBytes) / (per_traj > 0 ? per_traj : 1));
        if (f32 && G < 1 && per_traj <= kMsdSmemBytes) G = 1;
        if (G > 32) G = 32;
    }
    cudaError_t e;
    if (G >= 1 && nframe < (1 << 30) && nlag < (1 << 30)) {
        const size_t smem = (size_t)G * (size_t)per_traj;
        const int64_t nblk = (ntraj + G - 1) / G;
        if (lean) {
            auto* kern = msd_smem_f32_kernel<128, 2, 16, true>;
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return (int)e;
            kern<<<(unsigned)nblk, 128, smem, s>>>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0);
        } else if (f32) {
            auto* kern = msd_smem_f32_kernel<kMsdBlock, 6, 4, false>;
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return (int)e;
            kern<<<(unsigned)nblk, kMsdBlock, smem, s>>>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0);
        } else {
            e = cudaFuncSetAttribute(msd_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return (int)e;
            msd_smem_kernel<<<(unsigned)nblk, kMsdBlock, smem, s>>>(frames, (int)nframe, ntraj, G, lags, (int)nlag,
                                                                   msd0);
        }
    } else {
        const int block = 256;
        dim3 grid((unsigned)((ntraj + 7) / 8), (unsigned)nlag);
        msd_traj_kernel<<<grid, block, 0, s>>>(frames, nframe, ntraj, lags, nlag, msd0);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    msd_reduce_kernel<256><<<(unsigned)nlag, 256, 0, s>>>(msd0, ntraj, msd_sum);
    return (int)cudaGetLastError();
}

}  // namespace ldp
