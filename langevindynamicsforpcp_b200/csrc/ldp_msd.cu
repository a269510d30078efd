// ldp_msd.cu -- mean-square displacement over saved frames.
//
// Device restatement of MeanSquareDisplacementBruteForce
// (src/langevinDynamicsSingleBarrier.h:24-45) for every trajectory, and of
// the run-level sum msd[t] += msd0[t] / nrun (S.h:3452-3461, 3893-3902).
//
// msd_smem_kernel: a block owns G trajectories.  It stages their whole frame
// series in shared memory (one coalesced pass over HBM, rows of G doubles),
// then each thread takes (lag, trajectory) pairs and sums over frame
// origins in the reference's order, so msd0 is bit-identical to a
// sequential host evaluation (compiled with -fmad=false).  HBM traffic is
// the frames once; the O(frames x lags) work runs from shared memory.
// msd_traj_kernel is the same computation from global memory, used only when
// one trajectory's frames do not fit in shared memory.
//
// msd_reduce_kernel: one block per lag sums msd0 over trajectories with
// Kahan compensation in a fixed order (per-thread strided partials, then a
// fixed shared-memory tree), so the result does not depend on scheduling.
#include <cuda_runtime.h>
#include <cstdint>

namespace ldp {

constexpr int kMsdSmemBytes = 96 * 1024;   // two blocks per SM

__global__ void __launch_bounds__(256) msd_smem_kernel(const double* __restrict__ frames, int64_t nframe,
                                                       int64_t ntraj, int G, const int64_t* __restrict__ lags,
                                                       int64_t nlag, double* __restrict__ msd0) {
    extern __shared__ double fs[];   // [G][nframe]
    const int64_t t0 = (int64_t)blockIdx.x * G;
    const int g_here = (int)((ntraj - t0) < G ? (ntraj - t0) : G);
    // Stage: element (k, j) -> fs[j * nframe + k]; consecutive threads read
    // consecutive trajectories of one frame row.
    const int64_t total = nframe * G;
    for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
        const int64_t k = e / G;
        const int j = (int)(e - k * G);
        fs[(int64_t)j * nframe + k] = (j < g_here) ? frames[k * ntraj + t0 + j] : 0.0;
    }
    __syncthreads();
    const int64_t work = nlag * g_here;
    for (int64_t wi = threadIdx.x; wi < work; wi += blockDim.x) {
        const int64_t ii = wi / g_here;
        const int j = (int)(wi - ii * g_here);
        const int64_t lag = lags[ii];
        const double* x = fs + (int64_t)j * nframe;
        double acc = 0.0;
        const int64_t cnt = nframe - lag;
        if (cnt > 0) {
            for (int64_t k = 0; k < cnt; ++k) {
                const double d = x[k + lag] - x[k];
                acc = acc + d * d;
            }
            acc = acc / (double)cnt;
        }
        msd0[ii * ntraj + t0 + j] = acc;
    }
}

__global__ void msd_traj_kernel(const double* __restrict__ frames, int64_t nframe, int64_t ntraj,
                                const int64_t* __restrict__ lags, int64_t nlag, double* __restrict__ msd0) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ii = blockIdx.y;
    if (t >= ntraj || ii >= nlag) return;
    const int64_t lag = lags[ii];
    double acc = 0.0;
    if (nframe - lag > 0) {
        const double* a = frames + t;
        const double* b = frames + lag * ntraj + t;
        const int64_t cnt = nframe - lag;
        for (int64_t k = 0; k < cnt; ++k) {
            const double d = b[k * ntraj] - a[k * ntraj];
            acc = acc + d * d;
        }
        acc = acc / (double)cnt;
    }
    msd0[ii * ntraj + t] = acc;
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

int launch_msd(const double* frames, int64_t nframe, int64_t ntraj, const int64_t* lags, int64_t nlag,
               double* msd0, double* msd_sum, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t per_traj = nframe * (int64_t)sizeof(double);
    int G = (int)(kMsdSmemBytes / (per_traj > 0 ? per_traj : 1));
    if (G > 32) G = 32;
    cudaError_t e;
    if (G >= 1) {
        const size_t smem = (size_t)G * (size_t)per_traj;
        e = cudaFuncSetAttribute(msd_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        const int64_t nblk = (ntraj + G - 1) / G;
        msd_smem_kernel<<<(unsigned)nblk, 256, smem, s>>>(frames, nframe, ntraj, G, lags, nlag, msd0);
    } else {
        const int block = 128;
        dim3 grid((unsigned)((ntraj + block - 1) / block), (unsigned)nlag);
        msd_traj_kernel<<<grid, block, 0, s>>>(frames, nframe, ntraj, lags, nlag, msd0);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    msd_reduce_kernel<256><<<(unsigned)nlag, 256, 0, s>>>(msd0, ntraj, msd_sum);
    return (int)cudaGetLastError();
}

}  // namespace ldp
