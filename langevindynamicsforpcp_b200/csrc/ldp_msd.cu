// ldp_msd.cu -- mean-square displacement over saved frames.
//
// Device restatement of MeanSquareDisplacementBruteForce
// (src/langevinDynamicsSingleBarrier.h:24-45) for every trajectory, and of
// the run-level sum msd[t] += msd0[t] / nrun (S.h:3452-3461, 3893-3902).
//
// msd_smem_kernel: a block owns G trajectories.  It stages their whole frame
// series in shared memory (one pass over HBM, rows of G doubles), then every
// thread takes one trajectory and R lags (lag slots q, q + Q, q + 2Q, ... of
// the ascending lag list, Q = threads per trajectory) and walks the frame
// origins once, with one accumulator per lag: each (trajectory, lag) sum
// still runs over origins in the reference's order, so msd0 is bit-identical
// to a sequential host evaluation (compiled with -fmad=false), while a thread
// keeps R independent chains in flight and loads x[k] once for all R lags.
// HBM traffic is the frames once; the O(frames x lags) work runs from shared
// memory at about 1 + 1/R shared loads and 3 FP64 operations per term.
// msd_traj_kernel is the same computation from global memory, used only when
// one trajectory's frames do not fit in shared memory.
//
// msd_reduce_kernel: one block per lag sums msd0 over trajectories with
// Kahan compensation in a fixed order (per-thread strided partials, then a
// fixed shared-memory tree), so the result does not depend on scheduling.
#include <cuda_runtime.h>
#include <cstdint>

namespace ldp {

constexpr int kMsdSmemBytes = 100 * 1024;   // two blocks per SM
constexpr int kMsdBlock = 256;

template <int R>
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
    const int Q = kMsdBlock / G;
    const int j = threadIdx.x % G;
    const int q = threadIdx.x / G;
    if (q >= Q || j >= gh) return;
    const double* x = fs + j * nframe;
    int lag[R], cnt[R];
    double acc[R];
    int kmax = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = q + r * Q;
        lag[r] = (i < nlag) ? (int)lags[i] : 0;
        cnt[r] = (i < nlag) ? nframe - lag[r] : 0;
        if (cnt[r] < 0) cnt[r] = 0;
        kmax = cnt[r] > kmax ? cnt[r] : kmax;
        acc[r] = 0.0;
    }
    for (int k = 0; k < kmax; ++k) {
        const double xk = x[k];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (k < cnt[r]) {
                const double d = x[k + lag[r]] - xk;
                acc[r] = acc[r] + d * d;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = q + r * Q;
        if (i < nlag) msd0[(int64_t)i * ntraj + t0 + j] = cnt[r] > 0 ? acc[r] / (double)cnt[r] : 0.0;
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

template <int R>
static cudaError_t launch_msd_smem(const double* frames, int nframe, int64_t ntraj, int G, const int64_t* lags,
                                   int nlag, double* msd0, cudaStream_t s) {
    const size_t smem = (size_t)G * (size_t)nframe * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(msd_smem_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t nblk = (ntraj + G - 1) / G;
    msd_smem_kernel<R><<<(unsigned)nblk, kMsdBlock, smem, s>>>(frames, nframe, ntraj, G, lags, nlag, msd0);
    return cudaGetLastError();
}

int launch_msd(const double* frames, int64_t nframe, int64_t ntraj, const int64_t* lags, int64_t nlag,
               double* msd0, double* msd_sum, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t per_traj = nframe * (int64_t)sizeof(double);
    int G = (int)(kMsdSmemBytes / (per_traj > 0 ? per_traj : 1));
    if (G > 32) G = 32;
    cudaError_t e = cudaErrorInvalidValue;
    bool done = false;
    if (G >= 1 && nframe < (1 << 30) && nlag < (1 << 30)) {
        const int Q = kMsdBlock / G;
        const int64_t R = (nlag + Q - 1) / Q;
        done = true;
        if (R <= 1) e = launch_msd_smem<1>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0, s);
        else if (R <= 2) e = launch_msd_smem<2>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0, s);
        else if (R <= 4) e = launch_msd_smem<4>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0, s);
        else if (R <= 8) e = launch_msd_smem<8>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0, s);
        else if (R <= 16) e = launch_msd_smem<16>(frames, (int)nframe, ntraj, G, lags, (int)nlag, msd0, s);
        else done = false;
    }
    if (!done) {
        const int block = 128;
        dim3 grid((unsigned)((ntraj + block - 1) / block), (unsigned)nlag);
        msd_traj_kernel<<<grid, block, 0, s>>>(frames, nframe, ntraj, lags, nlag, msd0);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return (int)e;
    msd_reduce_kernel<256><<<(unsigned)nlag, 256, 0, s>>>(msd0, ntraj, msd_sum);
    return (int)cudaGetLastError();
}

}  // namespace ldp
