// ldp_msd.h -- launchers of the MSD and per-trajectory mean kernels.
#pragma once
#include <cstdint>

namespace ldp {

// Which MSD kernel: FP64 (FP64 plain jobs, bit-identical to the oracle);
// FP32 staged (FP32 batched jobs); its lean instance (same results, sized to
// run beside the persistent FP32 kernel).
enum MsdMode { LDP_MSD_FP64 = 0, LDP_MSD_FP32 = 1, LDP_MSD_FP32_LEAN = 2 };

int launch_msd(const double* frames, int64_t nframe, int64_t ntraj, const int64_t* lags, int64_t nlag,
               double* msd0, double* msd_sum, void* stream, int mode);
int launch_traj_means(const int64_t* counts, const double* sums, double* means, int64_t n, int ncg, void* stream);

}  // namespace ldp
