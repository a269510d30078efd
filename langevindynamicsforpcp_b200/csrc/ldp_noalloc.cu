// ldp_noalloc.cu -- FP64 trajectory integration that allocates no memory.
//
// For callers that must not allocate device memory themselves or through
// the library: code that runs under a fixed device-memory budget owned by a
// host application or framework allocator, real-time loops that cannot
// afford an allocation (and the device synchronization cudaFree implies) in
// their critical path, and plugins that may only touch buffers their host
// hands them.  The caller passes the parameters and its own device buffers
// for the outputs; the per-trajectory working state the integration needs
// (positions, statistics state, cell-table rings) lives in one file-scope
// device array of fixed size, kScratchBytes, that every GPU which loads this
// library's module holds until the process exits.
//
// The kernels are the FP64 plain kernels of ldp_fp64.cu, launched with the
// same cell-table ring size and the same launch chunking a job uses, so the
// outputs equal those of ldp_job_create/ldp_submit for the same parameters,
// layout and table_slots.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "ldp_engine.h"

namespace {

// Bytes of working state per trajectory at `slots` cell-table ring slots:
// 9 FP64 and 9 int64 fields, 4 int32 fields, the FPTCG clocks and wells and
// the ring's tags and data.
constexpr int64_t per_traj_bytes(int64_t slots) {
    return 9 * 8 + 9 * 8 + 4 * 4 + 2 * LDP_MAX_CG * 8 + 2 * slots * 8;
}
// 12 arrays, each padded to 256 bytes.
constexpr size_t kScratchBytes =
    (size_t)LDP_NOALLOC_MAX_TRAJ * per_traj_bytes(LDP_NOALLOC_MAX_SLOTS) + 12 * 256;

// The working state shared by every call on a device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host-side device address of g_scratch, per device, valid for the CUDA
// context it was looked up in (the symbol name itself is not a device
// address in host code).  A context created after a cudaDeviceReset loads
// the module again, at another address, and has another id.
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    void* addr = nullptr;
};
std::mutex g_mu;
ScratchAddr g_addr[64];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context, through the driver entry
// points the runtime hands out (the library does not link libcuda itself).
cudaError_t current_ctx_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return e;
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return cudaErrorSymbolNotFound;
        get_current = (CtxGetCurrentFn)f0;
        get_id = (CtxGetIdFn)f1;
    }
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) return cudaErrorDeviceUninitialized;
    if (get_id(c, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
    return cudaSuccess;
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

void set_err(char* err, size_t n, const char* msg) {
    if (err && n) std::snprintf(err, n, "%s", msg);
}

}  // namespace

extern "C" ldp_status ldp_integrate_fp64_noalloc(const ldp_params* p, const ldp_job_opts* o, int64_t* d_counts,
                                                 double* d_sums, double* d_x_final, double* d_frames_x,
                                                 void* stream, char* err, size_t errlen) {
    if (!p || !o || !d_counts || !d_sums || !d_x_final) {
        set_err(err, errlen, "params, opts, counts, sums and x_final are required");
        return LDP_ERR_INVALID;
    }
    const int64_t ntraj = (int64_t)o->ranks * p->number_of_runs * o->lanes;
    if (o->ranks < 1 || o->lanes < 1 || p->number_of_runs < 1 || ntraj > LDP_NOALLOC_MAX_TRAJ) {
        char m[160];
        std::snprintf(m, sizeof(m), "ranks x runs x lanes = %lld trajectories; this entry point takes 1 to %d",
                      (long long)ntraj, LDP_NOALLOC_MAX_TRAJ);
        set_err(err, errlen, m);
        return LDP_ERR_INVALID;
    }
    if (o->first_rank < 0 || ((int64_t)o->first_rank + o->ranks) * p->number_of_runs * o->lanes > ((int64_t)1 << 32)) {
        set_err(err, errlen, "first_rank must be >= 0 and (first_rank + ranks) x runs x lanes at most 2^32");
        return LDP_ERR_INVALID;
    }
    const int slots = o->table_slots;
    if (slots < 16 || slots > LDP_NOALLOC_MAX_SLOTS || (slots & (slots - 1))) {
        char m[160];
        std::snprintf(m, sizeof(m), "table_slots = %d; this entry point takes a power of two from 16 to %d",
                      slots, LDP_NOALLOC_MAX_SLOTS);
        set_err(err, errlen, m);
        return LDP_ERR_UNSUPPORTED;
    }
    if (o->precision != LDP_PREC_FP64_PLAIN || o->mode != LDP_MODE_FIXED_STEPS || o->event_cap > 0 ||
        p->waiting_time || p->n_cg > LDP_MAX_CG || p->freq_save < 1 || !(p->timestep > 0.0) ||
        !(p->periodic_length > 0.0) || p->number_of_previous_steps) {
        set_err(err, errlen, "FP64 plain fixed-step runs only: no event lists (event_cap <= 0), WAITINGTIME off, at "
                             "most 16 FPTCG entries, positive TIMESTEP and PERIODICLENGTH, FREQSAVE >= 1, no "
                             "restart (NUMBEROFPREVIOUSSTEPS 0)");
        return LDP_ERR_UNSUPPORTED;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_err(err, errlen, "no current CUDA device");
        return LDP_ERR_DEVICE;
    }
    // Set-up, once per device and context, with that device current: the
    // device address of the scratch array.  cudaSetDevice makes the device's
    // primary context current on this thread (and creates it on first use),
    // so the context id below is the one the launches run in.
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        cudaError_t e = cudaSetDevice(dev);
        unsigned long long id = 0;
        if (e == cudaSuccess) e = current_ctx_id(&id);
        if (e == cudaSuccess && (!g_addr[dev].addr || g_addr[dev].ctx_id != id)) {
            void* a = nullptr;
            e = cudaGetSymbolAddress(&a, g_scratch);
            if (e == cudaSuccess) {
                g_addr[dev].addr = a;
                g_addr[dev].ctx_id = id;
            }
        }
        if (e != cudaSuccess) {
            set_err(err, errlen, cudaGetErrorString(e));
            return LDP_ERR_DEVICE;
        }
        base = g_addr[dev].addr;
    }

    ldp_job_opts opts = *o;
    opts.tick_cap = 0;
    ldp::KConst k;
    const uint32_t seed = (uint32_t)(p->random_seed < 0 ? 0 : p->random_seed);
    ldp::prepare_kconst(*p, opts, seed, &k);
    k.tick_cap = 0;

    // Carve the working state out of the scratch array.
    const int64_t n = ntraj;
    char* a = (char*)base;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* q = a + off; off += al256(bytes); return q; };
    ldp::TrajState S{};
    S.n = n;
    double* dd = (double*)take(sizeof(double) * 9 * n);
    S.x = d_x_final; S.v = dd + n; S.F = dd + 2 * n; S.rprev = dd + 3 * n; S.fpt_last = dd + 4 * n;
    S.fpt2_last = dd + 5 * n; S.tpt_last = dd + 6 * n; S.tpt2_last = dd + 7 * n; S.v0 = dd + 8 * n;
    int64_t* ii = (int64_t*)take(sizeof(int64_t) * 9 * n);
    S.cell = ii; S.well = ii + n; S.init_idx0 = ii + 2 * n; S.init_idx1 = ii + 3 * n; S.idx2_0 = ii + 4 * n;
    S.idx2_1 = ii + 5 * n; S.tpt2_well = ii + 6 * n; S.wt_tick = ii + 7 * n; S.nflip = ii + 8 * n;
    int32_t* i32 = (int32_t*)take(sizeof(int32_t) * 4 * n);
    S.state = i32; S.lb = i32 + n; S.bits = i32 + 2 * n; S.state0 = i32 + 3 * n;
    S.cg_last = (double*)take(sizeof(double) * LDP_MAX_CG * n);
    S.cg_well = (int64_t*)take(sizeof(int64_t) * LDP_MAX_CG * n);
    S.ring_tag = (int64_t*)take(sizeof(int64_t) * slots * n);
    S.ring_data = (int64_t*)take(sizeof(int64_t) * slots * n);
    S.counts = d_counts;
    S.sums = d_sums;
    S.ticks = nullptr;
    S.fx = d_frames_x;
    S.fv = S.ff = S.fb = S.fpe = S.fke = S.fst = nullptr;
    if (off > kScratchBytes) {
        set_err(err, errlen, "scratch layout exceeds the static array");
        return LDP_ERR_INVALID;
    }
    // WRITEX series need caller buffers this entry point does not take.
    k.write_x = 0;

    // The init kernel writes every field of every trajectory, clears the
    // cell-table rings and zeroes the counts and sums: no state of an earlier
    // call survives into this one.
    int e = ldp::launch_fp64_init(k, S, k.g0, 128, stream);
    if (e) {
        set_err(err, errlen, cudaGetErrorString((cudaError_t)e));
        return LDP_ERR_DEVICE;
    }
    // Steps per launch as a job chooses them: o->steps_per_launch, else about
    // 2^31 trajectory-steps per launch (clamped to 4096 .. 2^24 steps).
    uint64_t spl = o->steps_per_launch;
    if (!spl) {
        spl = (uint64_t)(((int64_t)1 << 31) / std::max<int64_t>(n, 1));
        spl = std::min<uint64_t>(std::max<uint64_t>(spl, 4096), (uint64_t)1 << 24);
    }
    const uint64_t nsteps = ldp::effective_steps(*p);
    for (uint64_t s0 = 1; s0 <= nsteps; s0 += spl) {
        const uint64_t s1 = std::min<uint64_t>(s0 + spl, nsteps + 1);
        e = ldp::launch_fp64_steps(k, S, k.g0, s0, s1, 128, stream);
        if (e) {
            set_err(err, errlen, cudaGetErrorString((cudaError_t)e));
            return LDP_ERR_DEVICE;
        }
    }
    set_err(err, errlen, "");
    return LDP_OK;
}
