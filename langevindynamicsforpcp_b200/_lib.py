"""ctypes binding of include/ldp.h (libldp.so, built in-tree by ``make``).

The structures below mirror the C declarations field for field.  Loading
fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libldp.so")

LDP_MAX_CG = 16
LDP_PATH_MAX = 512

MODEL_SINGLE, MODEL_DOUBLE = 0, 1
PREC_FP64_PLAIN, PREC_FP32_BATCHED = 0, 1
MODE_FIXED_STEPS, MODE_FIRST_PASSAGE = 0, 1

# enum ldp_count_field
(C_FPT, C_FPT2, C_TPT, C_TPT2, C_INIT0, C_INIT1, C_INST0, C_INST1, C_STATE0, C_STATE1,
 C_WT, C_EVICT, C_FLAGS, C_STEPS, C_CG0) = range(15)
NCOUNT = C_CG0 + LDP_MAX_CG
# enum ldp_sum_field
S_FPT, S_FPT2, S_TPT, S_TPT2, S_FIRST_FPT, S_FIRST_FPT2, S_FIRST_TPT, S_FIRST_TPT2, S_CG0 = range(9)
NSUM = S_CG0 + LDP_MAX_CG

FLAG_NONFINITE, FLAG_TICK_OVERFLOW, FLAG_CENSORED, FLAG_EVENT_OVERFLOW = 1, 2, 4, 8
# enum ldp_event_list
E_FPT, E_FPT2, E_TPT, E_TPT2, E_CG0 = range(5)
NOALLOC_MAX_TRAJ = 4096
NOALLOC_MAX_SLOTS = 256

STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "device error", 4: "timeout",
          5: "i/o error", 6: "parse error", 7: "unsupported", 8: "not ready", 9: "restart error"}


class Params(C.Structure):
    _fields_ = [
        ("model", C.c_int32), ("overdamped", C.c_int32),
        ("x0", C.c_double), ("v0", C.c_double), ("gamma", C.c_double), ("kb", C.c_double),
        ("temperature", C.c_double), ("mass", C.c_double),
        ("randomize_v", C.c_int32),
        ("periodic_length", C.c_double),
        ("barrier_heights", (C.c_double * 2) * 2),
        ("barrier_half_width", C.c_double * 2),
        ("barrier_position", C.c_double * 2),
        ("timestep", C.c_double),
        ("number_of_steps", C.c_uint64), ("number_of_previous_steps", C.c_uint64),
        ("number_of_runs", C.c_int32),
        ("freq_save", C.c_uint64), ("freq_stat", C.c_uint64),
        ("distribution_v0", C.c_int32), ("distribution_s0", C.c_int32),
        ("tau", C.c_double),
        ("initial_state", C.c_int32), ("randomize_states", C.c_int32), ("uniform_initial_states", C.c_int32),
        ("eq", C.c_int32), ("eq_constant", C.c_double),
        ("waiting_time", C.c_int32), ("fpt", C.c_int32), ("tpt", C.c_int32), ("fptcg", C.c_int32),
        ("n_cg", C.c_int32), ("cg_sizes", C.c_int32 * LDP_MAX_CG),
        ("read_restart", C.c_int32), ("write_restart", C.c_int32),
        ("input_restart", C.c_char * LDP_PATH_MAX), ("output_restart", C.c_char * LDP_PATH_MAX),
        ("output_base", C.c_char * LDP_PATH_MAX),
        ("write_x", C.c_int32),
        ("number_of_log_samples", C.c_uint64),
        ("random_seed", C.c_int64),
        ("print_timer", C.c_int32),
    ]


class JobOpts(C.Structure):
    _fields_ = [
        ("lanes", C.c_int32), ("ranks", C.c_int32), ("precision", C.c_int32), ("mode", C.c_int32),
        ("step_cap", C.c_uint64), ("table_slots", C.c_int32), ("tick_cap", C.c_int64),
        ("job_id", C.c_uint32), ("steps_per_launch", C.c_uint64), ("block_size", C.c_int32),
        ("keep_frames", C.c_int32), ("first_rank", C.c_int32), ("event_cap", C.c_int64),
    ]


class JobInfo(C.Structure):
    _fields_ = [("ntraj", C.c_int64), ("nframe", C.c_int64), ("nlag", C.c_int64), ("steps", C.c_int64),
                ("tick_cap", C.c_int64), ("n_cg", C.c_int32), ("precision", C.c_int32), ("mode", C.c_int32),
                ("done", C.c_int32), ("device_bytes", C.c_int64), ("event_cap", C.c_int64),
                ("steps_before", C.c_int64)]


_DP = C.POINTER(C.c_double)
_I64P = C.POINTER(C.c_int64)
_I32P = C.POINTER(C.c_int32)


class TrajResults(C.Structure):
    _fields_ = [("counts", _I64P), ("sums", _DP), ("state0", _I32P), ("v0", _DP), ("x_final", _DP),
                ("v_final", _DP), ("state_final", _I32P), ("ticks", _I64P), ("frames_x", _DP),
                ("frames_v", _DP), ("frames_f", _DP), ("frames_barrier", _DP), ("frames_pe", _DP),
                ("frames_ke", _DP), ("frames_state", _DP), ("events", _DP),
                ("event_states", C.POINTER(C.c_uint8))]


class RestartSummary(C.Structure):
    _fields_ = [("lanes", C.c_int32), ("rank", C.c_int32), ("steps", C.c_uint64), ("frames", C.c_int64),
                ("has_exact_resume", C.c_int32), ("pad", C.c_int32), ("ncell", C.c_int64 * 2),
                ("min_id", C.c_int32 * 2)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget", C.c_int64), ("pair_budget", C.c_int64), ("max_inflight", C.c_int32),
                ("region", C.c_int32)]


class ServerInfo(C.Structure):
    _fields_ = [("queued", C.c_int64), ("running", C.c_int64), ("finishing", C.c_int64), ("done", C.c_int64),
                ("hbm_in_use", C.c_int64), ("hbm_budget", C.c_int64), ("launches", C.c_int64), ("steps", C.c_int64),
                ("phase_s", C.c_double * 6), ("phase_max_s", C.c_double * 6)]


SRV_QUEUED, SRV_RUNNING, SRV_FINISHING, SRV_DONE, SRV_FAILED = range(5)


class Timing(C.Structure):
    _fields_ = [("integrate_ms", C.c_double), ("msd_ms", C.c_double), ("reduce_ms", C.c_double),
                ("launches", C.c_int64), ("particle_steps", C.c_int64)]


# Every function declared in include/ldp.h, with its ctypes signature.
SIGNATURES = {
    "ldp_abi_version": (C.c_int, []),
    "ldp_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "ldp_destroy": (None, [C.c_void_p]),
    "ldp_last_error": (C.c_char_p, [C.c_void_p]),
    "ldp_status_string": (C.c_char_p, [C.c_int]),
    "ldp_ctx_set_fp32_shape": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int]),
    "ldp_ctx_get_fp32_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_uint64), C.POINTER(C.c_int)]),
    "ldp_params_default": (None, [C.c_int, C.POINTER(Params)]),
    "ldp_params_from_inp": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(Params), C.c_char_p, C.c_size_t]),
    "ldp_params_from_inp_text": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(Params), C.c_char_p,
                                           C.c_size_t]),
    "ldp_write_default_inp": (C.c_int, [C.c_char_p, C.c_int]),
    "ldp_job_opts_default": (None, [C.POINTER(JobOpts)]),
    "ldp_job_create": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(JobOpts), C.POINTER(C.c_void_p)]),
    "ldp_job_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "ldp_submit": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ldp_submit_batch": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int]),
    "ldp_submit_batch_graph": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int]),
    "ldp_ctx_mark": (C.c_int, [C.c_void_p, C.c_int]),
    "ldp_ctx_elapsed_ms": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "ldp_ctx_synchronize": (C.c_int, [C.c_void_p]),
    "ldp_poll": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "ldp_wait": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ldp_job_info_get": (C.c_int, [C.c_void_p, C.POINTER(JobInfo)]),
    "ldp_job_timing_get": (C.c_int, [C.c_void_p, C.POINTER(Timing)]),
    "ldp_job_destroy": (None, [C.c_void_p]),
    "ldp_job_traj_results": (C.c_int, [C.c_void_p, C.POINTER(TrajResults)]),
    "ldp_job_msd": (C.c_int, [C.c_void_p, _I64P, _DP, C.c_int64]),
    "ldp_job_msd_traj": (C.c_int, [C.c_void_p, _DP]),
    "ldp_job_traj_means": (C.c_int, [C.c_void_p, _DP]),
    "ldp_job_write_outputs": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ldp_run_inp": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(JobOpts), C.c_char_p]),
    "ldp_server_opts_default": (None, [C.POINTER(ServerOpts)]),
    "ldp_server_create": (C.c_int, [C.c_void_p, C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]),
    "ldp_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(JobOpts), C.POINTER(C.c_uint64)]),
    "ldp_server_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "ldp_server_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "ldp_server_job": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_void_p)]),
    "ldp_server_job_times": (C.c_int, [C.c_void_p, C.c_uint64, _DP]),
    "ldp_server_take_ended": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.c_int64, C.POINTER(C.c_int64)]),
    "ldp_server_release": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ldp_server_info_get": (C.c_int, [C.c_void_p, C.POINTER(ServerInfo)]),
    "ldp_server_destroy": (None, [C.c_void_p]),
    "ldp_ctx_set_fp64_latency": (C.c_int, [C.c_void_p, C.c_int64]),
    "ldp_ctx_set_fp64_group": (C.c_int, [C.c_void_p, C.c_int64]),
    "ldp_job_keep_state": (C.c_int, [C.c_void_p]),
    "ldp_job_save_state": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ldp_job_load_state": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ldp_inp_print_values": (C.c_int, [C.c_char_p, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "ldp_integrate_fp64_noalloc": (C.c_int, [C.POINTER(Params), C.POINTER(JobOpts), C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]),
    "ldp_job_restore": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ldp_job_save_restart": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ldp_restart_inspect": (C.c_int, [C.POINTER(Params), C.c_char_p, C.POINTER(RestartSummary), _I64P, _DP,
                                      C.c_char_p, C.c_size_t]),
    "ldp_restart_rewrite": (C.c_int, [C.POINTER(Params), C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]),
}

_lib = None


class LdpError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}" if msg else STATUS.get(status, str(status)))


ABI_VERSION = 2   # LDP_ABI_VERSION of include/ldp.h that these structures mirror


def lib() -> C.CDLL:
    """Loads libldp.so once; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
                               "(there is no CPU fallback)")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        if h.ldp_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {h.ldp_abi_version()}, these bindings expect "
                               f"{ABI_VERSION}: rebuild it with `make -C {HERE}`")
        _lib = h
    return _lib
