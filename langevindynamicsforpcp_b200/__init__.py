"""B200 trajectory engine for the single- and double-barrier Langevin models
of LangevinDynamicsForPCP.

Python mirror of the C ABI in include/ldp.h.  The names follow the
reference: a :class:`Job` is one ``.inp`` run of ``ranks x runs x lanes``
trajectories (the reference's ``nrun``); its results are the per-trajectory
event counts and sums behind ``GetFirstPassageTimeAverage`` & co., the saved
frames, and the MSD curve of ``LangevinEquationRunnerMPI::Run``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import (MODEL_SINGLE, MODEL_DOUBLE, PREC_FP64_PLAIN, PREC_FP32_BATCHED,  # noqa: F401
                   MODE_FIXED_STEPS, MODE_FIRST_PASSAGE, LdpError, Params, JobOpts)

__all__ = ["Context", "Job", "default_params", "params_from_inp", "params_from_inp_text",
           "restart_inspect", "restart_rewrite", "MODEL_SINGLE", "MODEL_DOUBLE", "LdpError"]


def _check(st: int, ctx=None):
    if st != 0:
        msg = ""
        if ctx is not None and ctx.handle:
            msg = (L.lib().ldp_last_error(ctx.handle) or b"").decode()
        raise LdpError(st, msg)


def default_params(model: int = MODEL_SINGLE) -> Params:
    p = Params()
    L.lib().ldp_params_default(model, C.byref(p))
    return p


def params_from_inp(path: str, model: int = MODEL_SINGLE) -> Params:
    p = Params()
    err = C.create_string_buffer(1024)
    st = L.lib().ldp_params_from_inp(path.encode(), model, C.byref(p), err, 1024)
    if st != 0:
        raise LdpError(st, err.value.decode())
    return p


def params_from_inp_text(text: str, model: int = MODEL_SINGLE, base_dir: str = "") -> Params:
    p = Params()
    err = C.create_string_buffer(1024)
    st = L.lib().ldp_params_from_inp_text(text.encode(), base_dir.encode(), model, C.byref(p), err, 1024)
    if st != 0:
        raise LdpError(st, err.value.decode())
    return p


class Context:
    """One CUDA device and its stream (ldp_create / ldp_destroy)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = L.lib().ldp_create(C.byref(h), device)
        if st != 0:
            raise LdpError(st, f"ldp_create(device={device})")
        self.handle = h

    def last_error(self) -> str:
        return (L.lib().ldp_last_error(self.handle) or b"").decode()

    def set_fp64_latency(self, max_traj: int) -> None:
        """FP64 plain fixed-step jobs with at most max_traj trajectories run
        in latency mode (ldp_ctx_set_fp64_latency; 0 disables it)."""
        st = L.lib().ldp_ctx_set_fp64_latency(self.handle, max_traj)
        if st != 0:
            raise LdpError(st, "ldp_ctx_set_fp64_latency")

    def set_fp64_group(self, max_traj: int) -> None:
        """FP64 plain fixed-step jobs above the latency-mode limit and with at
        most max_traj trajectories run in group mode (ldp_ctx_set_fp64_group;
        0 disables it)."""
        st = L.lib().ldp_ctx_set_fp64_group(self.handle, max_traj)
        if st != 0:
            raise LdpError(st, "ldp_ctx_set_fp64_group")

    def close(self):
        if self.handle:
            L.lib().ldp_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Job:
    """One run of a parameter set (ldp_job_create ... ldp_job_destroy)."""

    def __init__(self, ctx: Context, params: Params, lanes: int = 8, ranks: int = 1,
                 precision: int = PREC_FP64_PLAIN, mode: int = MODE_FIXED_STEPS,
                 step_cap: int = 100_000_000, table_slots: int = 256, tick_cap: int = -1,
                 job_id: int = 0, steps_per_launch: int = 0, block_size: int = 0, event_cap: int = 0,
                 first_rank: int = 0):
        self.ctx = ctx
        o = JobOpts()
        L.lib().ldp_job_opts_default(C.byref(o))
        o.lanes, o.ranks, o.precision, o.mode = lanes, ranks, precision, mode
        o.step_cap, o.table_slots, o.tick_cap, o.job_id = step_cap, table_slots, tick_cap, job_id
        o.steps_per_launch, o.block_size, o.event_cap = steps_per_launch, block_size, event_cap
        o.first_rank = first_rank
        self.opts = o
        self.params = params
        h = C.c_void_p()
        _check(L.lib().ldp_job_create(ctx.handle, C.byref(params), C.byref(o), C.byref(h)), ctx)
        self.handle = h

    @classmethod
    def borrowed(cls, ctx: Context, handle) -> "Job":
        """A view of a job owned elsewhere (a serving loop): results only;
        close() does not destroy it."""
        j = cls.__new__(cls)
        j.ctx, j.opts, j.params = ctx, None, None
        j.handle = C.c_void_p(handle.value if isinstance(handle, C.c_void_p) else handle)
        j._borrowed = True
        return j

    # -- execution ---------------------------------------------------------
    def submit(self) -> "Job":
        _check(L.lib().ldp_submit(self.ctx.handle, self.handle), self.ctx)
        return self

    def poll(self) -> bool:
        d = C.c_int(0)
        _check(L.lib().ldp_poll(self.ctx.handle, self.handle, C.byref(d)), self.ctx)
        return bool(d.value)

    def wait(self) -> "Job":
        _check(L.lib().ldp_wait(self.ctx.handle, self.handle), self.ctx)
        return self

    def run(self) -> "Job":
        return self.submit().wait()

    # -- restart files (ReadRestartFile / WriteRestartFile) -----------------
    def restore(self, input_base: str) -> "Job":
        """Loads <input_base>_<rank>_<trial>.restart before submission; the
        params' NUMBEROFPREVIOUSSTEPS must equal the files' step count."""
        _check(L.lib().ldp_job_restore(self.handle, input_base.encode()), self.ctx)
        return self

    def save_restart(self, output_base: str) -> "Job":
        """Writes <output_base>_<rank>_<trial>.restart after the run (needs
        event_cap > 0, or -1 with WRITERESTART true)."""
        _check(L.lib().ldp_job_save_restart(self.handle, output_base.encode()), self.ctx)
        return self

    def keep_state(self) -> "Job":
        """FP32 batched: keep every trajectory's state at its last step, so
        that save_state can write it (before submission)."""
        _check(L.lib().ldp_job_keep_state(self.handle), self.ctx)
        return self

    def save_state(self, path: str) -> "Job":
        """FP32 batched: writes the kept state (ldp_job_save_state)."""
        _check(L.lib().ldp_job_save_state(self.handle, path.encode()), self.ctx)
        return self

    def load_state(self, path: str) -> "Job":
        """FP32 batched: continues from a saved state (before submission);
        NUMBEROFPREVIOUSSTEPS must equal its step count."""
        _check(L.lib().ldp_job_load_state(self.handle, path.encode()), self.ctx)
        return self

    # -- introspection -----------------------------------------------------
    @property
    def info(self) -> L.JobInfo:
        i = L.JobInfo()
        _check(L.lib().ldp_job_info_get(self.handle, C.byref(i)), self.ctx)
        return i

    def timing(self) -> dict:
        t = L.Timing()
        _check(L.lib().ldp_job_timing_get(self.handle, C.byref(t)), self.ctx)
        return {k: getattr(t, k) for k, _ in L.Timing._fields_}

    # -- results -----------------------------------------------------------
    def results(self, frames: bool = True, ticks: bool = True) -> dict:
        i = self.info
        n, nf, tc = i.ntraj, i.nframe, i.tick_cap
        out = {
            "counts": np.zeros((L.NCOUNT, n), np.int64),
            "sums": np.zeros((L.NSUM, n), np.float64),
            "state0": np.zeros(n, np.int32),
            "v0": np.zeros(n, np.float64),
            "x_final": np.zeros(n, np.float64),
            "v_final": np.zeros(n, np.float64),
            "state_final": np.zeros(n, np.int32),
        }
        r = L.TrajResults()
        r.counts = _ptr(out["counts"], C.c_int64)
        r.sums = _ptr(out["sums"], C.c_double)
        r.state0 = _ptr(out["state0"], C.c_int32)
        r.v0 = _ptr(out["v0"], C.c_double)
        r.x_final = _ptr(out["x_final"], C.c_double)
        r.v_final = _ptr(out["v_final"], C.c_double)
        r.state_final = _ptr(out["state_final"], C.c_int32)
        if ticks and tc > 0:
            out["ticks"] = np.zeros((n, tc), np.int64)
            r.ticks = _ptr(out["ticks"], C.c_int64)
        if i.event_cap > 0:
            out["events"] = np.zeros((L.E_CG0 + i.n_cg, n, i.event_cap), np.float64)
            out["event_states"] = np.zeros((n, i.event_cap), np.uint8)
            r.events = _ptr(out["events"], C.c_double)
            r.event_states = _ptr(out["event_states"], C.c_uint8)
        if frames and nf > 0:
            out["frames_x"] = np.zeros((nf, n), np.float64)
            r.frames_x = _ptr(out["frames_x"], C.c_double)
            if self.params.write_x:
                for k in ("frames_v", "frames_f", "frames_barrier", "frames_pe", "frames_ke", "frames_state"):
                    out[k] = np.zeros((nf, n), np.float64)
                    setattr(r, k, _ptr(out[k], C.c_double))
        _check(L.lib().ldp_job_traj_results(self.handle, C.byref(r)), self.ctx)
        return out

    def msd(self):
        i = self.info
        lags = np.zeros(i.nlag, np.int64)
        msd = np.zeros(i.nlag, np.float64)
        _check(L.lib().ldp_job_msd(self.handle, _ptr(lags, C.c_int64), _ptr(msd, C.c_double), i.nlag), self.ctx)
        return lags, msd

    def means(self) -> np.ndarray:
        """Per-trajectory mean event times [list][traj] (ldp_job_traj_means):
        the reference's per-lane averages, computed on the device."""
        i = self.info
        m = np.zeros((L.E_CG0 + i.n_cg, i.ntraj), np.float64)
        _check(L.lib().ldp_job_traj_means(self.handle, _ptr(m, C.c_double)), self.ctx)
        return m

    def msd_traj(self) -> np.ndarray:
        i = self.info
        m = np.zeros((i.nlag, i.ntraj), np.float64)
        _check(L.lib().ldp_job_msd_traj(self.handle, _ptr(m, C.c_double)), self.ctx)
        return m

    def write_outputs(self, directory: str = "."):
        _check(L.lib().ldp_job_write_outputs(self.handle, directory.encode()), self.ctx)

    def close(self):
        if self.handle and not getattr(self, "_borrowed", False):
            L.lib().ldp_job_destroy(self.handle)
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def restart_inspect(params: Params, path: str) -> dict:
    """Summary of one .restart file and the per-lane counts and sums a job
    restored from it starts with (ldp_restart_inspect)."""
    s = L.RestartSummary()
    err = C.create_string_buffer(1024)
    st = L.lib().ldp_restart_inspect(C.byref(params), path.encode(), C.byref(s), None, None, err, 1024)
    if st != 0:
        raise LdpError(st, err.value.decode())
    counts = np.zeros((L.NCOUNT, s.lanes), np.int64)
    sums = np.zeros((L.NSUM, s.lanes), np.float64)
    st = L.lib().ldp_restart_inspect(C.byref(params), path.encode(), C.byref(s), _ptr(counts, C.c_int64),
                                     _ptr(sums, C.c_double), err, 1024)
    if st != 0:
        raise LdpError(st, err.value.decode())
    return {"lanes": s.lanes, "rank": s.rank, "steps": s.steps, "frames": s.frames,
            "has_exact_resume": bool(s.has_exact_resume), "ncell": list(s.ncell), "min_id": list(s.min_id),
            "counts": counts, "sums": sums}


def restart_rewrite(params: Params, src: str, dst: str) -> None:
    """Reads a .restart file and writes it again (ldp_restart_rewrite)."""
    err = C.create_string_buffer(1024)
    st = L.lib().ldp_restart_rewrite(C.byref(params), src.encode(), dst.encode(), err, 1024)
    if st != 0:
        raise LdpError(st, err.value.decode())


def submit_batch(ctx: Context, jobs, graph: bool = False) -> None:
    """Submits several jobs together (ldp_submit_batch): FP32 batched jobs
    share every persistent launch.  graph=True (FP32 batched jobs only) runs
    all launches and post-processing as one CUDA graph
    (ldp_submit_batch_graph)."""
    arr = (C.c_void_p * len(jobs))(*[j.handle for j in jobs])
    fn = L.lib().ldp_submit_batch_graph if graph else L.lib().ldp_submit_batch
    _check(fn(ctx.handle, arr, len(jobs)), ctx)


def _ctx_mark(self, mark: int) -> None:
    _check(L.lib().ldp_ctx_mark(self.handle, mark), self)


def _ctx_elapsed_ms(self, a: int, b: int) -> float:
    ms = C.c_double()
    _check(L.lib().ldp_ctx_elapsed_ms(self.handle, a, b, C.byref(ms)), self)
    return ms.value


def _ctx_synchronize(self) -> None:
    _check(L.lib().ldp_ctx_synchronize(self.handle), self)


Context.mark = _ctx_mark
Context.elapsed_ms = _ctx_elapsed_ms
Context.synchronize = _ctx_synchronize
