"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the cpu_baseline leg of bench.py, as the checker.  The product never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, os.path.dirname(HERE))
from langevindynamicsforpcp_b200 import _lib as L  # noqa: E402  (struct layouts only)


class Cfg(C.Structure):
    _fields_ = [("traj_begin", C.c_int64), ("traj_end", C.c_int64), ("lanes", C.c_int32), ("ranks", C.c_int32),
                ("table_slots", C.c_int32), ("tick_cap", C.c_int64), ("seed", C.c_uint32), ("job_id", C.c_uint32),
                ("mode", C.c_int32), ("step_cap", C.c_uint64), ("event_cap", C.c_int64)]


_h = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _h
    if _h is None:
        if not os.path.exists(LIB):
            build()
        h = C.CDLL(LIB)
        h.ldpo_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        h.ldpo_log.restype = C.c_double
        h.ldpo_log.argtypes = [C.c_double]
        h.ldpo_sincos2pi.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        h.ldpo_expm1.restype = C.c_double
        h.ldpo_expm1.argtypes = [C.c_double]
        h.ldpo_prob_to_u64.restype = C.c_uint64
        h.ldpo_prob_to_u64.argtypes = [C.c_double]
        h.ldpo_effective_steps.restype = C.c_uint64
        h.ldpo_effective_steps.argtypes = [C.POINTER(L.Params)]
        h.ldpo_nframe.restype = C.c_int64
        h.ldpo_nframe.argtypes = [C.POINTER(L.Params)]
        h.ldpo_lags.restype = C.c_int64
        h.ldpo_lags.argtypes = [C.POINTER(L.Params), C.POINTER(C.c_int64), C.c_int64]
        h.ldpo_run.restype = C.c_int
        h.ldpo_run.argtypes = [C.POINTER(L.Params), C.POINTER(Cfg), C.POINTER(L.TrajResults)]
        h.ldpo_msd_traj.argtypes = [C.POINTER(C.c_double), C.c_int64, C.c_int64, C.POINTER(C.c_int64), C.c_int64,
                                    C.POINTER(C.c_double)]
        _h = h
    return _h


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().ldpo_philox4x32_10(c, k, o)
    return list(o)


def log(u):
    return lib().ldpo_log(u)


def sincos2pi(t):
    s, c = C.c_double(), C.c_double()
    lib().ldpo_sincos2pi(t, C.byref(s), C.byref(c))
    return s.value, c.value


def expm1(x):
    return lib().ldpo_expm1(x)


def lags(params):
    buf = np.zeros(4096, np.int64)
    n = lib().ldpo_lags(C.byref(params), buf.ctypes.data_as(C.POINTER(C.c_int64)), 4096)
    assert n > 0
    return buf[:n].copy()


def run(params, seed, lanes=8, ranks=1, traj_begin=0, traj_end=None, table_slots=256, tick_cap=0, job_id=0,
        mode=0, step_cap=0, frames=True, event_cap=0):
    """Runs the oracle; returns the same dict layout as Job.results()."""
    ntot = ranks * params.number_of_runs * lanes
    if traj_end is None:
        traj_end = ntot
    n = traj_end - traj_begin
    cfg = Cfg(traj_begin, traj_end, lanes, ranks, table_slots, tick_cap, seed & 0xffffffff, job_id, mode, step_cap,
              event_cap)
    nf = int(lib().ldpo_nframe(C.byref(params))) if mode == 0 else 0
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

    def p(a, ct):
        return a.ctypes.data_as(C.POINTER(ct))

    r.counts = p(out["counts"], C.c_int64)
    r.sums = p(out["sums"], C.c_double)
    r.state0 = p(out["state0"], C.c_int32)
    r.v0 = p(out["v0"], C.c_double)
    r.x_final = p(out["x_final"], C.c_double)
    r.v_final = p(out["v_final"], C.c_double)
    r.state_final = p(out["state_final"], C.c_int32)
    if tick_cap > 0:
        out["ticks"] = np.zeros((n, tick_cap), np.int64)
        r.ticks = p(out["ticks"], C.c_int64)
    if event_cap > 0:
        out["events"] = np.zeros((L.E_CG0 + params.n_cg, n, event_cap), np.float64)
        out["event_states"] = np.zeros((n, event_cap), np.uint8)
        r.events = p(out["events"], C.c_double)
        r.event_states = p(out["event_states"], C.c_uint8)
    if frames and nf > 0:
        out["frames_x"] = np.zeros((nf, n), np.float64)
        r.frames_x = p(out["frames_x"], C.c_double)
        if params.write_x:
            for k in ("frames_v", "frames_f", "frames_barrier", "frames_pe", "frames_ke", "frames_state"):
                out[k] = np.zeros((nf, n), np.float64)
                setattr(r, k, p(out[k], C.c_double))
    rc = lib().ldpo_run(C.byref(params), C.byref(cfg), C.byref(r))
    assert rc == 0
    return out


def msd_traj(frames_x, lag_list):
    nf, n = frames_x.shape
    fx = np.ascontiguousarray(frames_x)
    lg = np.ascontiguousarray(lag_list, dtype=np.int64)
    out = np.zeros((len(lg), n), np.float64)
    lib().ldpo_msd_traj(fx.ctypes.data_as(C.POINTER(C.c_double)), nf, n, lg.ctypes.data_as(C.POINTER(C.c_int64)),
                        len(lg), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out
