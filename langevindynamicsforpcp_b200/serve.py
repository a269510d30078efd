"""Serving: a request loop over the library's serving loop (ldp_server_*).

Jobs (.inp parameter sets) arrive over time; the C++ serving loop admits
them by device-memory footprint, runs them in the shared persistent launches
(one launch covers every model type) while other jobs are in flight
(continuous batching) and finishes each one as soon as its trajectories have
all retired.  This module
adds the request side: a Poisson arrival stream, per-job latency, and the
"serving" workload -- jobs of random type (single or double barrier, under-
or overdamped), parameters from the precision / batching / scan ranges,
trajectory counts 2^U[10, 18], seed 1234.  The reference runs one .inp per
MPI process; serving has no counterpart there.

    python -m langevindynamicsforpcp_b200.serve [--jobs N] [--loads 0.5 0.8]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import (Context, Job, MODEL_DOUBLE, MODEL_SINGLE, MODE_FIXED_STEPS, PREC_FP32_BATCHED, _check,
               params_from_inp_text)
from . import _lib as L

COMMON = """\
OUTPUTBASE serve
OVERDAMPED {over}
V0 1.0
GAMMA {gamma!r}
KB 1.0
TEMPERATURE 1.0
MASS 1.0
RANDOMIZEV true
PERIODICLENGTH 5.8
X0 -2.9
TIMESTEP 1.0e-5
NUMBEROFSTEPS {steps}
NUMBEROFPREVIOUSSTEPS 0
NUMBEROFRUNS 1
FREQSAVE {freq}
FREQSTAT 1
DISTRIBUTIONV0 false
DISTRIBUTIONS0 true
TAU {tau!r}
INITIALSTATE 0
RANDOMIZESTATES true
UNIFORMINITALSTATES false
EQ true 1.0
WAITINGTIME false
FPT true
TPT true
FPTCG true 2
FPTCG true 10
READRESTART false
WRITERESTART false
INPUTRESTART none
OUTPUTRESTART none
WRITEX false
NUMBEROFLOGSAMPLES 40
RANDOMSEED {seed}
PRINTTIMER false
"""
SINGLE = "BARRIERHEIGHTS {high!r} {low!r}\nBARRIERHALFWIDTH 0.65\n"
DOUBLE = ("BARRIERHEIGHTS0 {mid!r} {low!r}\nBARRIERHEIGHTS1 {high!r} {low!r}\nBARRIERHALFWIDTH0 0.70\n"
          "BARRIERHALFWIDTH1 0.65\nBARRIERPOSITION0 -1.42\nBARRIERPOSITION1 -0.56\n")


class Server:
    """The library's serving loop (ldp_server_create ... ldp_server_destroy)."""

    def __init__(self, ctx: Context, hbm_budget: int = 0, pair_budget: int = 1024, max_inflight: int = 2,
                 region: bool = True):
        """hbm_budget: bytes of job arenas resident at once (0: 80 % of the
        free device memory); region: allocate that budget once as one device
        region that arenas are placed in (else one pool allocation per job)."""
        self.ctx = ctx
        o = L.ServerOpts()
        L.lib().ldp_server_opts_default(C.byref(o))
        o.hbm_budget, o.pair_budget, o.max_inflight = hbm_budget, pair_budget, max_inflight
        o.region = int(region)
        h = C.c_void_p()
        _check(L.lib().ldp_server_create(ctx.handle, C.byref(o), C.byref(h)), ctx)
        self.handle = h
        self._ended = (C.c_uint64 * 4096)()

    def submit(self, params, lanes: int, job_id: int = 0) -> int:
        o = L.JobOpts()
        L.lib().ldp_job_opts_default(C.byref(o))
        o.lanes, o.ranks, o.precision, o.mode, o.job_id = lanes, 1, PREC_FP32_BATCHED, MODE_FIXED_STEPS, job_id
        t = C.c_uint64()
        _check(L.lib().ldp_server_submit(self.handle, C.byref(params), C.byref(o), C.byref(t)), self.ctx)
        return t.value

    def step(self) -> int:
        n = C.c_int(0)
        _check(L.lib().ldp_server_step(self.handle, C.byref(n)), self.ctx)
        return n.value

    def poll(self, ticket: int):
        st, lat = C.c_int(0), C.c_double(0)
        _check(L.lib().ldp_server_poll(self.handle, ticket, C.byref(st), C.byref(lat)), self.ctx)
        return st.value, lat.value

    def ended(self) -> list:
        """Tickets of the jobs that ended (done or failed) since the last call."""
        buf = self._ended
        cap = len(buf)
        n = C.c_int64(0)
        out = []
        while True:
            _check(L.lib().ldp_server_take_ended(self.handle, buf, cap, C.byref(n)), self.ctx)
            out.extend(buf[:n.value])
            if n.value < cap:
                return out

    def times(self, ticket: int):
        """(admitted, trajectories retired, done), seconds after submission."""
        t = (C.c_double * 3)()
        _check(L.lib().ldp_server_job_times(self.handle, ticket, t), self.ctx)
        return tuple(t)

    def job(self, ticket: int) -> Job:
        h = C.c_void_p()
        _check(L.lib().ldp_server_job(self.handle, ticket, C.byref(h)), self.ctx)
        return Job.borrowed(self.ctx, h)

    def release(self, ticket: int) -> None:
        _check(L.lib().ldp_server_release(self.handle, ticket), self.ctx)

    def info(self) -> dict:
        i = L.ServerInfo()
        _check(L.lib().ldp_server_info_get(self.handle, C.byref(i)), self.ctx)
        out = {k: getattr(i, k) for k, _ in L.ServerInfo._fields_}
        out["phase_s"], out["phase_max_s"] = list(i.phase_s), list(i.phase_max_s)
        return out

    def close(self):
        if self.handle:
            L.lib().ldp_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def serving_workload(n: int, seed: int = 1234, exp_lo: float = 10, exp_hi: float = 18, steps: int = 24000,
                     freq: int = 20):
    """n jobs: (params, ntraj, label).  Type uniform over {single, double} x
    {over-, underdamped}; H_low in {2, 3, 4, 5} (single: high 3.6 H; double:
    barrier 0 high 1.7 H, barrier 1 high 3.6 H), flip rate k logU[1e-2, 1e2]
    (TAU = 1/k), friction logU[0.1, 10]; CuIDB single/double geometry."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        dbl = bool(rng.integers(2))
        over = bool(rng.integers(2))
        h = float(rng.choice([2.0, 3.0, 4.0, 5.0]))
        k = float(10 ** rng.uniform(-2, 2))
        g = float(10 ** rng.uniform(-1, 1))
        ntraj = int(2 ** rng.uniform(exp_lo, exp_hi))
        text = COMMON.format(over="true" if over else "false", gamma=g, steps=steps, freq=freq, tau=1.0 / k,
                             seed=seed)
        text += (DOUBLE.format(mid=1.7 * h, high=3.6 * h, low=h) if dbl else SINGLE.format(high=3.6 * h, low=h))
        p = params_from_inp_text(text, MODEL_DOUBLE if dbl else MODEL_SINGLE)
        out.append((p, ntraj, {"double": dbl, "overdamped": over, "H": h, "k": k, "gamma": g, "ntraj": ntraj}))
    return out


def run_stream(server: Server, work, arrivals, on_done=None, timeout_s: float = 900.0, stages=None):
    """Submits work[i] at time arrivals[i] (seconds from now), drives the
    loop until every job is done; returns per-job latency (submission to
    done, seconds).  on_done(i, job) is called before each job is released;
    stages (an n x 3 array) receives each job's server.times()."""
    n = len(work)
    lat = np.full(n, np.nan)
    tickets = {}
    nxt = 0
    t0 = time.perf_counter()
    while nxt < n or tickets:
        now = time.perf_counter() - t0
        if now > timeout_s:
            raise TimeoutError(f"serving stream not finished after {timeout_s} s")
        while nxt < n and arrivals[nxt] <= now:
            p, ntraj, _ = work[nxt]
            tickets[server.submit(p, ntraj, job_id=nxt)] = nxt
            nxt += 1
        server.step()
        for t in server.ended():
            if t not in tickets:
                continue
            st, l = server.poll(t)
            i = tickets.pop(t)
            if st == L.SRV_FAILED:
                raise RuntimeError(f"job {i} failed: {server.ctx.last_error()}")
            lat[i] = l
            if stages is not None:
                stages[i] = server.times(t)
            if on_done:
                on_done(i, server.job(t))
            server.release(t)
        if not tickets and nxt < n:
            time.sleep(max(0.0, min(arrivals[nxt] - (time.perf_counter() - t0), 0.01)))
    return lat


def measure(jobs: int = 10000, exp_lo: float = 10, exp_hi: float = 18, steps: int = 24000, loads=(0.5, 0.8),
            isolated_sample: int = 24, device: int = 0, pair_budget: int = 1024, max_inflight: int = 2,
            hbm_budget: int = 0) -> dict:
    """Capacity (every job submitted at once), the capacity the loop sustains
    under Poisson arrivals, isolated solve times and, per offered load (a
    fraction of the smaller capacity), the latency distribution of a
    Poisson stream of the serving workload's jobs."""
    a = argparse.Namespace(jobs=jobs, exp_lo=exp_lo, exp_hi=exp_hi, steps=steps, loads=list(loads),
                           isolated_sample=isolated_sample)
    work = serving_workload(a.jobs, exp_lo=a.exp_lo, exp_hi=a.exp_hi, steps=a.steps)
    psteps = float(sum(n for _, n, _ in work)) * a.steps
    out = {"workload": f"serving: {a.jobs} jobs, types single/double x over/underdamped, "
                       f"2^U[{a.exp_lo:g},{a.exp_hi:g}] trajectories, {a.steps} steps", "loads": {}}
    out["launch"] = {"pair_budget": pair_budget, "max_inflight": max_inflight}
    with Context(device) as ctx, Server(ctx, hbm_budget=hbm_budget, pair_budget=pair_budget,
                                        max_inflight=max_inflight) as srv:
        # warm-up (first launches of each kernel, first use of each queue)
        run_stream(srv, serving_workload(32, seed=99, exp_lo=a.exp_lo, exp_hi=a.exp_hi, steps=a.steps),
                   np.zeros(32))
        # capacity: every job submitted at once
        i0 = srv.info()
        t = time.perf_counter()
        run_stream(srv, work, np.zeros(len(work)))
        makespan = time.perf_counter() - t
        cap = len(work) / makespan
        out["capacity"] = {"jobs_per_s": cap, "particle_steps_per_s": psteps / makespan, "makespan_s": makespan}
        i1 = srv.info()
        out["capacity"]["host_loop"] = {
            "steps": i1["steps"] - i0["steps"], "launches": i1["launches"] - i0["launches"],
            "phase_s": [b - a for a, b in zip(i0["phase_s"], i1["phase_s"])], "phase_max_s": i1["phase_max_s"]}
        # capacity the loop sustains under arrivals: a Poisson stream offered
        # at the all-at-once capacity; jobs completed over the stream's wall
        # time (when the loop falls behind, the backlog grows and this is
        # its completion rate).  Loads below are fractions of the smaller.
        arr = np.cumsum(np.random.default_rng(4321).exponential(1.0 / cap, size=len(work)))
        t = time.perf_counter()
        run_stream(srv, work, arr)
        wall = time.perf_counter() - t
        sustained = len(work) / wall
        out["sustained"] = {"offered_jobs_per_s": cap, "jobs_per_s": sustained,
                            "particle_steps_per_s": psteps / wall, "wall_s": wall}
        base = min(cap, sustained)
        # isolated solve time: each job alone in the server (every job when
        # --isolated-sample covers them all, else a sample interpolated by
        # trajectory count within the job's model type)
        rng = np.random.default_rng(7)
        n_iso = min(a.isolated_sample, len(work))
        sample = range(len(work)) if n_iso == len(work) else rng.choice(len(work), size=n_iso, replace=False)
        iso = {}
        for i in sample:
            iso[int(i)] = float(run_stream(srv, [work[i]], [0.0])[0])
        kind = lambda i: (work[i][2]["double"], work[i][2]["overdamped"])

        def isolated(i):
            if i in iso:
                return iso[i]
            same = [j for j in iso if kind(j) == kind(i)] or list(iso)
            xs = np.array([np.log2(work[j][1]) for j in same])
            ys = np.array([iso[j] for j in same])
            o = np.argsort(xs)
            return float(np.interp(np.log2(work[i][1]), xs[o], ys[o]))

        for load in a.loads:
            rate = load * base
            arr = np.cumsum(np.random.default_rng(1234).exponential(1.0 / rate, size=len(work)))
            t = time.perf_counter()
            stg = np.zeros((len(work), 3))
            lat = run_stream(srv, work, arr, stages=stg)
            wall = time.perf_counter() - t
            iso_all = np.array([isolated(i) for i in range(len(work))])
            ratio = lat / iso_all
            size = np.array([np.log2(w[1]) for w in work])
            classes = {}
            for name, lo_, hi_ in (("2^10-2^13", 0, 13), ("2^13-2^16", 13, 16), ("2^16-2^18", 16, 99)):
                m = (size >= lo_) & (size < hi_)
                if m.any():
                    classes[name] = {"jobs": int(m.sum()), "p50_over_isolated": float(np.percentile(ratio[m], 50)),
                                     "p99_over_isolated": float(np.percentile(ratio[m], 99))}
            out["loads"][f"{load:g}"] = {
                "by_trajectory_count": classes,
                "rate_jobs_per_s": rate, "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)),
                "p50_over_isolated": float(np.percentile(ratio, 50)),
                "p99_over_isolated": float(np.percentile(ratio, 99)),
                # the latency distribution against the isolated one (p99 of
                # each), beside the per-job ratio above
                "p99_latency_over_p99_isolated": float(np.percentile(lat, 99) / np.percentile(iso_all, 99)),
                "particle_steps_per_s": psteps / wall,
                "p50_stage_s": {"queued": float(np.percentile(stg[:, 0], 50)),
                                "integrating": float(np.percentile(stg[:, 1] - stg[:, 0], 50)),
                                "post_processing": float(np.percentile(stg[:, 2] - stg[:, 1], 50))},
                "p99_stage_s": {"queued": float(np.percentile(stg[:, 0], 99)),
                                "integrating": float(np.percentile(stg[:, 1] - stg[:, 0], 99)),
                                "post_processing": float(np.percentile(stg[:, 2] - stg[:, 1], 99))},
                "worst_jobs": [{"job": int(i), "ntraj": work[i][1], "latency_s": float(lat[i]),
                                "isolated_s": isolated(int(i)), "stages_s": [float(x) for x in stg[i]]}
                               for i in np.argsort(-ratio)[:4]]}
        out["isolated"] = {"jobs": len(iso), "median_s": float(np.median(list(iso.values())))}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=10000)
    ap.add_argument("--exp-lo", type=float, default=10)
    ap.add_argument("--exp-hi", type=float, default=18)
    ap.add_argument("--steps", type=int, default=24000)
    ap.add_argument("--loads", type=float, nargs="*", default=[0.5, 0.8])
    ap.add_argument("--isolated-sample", type=int, default=24)
    ap.add_argument("--pair-budget", type=int, default=1024, help="step pairs per slot per persistent launch")
    ap.add_argument("--max-inflight", type=int, default=2, help="persistent launches in flight")
    ap.add_argument("--hbm-budget", type=float, default=0, help="GB of job arenas resident at once (0: 80 %% of free)")
    a = ap.parse_args(argv)
    print(json.dumps(measure(a.jobs, a.exp_lo, a.exp_hi, a.steps, a.loads, a.isolated_sample,
                             pair_budget=a.pair_budget, max_inflight=a.max_inflight,
                             hbm_budget=int(a.hbm_budget * 1e9))))


if __name__ == "__main__":
    main()
