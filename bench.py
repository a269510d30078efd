"""Benchmark: particle-steps/s of the FP32 batched path vs the FP64 plain
path on one B200 (and N replicas), on the "precision" workload:

  16 single-barrier jobs x 65536 trajectories = 2^20 trajectories, geometry
  of sample_input/CuIDB_single (L 5.8, w 0.65, X0 -2.9), overdamped, m 1,
  gamma 1, kT 1, dt 1e-5; per job H_low drawn from {2,3,4,5} with the high
  barrier 3.6 x H_low and the flip rate k log-uniform in [1e-2, 1e2]
  (TAU = 1/k), drawn with numpy default_rng(1234); FPT/TPT/FPTCG statistics
  on; 300000 steps per trajectory (3 time units) with frames every 100 steps (3001 frames,
  MSD on the reference's log-spaced lags).  Synthetic inputs: the reference
  ships no dataset.

One timed step = one complete pass of all 16 jobs (integration, renewal
statistics, frames, MSD, per-trajectory reductions), inputs resident on the
device.  `e2e` repeats it through the C ABI from host parameters to host
results (jobs created from host structs each step, per-trajectory counts and
sums and the MSD copied back).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

OPS_PER_STEP = 70   # lane instructions per overdamped single-barrier step (algorithmic count)
# Source-level count of the FP32 hot loop as built: a Philox block (58) per
# four steps, two Box-Muller pairs (14 each), update 3, tests 3.
OPS_PER_STEP_AS_BUILT = (58 + 2 * 14) / 4 + 3 + 3
NJOBS, NTRAJ, NSTEPS, FREQSAVE = 16, 65536, 300000, 100
FP64_STEPS = 2      # timed passes of the FP64 plain leg (one untimed before)
# Accuracy leg: the mix's most event-rich job (index 14: H_low 2, flip rate
# 4.84) with 65536 trajectories x 5e6 steps (50 time units), both precisions
# on the same noise: ~3 first passages per trajectory, ~2e5 events, so the
# FP64 mean's relative standard error is ~0.2 %.  Its device times also give
# both paths' throughput on an event-heavy workload.
ACC_JOB, ACC_NTRAJ, ACC_NSTEPS, ACC_FREQSAVE = 14, 65536, 5_000_000, 2500
# The reference's own sample run (quick_test): its .inp verbatim (overdamped
# single barrier, dt 1e-4, TAU 1e-5, all statistics, WRITEX), 4 ranks x 8
# lanes = 32 trajectories, with NUMBEROFSTEPS scaled from 3e9 to QT_STEPS
# (and FREQSAVE so that the run keeps >= 1100 frames); the FP64 plain path as
# the drop-in executable runs it.  The reference took 7.133 min on 4 Xeon
# ranks for 16 trajectories x 3e9 steps (its executed_job time.log).
QT_STEPS, QT_FULL_STEPS, QT_REF_S = 30_000_000, 3_000_000_000, 7.133333 * 60
# DRAM bytes per particle-step of the persistent kernel: 0.0870 B measured by
# ncu with frames every 100 steps, of which the frames are 8 B per frame
# (0.0801 B per step); the rest (0.0070 B: retire records, ring) is kept and
# the frame part scaled to this workload's frame interval.
DRAM_BYTES_PER_STEP = 0.0070 + 8.0 / FREQSAVE
# Lane slots the persistent kernel issues per particle-step (warp
# instructions x 32 / particle-steps), measured by ncu on one wave of the
# bench geometry (113664 trajectories x 120000 steps, frames every 100): the
# hot loop plus the special steps and the idle lanes of divergent ones.
ISSUED_LANE_SLOTS_PER_STEP = 49.6


BASE_INP = os.path.join(ROOT, "tests", "golden", "inp", "CuIDB_single__2.0_7.2_m1.0_1.00e-05.inp")


def job_draws():
    """(H_low, flip rate) of the 64 jobs the mix cycles through."""
    rng = np.random.default_rng(1234)
    return [(float(rng.choice([2.0, 3.0, 4.0, 5.0])), float(10 ** rng.uniform(-2, 2))) for _ in range(64)]


def workload_params(ldp, job0=0, njobs=NJOBS, nsteps=NSTEPS, freqsave=FREQSAVE):
    draws = job_draws()
    out = []
    for j in range(job0, job0 + njobs):
        h, k = draws[j % 64]
        p = ldp.params_from_inp(BASE_INP)
        p.overdamped, p.timestep, p.tau = 1, 1e-5, 1.0 / k
        p.barrier_heights[0][0], p.barrier_heights[0][1] = 3.6 * h, h
        p.number_of_steps, p.freq_save = nsteps, freqsave
        p.waiting_time, p.write_x, p.write_restart = 0, 0, 0
        p.random_seed = 1234
        out.append(p)
    return out


def reference_inps(nproc, trials):
    """.inp files of the mix for the reference's executable, one per
    process: process i runs job i mod 16 (same model, parameters, step count
    and frame interval as the device jobs) with `trials` trials of its SIMD
    lanes and its own RANDOMSEED."""
    draws = job_draws()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    out = []
    for i in range(nproc):
        h, k = draws[i % NJOBS]
        out.append(refrun.inp_text(BASE_INP, {
            "OUTPUTBASE": "b", "OVERDAMPED": "true", "TIMESTEP": "1e-05", "TAU": repr(1.0 / k),
            "BARRIERHEIGHTS": f"{3.6 * h!r} {h!r}", "NUMBEROFSTEPS": str(NSTEPS), "NUMBEROFPREVIOUSSTEPS": "0",
            "NUMBEROFRUNS": str(trials), "FREQSAVE": str(FREQSAVE), "WAITINGTIME": "false", "WRITEX": "false",
            "READRESTART": "false", "WRITERESTART": "false", "RANDOMSEED": str(1234 + i), "PRINTTIMER": "false"}))
    return out


# Trials per process in one round of the reference arm: 32 x 8 lanes x
# 300000 steps is about 3 s per core at the AVX-512 build's ~2.5e7
# particle-steps/s.
REF_TRIALS = 32


def reference_round(trials=REF_TRIALS):
    """One round of the reference's own code (oracle/_ref, AVX-512 build) on
    every host core: one single-rank process per core, all started together;
    particle-steps over the wall time of the slowest.  None when the build
    is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    if not refrun.available("single"):
        return None
    cores = os.cpu_count() or 1
    lanes = refrun.lanes(True)
    with refrun.Runs(refrun.exe("single"), reference_inps(cores, trials)) as r:
        if not r.ok():
            raise RuntimeError("reference executable failed: " + next(e for e, c in zip(r.errors, r.returncodes)
                                                                     if c != 0))
        wall = r.wall_s
    steps = cores * trials * lanes * NSTEPS
    return {"value": steps / wall, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
            "sample": f"{cores} single-rank processes of the reference's AVX-512 build (oracle/_ref, GCC, "
                      f"MPI and MKL-VSL stand-ins), process i on job i mod {NJOBS} of the mix: {trials} trials x "
                      f"{lanes} lanes x {NSTEPS} steps each, {FREQSAVE}-step frames, all statistics as the device "
                      f"jobs; wall time of the slowest process"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            w = [x.strip() for x in ln.split(",")]
            if len(w) < 8:
                continue
            try:
                sm.append(float(w[1]))
                mx = max(mx, float(w[2]))
            except ValueError:
                continue
            for n, v in zip(names, w[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2():
    import torch
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    buf.zero_()
    torch.cuda.synchronize()
    del buf


def run_batch(ldp, ctx, params, precision, job_id0=0):
    """Creates, submits (one batch) and completes the jobs; returns them."""
    jobs = [ldp.Job(ctx, p, lanes=NTRAJ, precision=precision, job_id=job_id0 + i) for i, p in enumerate(params)]
    ldp.submit_batch(ctx, jobs)
    for j in jobs:
        j.wait()
    return jobs


def job_summary(job):
    """MSD curve, pooled renewal-event means with their standard errors, and
    the state-1 fraction of a finished job (host copies)."""
    from langevindynamicsforpcp_b200 import _lib as L
    r = job.results(frames=False, ticks=False)
    lags, msd = job.msd()
    c, s = r["counts"], r["sums"]
    out = {"msd": msd, "lags": lags, "ntraj": c.shape[1]}
    for name, ci, si in (("fpt", L.C_FPT, L.S_FPT), ("fpt2", L.C_FPT2, L.S_FPT2), ("tpt", L.C_TPT, L.S_TPT),
                         ("tpt2", L.C_TPT2, L.S_TPT2), ("fptcg2", L.C_CG0, L.S_CG0)):
        n = float(c[ci].sum())
        if n == 0:
            out[name] = (None, 0, None)
            continue
        mean = float(s[si].sum()) / n
        # standard error of the pooled ratio estimator over trajectories
        resid = s[si] - mean * c[ci]
        out[name] = (mean, int(n), float(np.sqrt((resid ** 2).sum()) / n))
    s0, s1 = float(c[L.C_STATE0].sum()), float(c[L.C_STATE1].sum())
    out["state1_fraction"] = s1 / (s0 + s1)
    return out


def compare_summaries(a, b):
    """FP32 batched against the FP64 plain run of the same job (same
    parameters, seed, job id and noise): relative differences, with the
    relative standard error of the FP64 estimate for scale."""
    out = {}
    ok = (b["lags"] > 0) & (b["msd"] > 0)
    rel = np.abs(a["msd"][ok] - b["msd"][ok]) / b["msd"][ok]
    out["msd_max_rel_err"] = float(rel.max())
    out["msd_mean_rel_err"] = float(rel.mean())
    for k in ("fpt", "fpt2", "tpt", "tpt2", "fptcg2"):
        (ma, na, _), (mb, nb, se) = a[k], b[k]
        if ma is not None and mb is not None:
            out[k] = {"fp32_mean": ma, "fp64_mean": mb, "rel_err": abs(ma - mb) / mb,
                      "fp64_rel_se": se / mb if se else None, "events_fp32": na, "events_fp64": nb,
                      "events_per_traj": nb / b["ntraj"]}
    fa, fb = a["state1_fraction"], b["state1_fraction"]
    out["state1_fraction"] = {"fp32": fa, "fp64": fb, "rel_err": abs(fa - fb) / fb}
    return out


def quick_test_leg(ldp, ctx, job_id0, nsteps=None):
    """The reference's sample (C1) through the FP64 plain path: ns per step
    of its 32 trajectories and the projected wall time of the full 3e9-step
    run, beside the reference's recorded time (nsteps: a shorter run, for
    profiling)."""
    steps = nsteps or QT_STEPS
    p = ldp.params_from_inp(os.path.join(ROOT, "tests", "golden", "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed = steps, steps // 2000, 1234
    p.write_restart = 0
    with ldp.Job(ctx, p, lanes=8, ranks=4, job_id=job_id0) as j:
        ctx.mark(4)
        j.submit()
        j.wait()
        ctx.mark(5)
        ms = ctx.elapsed_ms(4, 5)
    ns_step = ms * 1e6 / steps
    return {"workload": "sample_input/quick_test .inp verbatim, 4 ranks x 8 lanes = 32 trajectories, "
                        f"{steps} steps (FREQSAVE {steps // 2000})",
            "ms": ms, "ns_per_step": ns_step, "particle_steps_per_s": 32 * steps / (ms * 1e-3),
            "projected_full_run_s": ns_step * 1e-9 * QT_FULL_STEPS,
            "reference_full_run_s": QT_REF_S,
            "reference_note": "16 trajectories x 3e9 steps on 4 Xeon Gold 6136 ranks (executed_job time.log)"}


# Serving leg: SERVE_JOBS jobs of the serving workload (types single/double x
# over/underdamped, 2^U[10,18] trajectories, 24000 steps, parameters from the
# precision / batching / scan ranges): capacity with every job submitted at
# once, the capacity sustained under Poisson arrivals offered at that rate,
# then Poisson streams at 50 % and 80 % of the smaller.  The full workload is
# 10^4 jobs (langevindynamicsforpcp_b200.serve); this many fit the bench.
SERVE_JOBS = 1000


def serving_leg(device):
    """p50 / p99 job latency of the serving loop (its own context)."""
    from langevindynamicsforpcp_b200 import serve
    r = serve.measure(jobs=SERVE_JOBS, loads=(0.5, 0.8), isolated_sample=24, device=device)
    out = {"workload": r["workload"], "capacity": r["capacity"], "sustained": r["sustained"],
           "isolated": r["isolated"], "loads": {}}
    for load, v in r["loads"].items():
        out["loads"][load] = {k: v[k] for k in ("rate_jobs_per_s", "p50_latency_s", "p99_latency_s",
                                                "p50_over_isolated", "p99_over_isolated",
                                                "p99_latency_over_p99_isolated", "particle_steps_per_s",
                                                "by_trajectory_count", "p50_stage_s", "p99_stage_s")}
    return out


def accuracy_leg(ldp, ctx, job_id0):
    """FP32 batched vs FP64 plain on one job of the mix, sized for a small
    FP64 standard error (outside the timed region; each run's device time is
    reported as an event-heavy throughput figure)."""
    p = workload_params(ldp, ACC_JOB, 1, nsteps=ACC_NSTEPS, freqsave=ACC_FREQSAVE)[0]
    sums, rate = {}, {}
    for prec in (ldp.PREC_FP32_BATCHED, ldp.PREC_FP64_PLAIN):
        with ldp.Job(ctx, p, lanes=ACC_NTRAJ, precision=prec, job_id=job_id0 + ACC_JOB) as j:
            j.run()
            sums[prec] = job_summary(j)
            t = j.timing()
            rate[prec] = ACC_NTRAJ * ACC_NSTEPS / ((t["integrate_ms"] + t["msd_ms"]) * 1e-3)
    out = compare_summaries(sums[ldp.PREC_FP32_BATCHED], sums[ldp.PREC_FP64_PLAIN])
    out["sample"] = (f"job {ACC_JOB} of the mix (H_low 2, flip rate 4.84), {ACC_NTRAJ} trajectories x "
                     f"{ACC_NSTEPS} steps, both precisions on the same noise")
    out["event_heavy_throughput"] = {
        "fp32": rate[ldp.PREC_FP32_BATCHED], "fp64": rate[ldp.PREC_FP64_PLAIN],
        "ratio": rate[ldp.PREC_FP32_BATCHED] / rate[ldp.PREC_FP64_PLAIN], "unit": "particle-steps/s",
        "fpt_events_per_traj": out.get("fpt", {}).get("events_per_traj")}
    return out


def cpu_baseline_worker(args):
    seed, traj_begin, ntraj, nsteps = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import langevindynamicsforpcp_b200 as ldp
    import pyoracle
    p = workload_params(ldp, 0, 1, nsteps=nsteps, freqsave=max(1, nsteps // 1000))
    t = time.perf_counter()
    pyoracle.run(p[0], seed, lanes=NTRAJ, traj_begin=traj_begin, traj_end=traj_begin + ntraj, frames=False)
    return ntraj * nsteps, time.perf_counter() - t


def cpu_baseline_port():
    """The CPU oracle (scalar C port of the reference's per-step algorithm)
    on every host core for a bounded sample of job 0: the stand-in when the
    reference's own build is absent."""
    cores = os.cpu_count() or 1
    nsteps = 200_000
    ntraj = 8          # trajectories per worker; ~6e6 steps/s per core
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(cpu_baseline_worker, [(1234, i * ntraj, ntraj, nsteps) for i in range(cores)])
    steps = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    return {"value": steps / wall, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{cores} processes x {ntraj} trajectories x {nsteps} steps of job 0 (oracle/ldp_oracle.c)"}


def cpu_baseline():
    """The reference's CPU path timed on the host cores (one round of its own
    build), else the oracle port."""
    return reference_round() or cpu_baseline_port()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="2 jobs x 16384 trajectories (for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg (profiling cases)")
    ap.add_argument("--nsteps", type=int, default=None, help="steps per trajectory (profiling cases)")
    ap.add_argument("--njobs", type=int, default=None, help="jobs per batch (profiling cases)")
    ap.add_argument("--freqsave", type=int, default=None, help="steps between frames (profiling cases)")
    ap.add_argument("--ntraj", type=int, default=None, help="trajectories per job (profiling cases)")
    ap.add_argument("--leg", default="all", choices=["all", "fp32", "fp64", "quick_test"],
                    help="profiling cases: run one leg and print its timing only (not a bench line)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return bench_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    from langevindynamicsforpcp_b200.replicas import Replicas
    rep = Replicas("nccl", timeout_s=120)

    import langevindynamicsforpcp_b200 as ldp
    from langevindynamicsforpcp_b200 import _tune

    global NJOBS, NTRAJ, NSTEPS, FREQSAVE, DRAM_BYTES_PER_STEP
    if args.small:
        NJOBS, NTRAJ = 2, 16384
    if args.nsteps:
        NSTEPS = args.nsteps
    if args.njobs:
        NJOBS = args.njobs
    if args.freqsave:
        DRAM_BYTES_PER_STEP += 8.0 / args.freqsave - 8.0 / FREQSAVE
        FREQSAVE = args.freqsave
    if args.ntraj:
        NTRAJ = args.ntraj
    ctx = ldp.Context(local)
    shape = _tune.apply_tuned(ctx, "single_over")
    params = workload_params(ldp, 0, NJOBS, nsteps=NSTEPS, freqsave=FREQSAVE)
    job_id0 = rep.job_id_base   # replicas integrate different trajectories
    psteps = NJOBS * NTRAJ * NSTEPS

    def barrier():
        rep.barrier()
        torch.cuda.synchronize()

    if args.leg == "quick_test":
        print(json.dumps({"leg": "quick_test", **quick_test_leg(ldp, ctx, job_id0, args.nsteps)}), flush=True)
        ctx.close()
        rep.close()
        return

    # ---- FP32 batched, device-resident timing ----
    for _ in range(args.warmup if args.leg in ("all", "fp32") else 0):
        for j in run_batch(ldp, ctx, params, ldp.PREC_FP32_BATCHED, job_id0):
            j.close()
    times, kernel_ms, msd_ms, launches = [], [], [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps if args.leg in ("all", "fp32") else 0):
            jobs = [ldp.Job(ctx, p, lanes=NTRAJ, precision=ldp.PREC_FP32_BATCHED, job_id=job_id0 + i)
                    for i, p in enumerate(params)]
            flush_l2()
            barrier()
            ctx.mark(0)
            ldp.submit_batch(ctx, jobs)
            for j in jobs:
                j.wait()
            ctx.mark(1)
            times.append(ctx.elapsed_ms(0, 1))
            # integration ends with the last job's launch bound; each job's
            # post-processing (event sums, MSD) starts at its own bound, beside
            # the later jobs' launches, so post_ms is what remains after the
            # integration
            kernel_ms.append(max(j.timing()["integrate_ms"] for j in jobs))
            msd_ms.append(times[-1] - kernel_ms[-1])
            launches += sum(j.timing()["launches"] for j in jobs)
            for j in jobs:
                j.close()
    clocks = clk.summary()
    if args.leg == "fp32":
        print(json.dumps({"leg": "fp32", "ms_per_step": sum(times) / len(times),
                          "kernel_ms": sum(kernel_ms) / len(kernel_ms),
                          "particle_steps_per_s": psteps / (sum(times) / len(times) * 1e-3)}), flush=True)
        ctx.close()
        rep.close()
        return
    step_ms = rep.max_over_ranks(sum(times) / len(times)) if times else float("nan")
    value = psteps * world / (step_ms * 1e-3)
    shape_used = _tune.get_fp32_shape(ctx)

    # ---- FP64 plain leg: the same 16 jobs (2^20 trajectories), one batch ----
    # (the batch runs the FP64 jobs side by side on two streams); one
    # untimed pass, then FP64_STEPS timed passes.
    t64 = []
    for it in range(1 + (FP64_STEPS if args.leg == "all" else args.steps)):
        jobs64 = [ldp.Job(ctx, p, lanes=NTRAJ, precision=ldp.PREC_FP64_PLAIN, job_id=job_id0 + i)
                  for i, p in enumerate(params)]
        flush_l2()
        barrier()
        ctx.mark(2)
        ldp.submit_batch(ctx, jobs64)
        for j in jobs64:
            j.wait()
        ctx.mark(3)
        if it >= 1:
            t64.append(ctx.elapsed_ms(2, 3))
        for j in jobs64:
            j.close()
    fp64_ms = rep.max_over_ranks(sum(t64) / len(t64))
    fp64_value = psteps / (fp64_ms * 1e-3)
    if args.leg == "fp64":
        print(json.dumps({"leg": "fp64", "ms_per_step": fp64_ms, "particle_steps_per_s": fp64_value}), flush=True)
        ctx.close()
        rep.close()
        return
    accuracy = accuracy_leg(ldp, ctx, job_id0)
    quick_test = quick_test_leg(ldp, ctx, job_id0)
    serving = serving_leg(local) if not args.no_serving else None

    # ---- end to end through the C ABI: host params in, host results out ----
    e2e_t = []
    h2d = d2h = 0
    for it in range(args.warmup + args.steps):
        barrier()
        t0 = time.perf_counter()
        jobs = [ldp.Job(ctx, p, lanes=NTRAJ, precision=ldp.PREC_FP32_BATCHED, job_id=job_id0 + i)
                for i, p in enumerate(params)]
        ldp.submit_batch(ctx, jobs)
        b_in = len(jobs) * (C_sizeof_params())
        b_out = 0
        for j in jobs:
            # each job's results as the reference reports them (per-trajectory
            # mean event times and the MSD curve), read as soon as that job is
            # done, while the later jobs still integrate
            j.wait()
            means = j.means()
            lags, msd = j.msd()
            b_out += means.nbytes + msd.nbytes
            j.close()
        torch.cuda.synchronize()
        if it >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
            h2d, d2h = b_in, b_out
    e2e_s = rep.max_over_ranks(sum(e2e_t) / len(e2e_t))
    e2e_value = psteps * world / e2e_s

    # ---- roofline of the persistent kernel (issue-bound) ----
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            peaks = json.load(f)
    props = torch.cuda.get_device_properties(local)
    sms = props.multi_processor_count
    if peaks.get("sm_max_mhz"):
        fmax = float(peaks["sm_max_mhz"])
        fsrc = "sm_max_mhz of the measured peaks file"
    else:
        fmax = float(clocks.get("sm_max_mhz") or 1965.0)
        fsrc = "clocks.max.sm sampled by nvidia-smi during the timed region (no measured peaks file)"
    peak_issue = sms * 4 * 32 * fmax * 1e6 / 1e9            # Glane-instr/s at the max clock
    kms = sum(kernel_ms) / len(kernel_ms)
    achieved = psteps * OPS_PER_STEP / (kms * 1e-3) / 1e9
    fclk = clocks.get("sm_mhz") or fmax
    roofline = {"bound": "issue", "achieved": achieved, "peak": peak_issue, "unit": "Ginstr/s",
                "frac": achieved / peak_issue, "traffic": DRAM_BYTES_PER_STEP * psteps,
                "traffic_scope": "DRAM bytes of the persistent kernel per bench step (all its launches): "
                                 f"{DRAM_BYTES_PER_STEP:.4f} B per particle-step, from an ncu capture of the kernel "
                                 "on 113664 trajectories x 120000 steps with frames every 100 steps, the frame "
                                 "part scaled to this workload's frame interval; algorithmic bytes: the frames, "
                                 "8 B per FREQSAVE steps",
                "kernel": "fp32_persistent_kernel<single, overdamped>",
                "ops_per_step": OPS_PER_STEP, "kernel_ms": kms,
                "ops_per_step_as_built": OPS_PER_STEP_AS_BUILT,
                "issued_lane_slots_per_step_ncu": ISSUED_LANE_SLOTS_PER_STEP,
                "issue_frac_ncu": psteps * ISSUED_LANE_SLOTS_PER_STEP / (kms * 1e-3) / 1e9 / peak_issue,
                "frac_as_built": psteps * OPS_PER_STEP_AS_BUILT / (kms * 1e-3) / 1e9 / peak_issue,
                "peak_basis": f"{sms} SMs x 128 lanes x {fmax:g} MHz ({fsrc})",
                "frac_at_sampled_clock": achieved / (sms * 128 * fclk * 1e6 / 1e9)}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(world), fp32_shape=shape_used, tuned=bool(shape)),
            "fp64_plain": {"value": fp64_value * world, "unit": "particle-steps/s", "ms_per_step": fp64_ms,
                           "sample": f"the same {NJOBS} jobs x {NTRAJ} trajectories x {NSTEPS} steps in one batch "
                                     f"(FP64 jobs side by side on two streams), {FP64_STEPS} timed passes"},
            "fp32_over_fp64": value / (fp64_value * world),
            "accuracy_vs_fp64": accuracy,
            "quick_test_fp64": quick_test,
            "serving": serving,
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches / max(1, args.steps)),
            "post_ms": sum(msd_ms) / len(msd_ms),
            "roofline": roofline,
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    ctx.close()
    rep.close()


# The metric both arms report (the reference arm on a bounded sample).
METRIC = "particle-steps/s, FP32 batched (vs FP64 plain), 1xB200"


def workload_config(world):
    """The workload both arms measure (the reference arm on a bounded sample
    of it, described in its cpu_baseline)."""
    return {"workload": f"precision: {NJOBS} single-barrier jobs x {NTRAJ} trajectories, dt 1e-5, "
                        f"{NSTEPS} steps, {NSTEPS // FREQSAVE + 1} frames, per-job H in {{2,3,4,5}}, "
                        "high 3.6H, flip rate logU[1e-2,1e2]",
            "trajectories": NJOBS * NTRAJ * world, "steps_per_trajectory": NSTEPS,
            "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MB write) before each step; frames 25 GB per step"}


def C_sizeof_params():
    import ctypes
    from langevindynamicsforpcp_b200 import _lib
    return ctypes.sizeof(_lib.Params)


def bench_reference(args, rank, world):
    """The reference's CPU path for this workload on the host cores: the
    reference's own build in oracle/_ref (one process per core, each round a
    bounded sample of the mix), else the CPU oracle port.  Rank 0 alone runs
    it; the product library is not loaded."""
    if rank != 0:
        return
    vals, r = [], None
    for it in range(args.warmup + args.steps):
        r = cpu_baseline()
        if it >= args.warmup:
            vals.append(r["value"])
    value = sum(vals) / len(vals)
    line = {"impl": "reference", "metric": METRIC,
            "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(world),
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
