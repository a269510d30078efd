"""Parameter scans run as one batch: every parameter set is an FP32 batched
job, all jobs share the persistent launches, and the launches plus every
job's post-processing are one CUDA graph (ldp_submit_batch_graph).

The default grid is the "parameter scan in one launch" workload: the CuOPTz
single-barrier geometry (sample_input/CuOPTz: L 2.1, w 0.6, X0 -1.05, high
barrier 2.7 x low), barrier height H in linspace(3.5, 6.5, 4), flip rate k in
logspace(-2, 2, 4) (TAU = 1/k), friction gamma in logspace(-1, 1, 4): 64
sets, overdamped and underdamped on alternate grid points (a checkerboard,
32 each, so that two persistent kernels share the graph), trajectory counts
2^U[12, 18] drawn with numpy default_rng(seed).  The reference runs one .inp per process; the scan
has no counterpart there.

    python -m langevindynamicsforpcp_b200.scan [--steps N] [--exp-lo 12 --exp-hi 18]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import (Context, Job, MODEL_SINGLE, PREC_FP32_BATCHED, params_from_inp_text, submit_batch)

INP = """\
OUTPUTBASE scan
OVERDAMPED {over}
X0 -1.05
V0 1.0
GAMMA {gamma!r}
KB 1.0
TEMPERATURE 1.0
MASS 1.0
RANDOMIZEV true
PERIODICLENGTH 2.1
BARRIERHEIGHTS {high!r} {low!r}
BARRIERHALFWIDTH 0.6
TIMESTEP 1.0e-5
NUMBEROFSTEPS {steps}
NUMBEROFPREVIOUSSTEPS 0
NUMBEROFRUNS 1
FREQSAVE {freq}
FREQSTAT 1
DISTRIBUTIONV0 false
DISTRIBUTIONS0 true
INITIALSTATE 0
UNIFORMINITALSTATES false
READRESTART false
WRITERESTART false
INPUTRESTART none
OUTPUTRESTART none
PRINTTIMER false
TAU {tau!r}
RANDOMIZESTATES true
EQ true 1.0
WAITINGTIME false
FPT true
TPT true
FPTCG true 2
FPTCG true 3
FPTCG true 10
WRITEX false
NUMBEROFLOGSAMPLES 40
RANDOMSEED {seed}
"""


def scan_grid(steps: int = 24000, freq: int = 20, exp_lo: int = 12, exp_hi: int = 18, seed: int = 1234):
    """The scan's parameter sets: a list of (params, ntraj, label)."""
    rng = np.random.default_rng(seed)
    out = []
    for a, h in enumerate(np.linspace(3.5, 6.5, 4)):
        for b, k in enumerate(np.logspace(-2, 2, 4)):
            for c, g in enumerate(np.logspace(-1, 1, 4)):
                over = (a + b + c) % 2 == 0   # checkerboard: 32 sets each
                ntraj = int(2 ** rng.uniform(exp_lo, exp_hi))
                text = INP.format(over="true" if over else "false", gamma=float(g), high=float(2.7 * h),
                                  low=float(h), steps=steps, freq=freq, tau=float(1.0 / k), seed=seed)
                p = params_from_inp_text(text, MODEL_SINGLE)
                out.append((p, ntraj, {"H": float(h), "k": float(k), "gamma": float(g), "overdamped": over}))
    return out


def run_scan(ctx: Context, sets, graph: bool = True):
    """Runs every set as one batch; returns (jobs, device ms of the batch)."""
    jobs = [Job(ctx, p, lanes=n, precision=PREC_FP32_BATCHED, job_id=i) for i, (p, n, _) in enumerate(sets)]
    ctx.mark(0)
    submit_batch(ctx, jobs, graph=graph)
    for j in jobs:
        j.wait()
    ctx.mark(1)
    return jobs, ctx.elapsed_ms(0, 1)


def summarize(jobs, sets):
    rows = []
    for j, (_, n, label) in zip(jobs, sets):
        r = j.results(frames=False, ticks=False)
        from . import _lib as L
        c, s = r["counts"], r["sums"]
        nfpt2 = c[L.C_FPT2].sum()
        rows.append(dict(label, ntraj=n, fpt2_events=int(nfpt2),
                         mfpt2=float(s[L.S_FPT2].sum() / nfpt2) if nfpt2 else None))
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=24000)
    ap.add_argument("--exp-lo", type=int, default=12)
    ap.add_argument("--exp-hi", type=int, default=18)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args(argv)
    sets = scan_grid(steps=a.steps, exp_lo=a.exp_lo, exp_hi=a.exp_hi)
    psteps = sum(n for _, n, _ in sets) * a.steps
    with Context(0) as ctx:
        best = None
        for _ in range(a.repeat):
            t0 = time.perf_counter()
            jobs, ms = run_scan(ctx, sets, graph=not a.no_graph)
            wall = time.perf_counter() - t0
            rows = summarize(jobs, sets)
            for j in jobs:
                j.close()
            best = (ms, wall) if best is None or ms < best[0] else best
    print(json.dumps({"workload": "parameter scan: 64 sets (32 overdamped, 32 underdamped), CuOPTz geometry",
                      "jobs": len(sets), "trajectories": sum(n for _, n, _ in sets), "steps": a.steps,
                      "graph": not a.no_graph, "device_ms": best[0], "wall_s": best[1],
                      "particle_steps_per_s": psteps / (best[0] * 1e-3), "sets": rows[:4]}))


if __name__ == "__main__":
    main()
