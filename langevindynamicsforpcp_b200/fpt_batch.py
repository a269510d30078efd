"""First-passage batches: trajectories of very uneven length in one batch.

The "batching" workload: the double-barrier model (CuIDB double geometry:
barriers at -1.42 / -0.56 with half-widths 0.70 / 0.65, L 5.8, X0 -2.9),
H_low in {2, 3, 4, 5} (barrier 1 high = 3.6 H_low, barrier 0 high =
1.7 H_low), dt 1e-5, each trajectory run to its first bottom-to-bottom
passage (FIRST_PASSAGE mode) with a step cap; first-passage times span
orders of magnitude, so slots retire at very different times and refill from
the device work queue.  All jobs run as one graph-captured batch.  The
reference runs one .inp per process (no counterpart).

    python -m langevindynamicsforpcp_b200.fpt_batch [--jobs 16] [--ntraj 65536] [--cap 10000000]
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import (Context, Job, MODEL_DOUBLE, MODE_FIRST_PASSAGE, PREC_FP32_BATCHED, params_from_inp_text,
               submit_batch, _tune)
from . import _lib as L
from .serve import COMMON, DOUBLE


def fpt_workload(njobs: int, seed: int = 1234):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(njobs):
        h = float(rng.choice([2.0, 3.0, 4.0, 5.0]))
        k = float(10 ** rng.uniform(-2, 2))
        text = COMMON.format(over="true", gamma=1.0, steps=24000, freq=20, tau=1.0 / k, seed=seed)
        text += DOUBLE.format(mid=1.7 * h, high=3.6 * h, low=h)
        out.append((params_from_inp_text(text, MODEL_DOUBLE), {"H": h, "k": k}))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=16)
    ap.add_argument("--ntraj", type=int, default=65536)
    ap.add_argument("--cap", type=int, default=10_000_000)
    a = ap.parse_args(argv)
    work = fpt_workload(a.jobs)
    with Context(0) as ctx:
        _tune.apply_tuned(ctx, "double_over")
        jobs = [Job(ctx, p, lanes=a.ntraj, precision=PREC_FP32_BATCHED, mode=MODE_FIRST_PASSAGE,
                    step_cap=a.cap, job_id=i) for i, (p, _) in enumerate(work)]
        ctx.mark(0)
        submit_batch(ctx, jobs, graph=True)
        for j in jobs:
            j.wait()
        ctx.mark(1)
        ms = ctx.elapsed_ms(0, 1)
        steps, cens, fpt = [], 0, []
        for j in jobs:
            r = j.results(frames=False, ticks=False)
            c = r["counts"]
            steps.append(c[L.C_STEPS])
            cens += int(((c[L.C_FLAGS] & 4) != 0).sum())
            fpt.append(r["sums"][L.S_FIRST_FPT2][c[L.C_FPT2] > 0])
            j.close()
    steps = np.concatenate(steps)
    fpt = np.concatenate(fpt)
    print(json.dumps({
        "workload": f"first passage, double barrier: {a.jobs} jobs x {a.ntraj} trajectories, cap {a.cap} steps",
        "device_ms": ms, "particle_steps": int(steps.sum()),
        "particle_steps_per_s": float(steps.sum()) / (ms * 1e-3),
        "steps_per_trajectory": {"min": int(steps.min()), "median": float(np.median(steps)),
                                 "p99": float(np.percentile(steps, 99)), "max": int(steps.max())},
        "censored": cens, "mean_first_fpt2": float(fpt.mean()) if fpt.size else None}))


if __name__ == "__main__":
    main()
