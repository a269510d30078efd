"""Trajectories whose position stops being finite.

The model's forces are bounded, so no valid input blows up; a negative
TEMPERATURE makes the noise amplitude NaN, which turns every position NaN at
its first step.  Such a trajectory is frozen with LDP_FLAG_NONFINITE (its
steps stop counting), on every path: FP64 equals the oracle exactly, FP32 batched sets the same flag and
counts, and the other trajectories of the batch are unaffected.  FP64 runs
in all three kernels (latency mode, group mode, one trajectory per thread).
"""
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L
import pyoracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


def params(overdamped, temperature):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.overdamped, p.temperature = 24_000, 20, overdamped, temperature
    p.random_seed, p.write_restart = 1234, 0
    return p


@pytest.mark.parametrize("overdamped", [1, 0])
@pytest.mark.parametrize("latency,group", [(4096, 0), (0, 1 << 30), (0, 0)])   # latency / group / thread
def test_fp64_nonfinite_trajectories_freeze_as_the_oracle(overdamped, latency, group):
    p = params(overdamped, -1.0)
    with ldp.Context(0) as ctx:
        ctx.set_fp64_latency(latency)
        ctx.set_fp64_group(group)
        with ldp.Job(ctx, p, lanes=8, ranks=2, table_slots=256) as job:
            job.run()
            dev = job.results()
    ref = O.run(p, 1234, lanes=8, ranks=2, table_slots=256, tick_cap=0, mode=0, step_cap=0, job_id=0)
    assert (dev["counts"][L.C_FLAGS] & L.FLAG_NONFINITE).all()
    np.testing.assert_array_equal(dev["counts"], ref["counts"])
    np.testing.assert_array_equal(dev["sums"], ref["sums"])
    for k in ("x_final", "v_final", "state_final"):
        np.testing.assert_array_equal(dev[k], ref[k], err_msg=k)


@pytest.mark.parametrize("overdamped", [1, 0])
def test_fp32_nonfinite_trajectories_are_flagged_and_do_not_touch_the_batch(overdamped):
    bad, good = params(overdamped, -1.0), params(overdamped, 1.0)
    with ldp.Context(0) as ctx:
        with ldp.Job(ctx, good, lanes=4096, precision=ldp.PREC_FP32_BATCHED, job_id=1) as alone:
            alone.run()
            ref = alone.results()
        jobs = [ldp.Job(ctx, bad, lanes=4096, precision=ldp.PREC_FP32_BATCHED, job_id=0),
                ldp.Job(ctx, good, lanes=4096, precision=ldp.PREC_FP32_BATCHED, job_id=1)]
        ldp.submit_batch(ctx, jobs)
        for j in jobs:
            j.wait()
        r_bad, r_good = jobs[0].results(), jobs[1].results()
        for j in jobs:
            j.close()
    assert (r_bad["counts"][L.C_FLAGS] & L.FLAG_NONFINITE).all()
    assert (r_bad["counts"][L.C_STEPS] == 0).all()
    assert not np.isfinite(r_bad["x_final"]).any()
    for k in ("counts", "sums", "x_final", "v_final", "state_final"):
        np.testing.assert_array_equal(r_good[k], ref[k], err_msg=k)
