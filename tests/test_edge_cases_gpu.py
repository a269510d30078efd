"""Edge cases of job sizes: ragged trajectory counts (not a multiple of a
warp), a single trajectory, and inputs the reference refuses.

A trajectory's random streams are keyed by (seed, job id, its index), so the
first n trajectories of a larger job are the same trajectories: a ragged job
must reproduce them bit for bit, whatever the slots and warps its lanes land
in.
"""
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


def params(steps=24_000, freq=20, **kw):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed, p.write_restart = steps, freq, 99, 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def run(ctx, p, lanes, precision):
    with ldp.Job(ctx, p, lanes=lanes, precision=precision, job_id=3) as j:
        j.run()
        return j.results()


@pytest.mark.parametrize("precision", [ldp.PREC_FP32_BATCHED, ldp.PREC_FP64_PLAIN])
@pytest.mark.parametrize("overdamped", [1, 0])
def test_ragged_and_single_trajectory_jobs_are_prefixes_of_a_larger_job(precision, overdamped):
    p = params(overdamped=overdamped)
    with ldp.Context(0) as ctx:
        full = run(ctx, p, 96, precision)
        for n in (1, 33, 95):
            part = run(ctx, p, n, precision)
            for k in ("counts", "sums"):
                np.testing.assert_array_equal(part[k], full[k][:, :n], err_msg=f"{k} n={n}")
            for k in ("x_final", "v_final", "state_final", "state0", "v0"):
                np.testing.assert_array_equal(part[k], full[k][:n], err_msg=f"{k} n={n}")
            fr = [k for k in part if k.startswith("frames_")]
            for k in fr:
                np.testing.assert_array_equal(part[k], full[k][:, :n], err_msg=f"{k} n={n}")
            assert (part["counts"][L.C_STEPS] == 24_000).all()


@pytest.mark.parametrize("precision", [ldp.PREC_FP32_BATCHED, ldp.PREC_FP64_PLAIN])
def test_inputs_the_reference_refuses_are_refused(precision):
    with ldp.Context(0) as ctx:
        # fewer than 1000 frames (NUMBEROFSTEPS / FREQSAVE + 1): the
        # reference refuses them (S.h:3221-3224), its MSD lag grid needs them
        with pytest.raises(ldp.LdpError, match="numberOfFrame"):
            ldp.Job(ctx, params(steps=0), lanes=8, precision=precision)
        with pytest.raises(ldp.LdpError, match="numberOfFrame"):
            ldp.Job(ctx, params(steps=19_960), lanes=8, precision=precision)
        for bad in ({"timestep": 0.0}, {"periodic_length": -1.0}, {"gamma": 0.0}, {"mass": 0.0}):
            with pytest.raises(ldp.LdpError):
                ldp.Job(ctx, params(**bad), lanes=8, precision=precision)
        with pytest.raises(ldp.LdpError):
            ldp.Job(ctx, params(), lanes=0, precision=precision)
        # 1000 frames, but a lag grid of fewer than 20 intervals: refused
        # too (S.h:3327-3332)
        with pytest.raises(ldp.LdpError, match="interval"):
            ldp.Job(ctx, params(steps=19_980), lanes=8, precision=precision)
        # 1201 frames are enough
        with ldp.Job(ctx, params(), lanes=8, precision=precision) as j:
            j.run()
            assert (j.results()["counts"][L.C_STEPS] == 24_000).all()
