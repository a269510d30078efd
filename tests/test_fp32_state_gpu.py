"""Continuation of FP32 batched runs (ldp_job_keep_state / save_state /
load_state): a run of N1 steps saved and continued for N2 more steps equals
the uninterrupted N1 + N2-step run bit for bit -- counts, duration sums,
final states, frames, waiting-time ticks and the MSD -- on every model type,
with WAITINGTIME and WRITEX, in one and several launches; files that do not
match the job are refused."""
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


def params(kind, steps, prev=0, **kw):
    if kind.startswith("double"):
        p = ldp.params_from_inp(os.path.join(GOLDEN, "CuIDB_double__2.0_7.2_m1.0_1.00e-05.inp"), ldp.MODEL_DOUBLE)
        p.barrier_heights[0][0], p.barrier_heights[0][1] = 1.2, 0.5
        p.barrier_heights[1][0], p.barrier_heights[1][1] = 1.5, 0.5
    else:
        p = ldp.params_from_inp(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
        p.barrier_heights[0][0], p.barrier_heights[0][1] = 1.5, 0.5
    p.overdamped = int(kind.endswith("over"))
    p.number_of_steps, p.number_of_previous_steps, p.freq_save = steps, prev, 20
    p.tau, p.random_seed, p.write_restart = 1e-3, 4321, 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def run(ctx, p, state_in=None, state_out=None, lanes=2048):
    with ldp.Job(ctx, p, lanes=lanes, precision=ldp.PREC_FP32_BATCHED, job_id=5) as j:
        if state_out:
            j.keep_state()
        if state_in:
            j.load_state(state_in)
        j.run()
        if state_out:
            j.save_state(state_out)
        r = j.results()
        r["lags"], r["msd"] = j.msd()
    return r


@pytest.mark.parametrize("kind,extra", [("single_over", {"waiting_time": 1}), ("single_under", {"write_x": 1}),
                                        ("double_over", {}), ("double_under", {})])
def test_chained_fp32_run_equals_uninterrupted(ctx, tmp_path, kind, extra):
    n1, n2 = 24_000, 36_000
    whole = run(ctx, params(kind, n1 + n2, **extra))
    path = str(tmp_path / "a.state")
    run(ctx, params(kind, n1, **extra), state_out=path)
    cont = run(ctx, params(kind, n2, prev=n1, **extra), state_in=path)
    for k in whole:
        if isinstance(whole[k], np.ndarray):
            np.testing.assert_array_equal(cont[k], whole[k], err_msg=k)
    assert cont["counts"][L.C_STEPS].min() == n1 + n2
    assert whole["counts"][L.C_FPT2].sum() > 0


def test_chain_of_three_with_small_launches(tmp_path):
    # Many short launches (trajectories crossing launch boundaries and
    # refills) on both sides of two continuations.
    from langevindynamicsforpcp_b200 import _tune
    with ldp.Context(0) as c:
        _tune.set_fp32_shape(c, block=128, blocks_per_sm=1, pair_budget=1500)
        f = {"freq_save": 10}        # 1200 frames per link (at least 1000)
        whole = run(c, params("single_over", 36_000, **f), lanes=30_000)
        a, b = str(tmp_path / "a.state"), str(tmp_path / "b.state")
        run(c, params("single_over", 12_000, **f), state_out=a, lanes=30_000)
        run(c, params("single_over", 12_000, prev=12_000, **f), state_in=a, state_out=b, lanes=30_000)
        cont = run(c, params("single_over", 12_000, prev=24_000, **f), state_in=b, lanes=30_000)
    for k in ("counts", "sums", "x_final", "v_final", "state_final", "frames_x", "msd"):
        np.testing.assert_array_equal(cont[k], whole[k], err_msg=k)


def test_mismatched_state_files_are_refused(ctx, tmp_path):
    path = str(tmp_path / "a.state")
    run(ctx, params("single_over", 24_000), state_out=path)
    for p in (params("single_over", 24_000, prev=20_000),            # wrong step count
              params("single_over", 24_000, prev=24_000, random_seed=1),   # other streams
              params("double_over", 24_000, prev=24_000)):            # other model
        with ldp.Job(ctx, p, lanes=2048, precision=ldp.PREC_FP32_BATCHED, job_id=5) as j:
            with pytest.raises(ldp.LdpError, match="state file does not match"):
                j.load_state(path)
    with ldp.Job(ctx, params("single_over", 24_000, prev=24_000), lanes=2048, precision=ldp.PREC_FP32_BATCHED,
                 job_id=5) as j:
        with pytest.raises(ldp.LdpError, match="continues a run"):
            j.run()
