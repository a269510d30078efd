"""Statistical parity with the reference's own quick_test run.

The reference's random numbers come from closed MKL streams, so parity with
its shipped outputs (sample_input/quick_test/executed_job, fixtures in
tests/golden) is statistical.  These tests run the FP64 device path -- which
is bit-identical to the CPU oracle -- on the quick_test model and compare:

* first-passage distributions (FPT bottom->top, TPT, FPT2 bottom->other
  bottom) with the per-event lists decoded from the reference's .restart
  files: two-sample Kolmogorov-Smirnov, p > 0.01.  Each of our trajectories
  contributes its first event (an unbiased first-passage sample: every
  trajectory starts exactly at a well bottom, like every renewal);
* the mean event times with the reference's mean of per-trajectory means:
  inside the 99% confidence interval of the difference (the 1% level of the
  KS tests; the reference's own two estimates, this mean of 16 per-trajectory
  means and the mean of its pooled event lists, differ by 2.0 (FPT) and 2.7
  (TPT) of the former's standard errors, so a 95% interval around it is
  tighter than the reference's own spread);
* the MSD at the reference's first lags: inside the 95% interval.
"""
import json
import os

import numpy as np
import pytest
from scipy import stats

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu
NTRAJ = 32768


def golden():
    with open(os.path.join(GOLDEN, "quick_test.json")) as f:
        return json.load(f)


def events():
    return np.load(os.path.join(GOLDEN, "quick_test_events.npz"))


@pytest.fixture(scope="module")
def fixed_run(ctx):
    # 32768 trajectories x 4e6 steps (400 time units, ~10 FPT events each),
    # frames every 2000 steps.
    p = ldp.params_from_inp(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed = 4_000_000, 2000, 20241203
    p.write_x, p.waiting_time = 0, 0
    with ldp.Job(ctx, p, lanes=NTRAJ) as job:
        job.run()
        r = job.results()
    r["params"] = p
    # FPT2 (mean ~78 time units) would be censored at 400: its first passages
    # come from first-passage mode, capped at 2e7 steps (2000 time units).
    with ldp.Job(ctx, p, lanes=NTRAJ, mode=ldp.MODE_FIRST_PASSAGE, step_cap=20_000_000) as job:
        job.run()
        fp = job.results()
    r["counts"][L.C_FPT2] = fp["counts"][L.C_FPT2]
    r["sums"][L.S_FIRST_FPT2] = fp["sums"][L.S_FIRST_FPT2]
    return r


def first_events(r, cfield, sfield):
    ok = r["counts"][cfield] > 0
    return r["sums"][sfield][ok], ok.mean()


@pytest.mark.parametrize("name,cf,sf", [("fpt", L.C_FPT, L.S_FIRST_FPT), ("tpt", L.C_TPT, L.S_FIRST_TPT),
                                        ("fpt2", L.C_FPT2, L.S_FIRST_FPT2)])
def test_first_passage_distribution_matches_reference(fixed_run, name, cf, sf):
    ours, frac = first_events(fixed_run, cf, sf)
    assert frac > 0.999          # censoring of the first event is negligible
    ref = events()[name].astype(np.float64) * 1e-4     # steps -> time (dt = 1e-4)
    ks = stats.ks_2samp(ours, ref)
    print(f"{name}: ours n={len(ours)} mean={ours.mean():.4f}  reference n={len(ref)} mean={ref.mean():.4f}  "
          f"KS D={ks.statistic:.4f} p={ks.pvalue:.3f}")
    assert ks.pvalue > 0.01


@pytest.mark.parametrize("name,cf,sf", [("firstPassageTime", L.C_FPT, L.S_FIRST_FPT),
                                        ("transitionPathTime", L.C_TPT, L.S_FIRST_TPT),
                                        ("firstPassageTime2", L.C_FPT2, L.S_FIRST_FPT2)])
def test_mean_event_times_inside_reference_ci(fixed_run, name, cf, sf):
    g = golden()[name]
    ours, _ = first_events(fixed_run, cf, sf)
    se_ref = g["sd"] / np.sqrt(g["count"])          # sd of 16 per-trajectory means
    se_ours = ours.std() / np.sqrt(len(ours))
    diff = ours.mean() - g["average"]
    print(f"{name}: ours {ours.mean():.4f} +- {se_ours:.4f}, reference {g['average']:.4f} +- {se_ref:.4f}")
    assert abs(diff) < 2.576 * np.hypot(se_ref, se_ours)


def test_msd_inside_reference_ci(fixed_run):
    # Reference: 16 trajectories, frames every 30 time units over 3e5; ours:
    # 32768 trajectories, frames every 0.2 over 400.  The time-averaged MSD
    # of each trajectory is evaluated at the reference's first lag times
    # (30, 60, 90, 120) from our frames, as MeanSquareDisplacementBruteForce
    # does.  At lag t the variance of one trajectory's time-averaged MSD
    # scales as 1 / (window); the reference's interval is our
    # per-trajectory spread rescaled to its window and trajectory count.
    g = golden()
    r = fixed_run
    ts = r["params"].timestep * r["params"].freq_save
    T_ours = r["params"].number_of_steps * r["params"].timestep
    T_ref = 3e9 * 1e-4
    fx = r["frames_x"]
    for tg, mg in g["msd"][1:5]:
        k = int(round(tg / ts))
        d = fx[k:] - fx[:-k]
        per = (d * d).mean(axis=0)
        ours = per.mean()
        se_ours = per.std() / np.sqrt(len(per))
        se_ref = per.std() * np.sqrt(T_ours / T_ref) / np.sqrt(16)
        print(f"MSD({tg:g}): ours {ours:.4f} +- {se_ours:.4f}  reference {mg:.4f} +- {se_ref:.4f}")
        assert abs(ours - mg) < 1.96 * np.hypot(se_ours, se_ref)


def test_state_fraction_matches_reference(fixed_run):
    g = golden()["stateCount"]
    c = fixed_run["counts"]
    f_ours = c[L.C_STATE1].sum() / (c[L.C_STATE0].sum() + c[L.C_STATE1].sum())
    f_ref = g[1] / (g[0] + g[1])
    # Flips are ~white at TAU = 1e-5 << dt: binomial spread over all steps.
    n = c[L.C_STATE0].sum() + c[L.C_STATE1].sum()
    assert abs(f_ours - f_ref) < 5 * np.sqrt(0.25 / n) + 5 * np.sqrt(0.25 / sum(g))
