"""FP32 batched persistent path.

* Deterministic: results do not depend on the launch shape (slots, blocks,
  step budget per launch) nor on which other jobs share the batch -- every
  random draw is keyed by (seed, job, trajectory, step).
* Accurate: its statistics agree with the FP64 device path (which is
  bit-identical to the CPU oracle) within the tolerances stated per test;
  both paths integrate the same Philox noise, so the comparison is tight.
"""
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


def quick(steps=120_000, freq=40, **kw):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed = steps, freq, 1234
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def double(steps=120_000, freq=40, **kw):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "CuIDB_double__2.0_7.2_m1.0_1.00e-05.inp"), ldp.MODEL_DOUBLE)
    p.number_of_steps, p.freq_save, p.random_seed = steps, freq, 1234
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def run(ctx, p, precision, **kw):
    with ldp.Job(ctx, p, precision=precision, **kw) as job:
        job.run()
        r = job.results()
        if kw.get("mode", 0) == 0:
            r["lags"], r["msd"] = job.msd()
        r["timing"] = job.timing()
    return r


def same(a, b):
    for k in ("counts", "sums", "state0", "v0", "x_final", "v_final", "state_final"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in a:
        if k.startswith("frames_") or k in ("ticks", "msd"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.fixture(scope="module")
def shapes():
    # Two contexts with different persistent launch shapes.
    a = ldp.Context(0)
    b = ldp.Context(0)
    L.lib()  # loaded
    import ctypes as C  # noqa: F401
    yield a, b
    a.close()
    b.close()


def set_shape(ctx, block, bps, budget, ring=64):
    # The launch shape lives in the context (set before first FP32 use).
    from langevindynamicsforpcp_b200 import _tune
    _tune.set_fp32_shape(ctx, block=block, blocks_per_sm=bps, pair_budget=budget, ring_slots=ring)


def test_fp32_results_independent_of_launch_shape():
    p = quick(write_x=1)
    with ldp.Context(0) as c1, ldp.Context(0) as c2:
        set_shape(c1, 256, 0, 1 << 15)
        set_shape(c2, 128, 1, 777)      # tiny budget: many launches, many refills
        a = run(c1, p, ldp.PREC_FP32_BATCHED, lanes=64, ranks=4)
        b = run(c2, p, ldp.PREC_FP32_BATCHED, lanes=64, ranks=4)
    same(a, b)
    assert a["counts"][L.C_STEPS].min() == 120_000


def test_fp32_launch_boundaries_on_the_barrier_flank():
    # Start on the barrier flank (nonzero force) and cut the run into very
    # short launches: the hot state carried across a launch boundary or a
    # refill (force, band, countdown) must give the same trajectory.
    p = quick(steps=24_000, freq=20, x0=-0.3)
    with ldp.Context(0) as c1, ldp.Context(0) as c2:
        set_shape(c1, 256, 0, 1 << 15)
        set_shape(c2, 64, 1, 37)
        a = run(c1, p, ldp.PREC_FP32_BATCHED, lanes=256)
        b = run(c2, p, ldp.PREC_FP32_BATCHED, lanes=256)
    same(a, b)


def test_fp32_double_and_underdamped_independent_of_launch_shape():
    for p in (double(), quick(overdamped=0), double(overdamped=0)):
        with ldp.Context(0) as c1, ldp.Context(0) as c2:
            set_shape(c1, 256, 0, 1 << 15)
            set_shape(c2, 64, 2, 333)
            a = run(c1, p, ldp.PREC_FP32_BATCHED, lanes=128)
            b = run(c2, p, ldp.PREC_FP32_BATCHED, lanes=128)
        same(a, b)


def test_fp32_job_results_same_alone_and_in_a_shared_batch(ctx):
    pa = quick(steps=60_000, freq=20)
    pb = quick(steps=200_000, freq=50, tau=1e-3)
    alone = run(ctx, pa, ldp.PREC_FP32_BATCHED, lanes=256, job_id=7)
    with ldp.Job(ctx, pb, precision=ldp.PREC_FP32_BATCHED, lanes=512, job_id=8) as jb, \
            ldp.Job(ctx, pa, precision=ldp.PREC_FP32_BATCHED, lanes=256, job_id=7) as ja:
        jb.submit()
        ja.submit()
        ja.wait()
        jb.wait()
        mixed = ja.results()
        mixed["lags"], mixed["msd"] = ja.msd()
    same(alone, mixed)


def test_batch_post_processing_at_each_jobs_launch_bound():
    # Jobs of different lengths and sizes in one batch, on a context with a
    # small pair budget (many launches): each job's post-processing starts
    # after its own launch bound (the list-scheduling bound of the jobs
    # published up to it), beside the later jobs' launches, and the job's
    # counter as copied just before it must be zero (checked by wait).
    # Every result equals the job run alone (which post-processes after its
    # last launch, with the full MSD instance).
    ps = [quick(steps=24000, freq=20), quick(steps=120000, freq=40), quick(steps=60000, freq=20, tau=1e-3),
          quick(steps=48000, freq=40, x0=-0.3)]
    lanes = [1000, 300, 2000, 700]
    got = []
    with ldp.Context(0) as c1:
        set_shape(c1, 256, 1, 2000)
        jobs = [ldp.Job(c1, p, lanes=n, precision=ldp.PREC_FP32_BATCHED, job_id=i)
                for i, (p, n) in enumerate(zip(ps, lanes))]
        ldp.submit_batch(c1, jobs)
        for j in jobs:
            j.wait()
            r = j.results()
            r["lags"], r["msd"] = j.msd()
            got.append(r)
            j.close()
    with ldp.Context(0) as c2:
        for i, (p, n) in enumerate(zip(ps, lanes)):
            same(got[i], run(c2, p, ldp.PREC_FP32_BATCHED, lanes=n, job_id=i))
    assert [int(r["counts"][L.C_STEPS].min()) for r in got] == [24000, 120000, 60000, 48000]


def test_fp32_first_passage_refill_independent_of_shape():
    p = quick()
    with ldp.Context(0) as c1, ldp.Context(0) as c2:
        set_shape(c1, 256, 0, 1 << 14)
        set_shape(c2, 32, 1, 5000)      # 4736 slots for 8192 trajectories: refills
        a = run(c1, p, ldp.PREC_FP32_BATCHED, lanes=8192, mode=1, step_cap=2_000_000)
        b = run(c2, p, ldp.PREC_FP32_BATCHED, lanes=8192, mode=1, step_cap=2_000_000)
    same(a, b)
    c = a["counts"]
    assert np.all((c[L.C_FPT2] == 1) ^ ((c[L.C_FLAGS] & L.FLAG_CENSORED) != 0))


def test_fp32_msd_matches_an_fp64_msd_of_its_own_frames(ctx):
    # The FP32 path's MSD kernel stages each trajectory's frames as FP32
    # offsets from its first frame, takes displacements in FP32 and sums
    # their squares in FP64.  Against an FP64 brute-force MSD of the same
    # saved frames, every per-trajectory value is within 1e-6 relative (the
    # staging and displacement roundings, ~1e-7).
    p = quick(steps=120_000, freq=40)
    with ldp.Job(ctx, p, precision=ldp.PREC_FP32_BATCHED, lanes=500) as job:
        job.run()
        fx = job.results()["frames_x"]
        lags, msd = job.msd()
        m0 = job.msd_traj()
    assert fx.shape == (3001, 500) and len(lags) > 20
    nf = fx.shape[0]
    want = np.stack([((fx[L:] - fx[:nf - L]) ** 2).mean(0) for L in lags])
    np.testing.assert_allclose(m0, want, rtol=1e-6)
    np.testing.assert_allclose(msd, want.mean(1), rtol=1e-6)


def test_fp32_first_passage_distribution_matches_fp64(ctx):
    # First bottom-to-other-bottom passage of 16384 trajectories in both
    # precisions: two-sample KS p > 0.01 and means within 3 standard errors.
    from scipy import stats
    p = quick()
    a = run(ctx, p, ldp.PREC_FP64_PLAIN, lanes=16384, mode=1, step_cap=10_000_000)
    b = run(ctx, p, ldp.PREC_FP32_BATCHED, lanes=16384, mode=1, step_cap=10_000_000)
    ok_a = a["counts"][L.C_FPT2] == 1
    ok_b = b["counts"][L.C_FPT2] == 1
    assert ok_a.mean() > 0.999 and ok_b.mean() > 0.999
    ta, tb = a["sums"][L.S_FPT2][ok_a], b["sums"][L.S_FPT2][ok_b]
    ks = stats.ks_2samp(ta, tb)
    print(f"FPT2 fp64 mean {ta.mean():.4f} fp32 mean {tb.mean():.4f} KS p={ks.pvalue:.3f}")
    assert ks.pvalue > 0.01
    se = np.sqrt(ta.var() / len(ta) + tb.var() / len(tb))
    assert abs(ta.mean() - tb.mean()) < 3 * se


@pytest.mark.parametrize("dbl", [False, True])
@pytest.mark.parametrize("eq,K,tau", [(True, 1.0, 1.0), (False, 3.0, 2.0)])
@pytest.mark.parametrize("precision", [ldp.PREC_FP64_PLAIN, ldp.PREC_FP32_BATCHED])
def test_unobserved_barriers_follow_the_two_state_chain(ctx, precision, eq, K, tau, dbl):
    # Zero barrier heights (the cells visited do not depend on the barrier
    # states), every barrier in state 0 at step 0, a cell change every few
    # hundred steps.  Each barrier flips as an independent two-state chain
    # whether observed or not, so the observed barrier is in state 1 at step
    # k with probability pi1 (1 - lam^k), lam = 1 - a - b for flip
    # probabilities a (0->1) and b (1->0): the mean time in state 1 over
    # 65536 trajectories is within 4 standard errors of the closed form.
    n = 10_000
    p = (double if dbl else quick)(steps=n, freq=5)     # 2001 frames, 89 MSD lags
    bh = p.barrier_heights
    for i in range(len(bh)):
        for j in range(len(bh[i])):
            bh[i][j] = 0.0
    p.temperature, p.tau, p.eq, p.eq_constant = 400.0, tau, int(eq), K
    p.initial_state, p.randomize_states, p.uniform_initial_states = 0, 0, 1
    p.write_x = p.waiting_time = p.tpt = 0
    p.fptcg = p.n_cg = 0
    r = run(ctx, p, precision, lanes=65536)
    c = r["counts"]
    assert np.all(r["state0"] == 0)
    assert np.all(c[L.C_EVICT] == 0)
    assert c[L.C_FPT2].mean() > 15
    lam, pi1 = (np.exp(-2.0 * p.timestep / tau), 0.5) if eq else (np.exp(-(K + 1.0) * p.timestep / tau), K / (1 + K))
    want = pi1 * ((n + 1) - (1.0 - lam ** (n + 1)) / (1.0 - lam))
    s1 = c[L.C_STATE1].astype(np.float64)
    se = s1.std() / np.sqrt(len(s1))
    print(f"state-1 steps: {s1.mean():.2f} +- {se:.2f}, chain {want:.2f}")
    assert abs(s1.mean() - want) < 4 * se
