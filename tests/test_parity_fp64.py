"""FP64 device path vs the CPU oracle, trajectory by trajectory.

Both evaluate the same per-step operation sequence on the same Philox
streams, so every integer (event counts, state counts, ticks, histogram
bins) must agree exactly and every FP64 value (event-time sums, positions,
frames, per-trajectory MSD) must agree bit for bit; the MSD summed over
trajectories is compared at 1e-12 relative (its device reduction order
differs from the oracle's sequential sum).
"""
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L
import pyoracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


def load(name, model):
    return ldp.params_from_inp(os.path.join(GOLDEN, name), model)


def _set(p, kw):
    for k, v in kw.items():
        if isinstance(v, tuple):
            getattr(p, k)[:] = v
        else:
            setattr(p, k, v)
    return p


def quick(steps=120_000, freq=40, **kw):
    p = load("quick_test__2.0_7.2_m1.0_1.00e-05.inp", ldp.MODEL_SINGLE)
    p.number_of_steps, p.freq_save = steps, freq
    return _set(p, kw)


def double(steps=120_000, freq=40, **kw):
    p = load("CuIDB_double__2.0_7.2_m1.0_1.00e-05.inp", ldp.MODEL_DOUBLE)
    p.number_of_steps, p.freq_save = steps, freq
    return _set(p, kw)


@pytest.fixture(scope="module")
def ctx_thread():
    # a context whose FP64 jobs run one trajectory per thread
    c = ldp.Context(0)
    c.set_fp64_latency(0)
    c.set_fp64_group(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_group():
    # a context whose FP64 jobs all run in group mode
    c = ldp.Context(0)
    c.set_fp64_latency(0)
    c.set_fp64_group(1 << 30)
    yield c
    c.close()


@pytest.fixture(scope="module", params=["latency", "thread", "group"])
def ctx(request, ctx_thread):
    # Every parity case runs three times: small jobs in latency mode (a CTA
    # per trajectory, the default up to 2048 trajectories), with one
    # trajectory per thread, and in group mode (32 trajectories per CTA with
    # producer warps); all must equal the oracle bit for bit.
    if request.param == "thread":
        return ctx_thread
    if request.param == "group":
        return request.getfixturevalue("ctx_group")
    c = request.getfixturevalue("ctx_default")
    return c


@pytest.fixture(scope="module")
def ctx_default():
    c = ldp.Context(0)
    yield c
    c.close()


def run_both(ctx, p, seed=1234, lanes=8, ranks=1, slots=256, tick_cap=-1, mode=0, step_cap=0, spl=0, job_id=0):
    p.random_seed = seed
    with ldp.Job(ctx, p, lanes=lanes, ranks=ranks, table_slots=slots, tick_cap=tick_cap, mode=mode,
                 step_cap=step_cap or 100_000_000, steps_per_launch=spl, job_id=job_id) as job:
        job.run()
        info = job.info
        dev = job.results()
        if mode == 0:
            dev["lags"], dev["msd"] = job.msd()
            dev["msd0"] = job.msd_traj()
    ref = O.run(p, seed, lanes=lanes, ranks=ranks, table_slots=slots, tick_cap=info.tick_cap, mode=mode,
                step_cap=step_cap, job_id=job_id)
    return dev, ref, info


def assert_same(dev, ref, info, p):
    np.testing.assert_array_equal(dev["counts"], ref["counts"])
    np.testing.assert_array_equal(dev["sums"], ref["sums"])
    for k in ("state0", "v0", "x_final", "v_final", "state_final"):
        np.testing.assert_array_equal(dev[k], ref[k], err_msg=k)
    if info.tick_cap > 0:
        n = np.minimum(dev["counts"][L.C_WT], info.tick_cap)
        for t in range(info.ntraj):
            np.testing.assert_array_equal(dev["ticks"][t, :n[t]], ref["ticks"][t, :n[t]])
    for k in dev:
        if k.startswith("frames_"):
            np.testing.assert_array_equal(dev[k], ref[k], err_msg=k)
    if "msd0" in dev:
        lags = O.lags(p)
        np.testing.assert_array_equal(dev["lags"], lags)
        m0 = O.msd_traj(ref["frames_x"], lags)
        np.testing.assert_array_equal(dev["msd0"], m0)
        msd = m0.sum(axis=1) / info.ntraj
        np.testing.assert_allclose(dev["msd"], msd, rtol=1e-12, atol=0)


def test_quick_test_overdamped_all_statistics(ctx):
    p = quick(steps=600_000, freq=200, write_x=1)
    dev, ref, info = run_both(ctx, p, lanes=8, ranks=2)
    assert info.ntraj == 16
    assert dev["counts"][L.C_FPT].sum() > 0 and dev["counts"][L.C_TPT2].sum() > 0
    assert dev["counts"][L.C_WT].sum() > 0
    assert_same(dev, ref, info, p)


def test_underdamped_single(ctx):
    p = quick(overdamped=0, write_x=1)
    dev, ref, info = run_both(ctx, p, lanes=8)
    assert_same(dev, ref, info, p)


def test_asymmetric_slow_flips_with_ring_evictions(ctx):
    # TAU = 1e-2 (100 steps of memory), EQ false 2.0, a 16-slot ring: the
    # lazy catch-up and the eviction policy are exercised.
    p = quick(steps=200_000, freq=50, tau=1e-2, eq=0, eq_constant=2.0, periodic_length=0.2,
              barrier_half_width=(0.05, 0.0), x0=-0.1)
    p.barrier_heights[0][:] = (0.5, 0.2)
    dev, ref, info = run_both(ctx, p, lanes=8, slots=16)
    assert dev["counts"][L.C_EVICT].sum() > 0
    assert_same(dev, ref, info, p)


def test_tau_zero_static_barriers(ctx):
    p = quick(tau=0.0)
    dev, ref, info = run_both(ctx, p, lanes=8)
    assert_same(dev, ref, info, p)


def test_double_barrier_overdamped(ctx):
    p = double(steps=600_000, freq=200)
    dev, ref, info = run_both(ctx, p, lanes=8, ranks=2)
    assert dev["counts"][L.C_FPT].sum() == 0          # cleared every step in the reference
    assert dev["counts"][L.C_FPT2].sum() > 0
    assert_same(dev, ref, info, p)


def test_double_barrier_underdamped_writex(ctx):
    p = double(overdamped=0, write_x=1)
    dev, ref, info = run_both(ctx, p, lanes=8)
    assert_same(dev, ref, info, p)


def test_uniform_initial_states_multiple_trials(ctx):
    p = quick(uniform_initial_states=1, number_of_runs=3, tau=1e-3)
    dev, ref, info = run_both(ctx, p, lanes=4, ranks=2)
    assert_same(dev, ref, info, p)


def test_nonbottom_start_and_odd_freqsave(ctx):
    # X0 off the well bottom; FREQSAVE < 10 takes the flat loop.
    p = quick(steps=21_000, freq=7, x0=-1.0)
    dev, ref, info = run_both(ctx, p, lanes=8)
    assert_same(dev, ref, info, p)


def test_steps_per_launch_does_not_change_results(ctx):
    p = quick()
    a, ref, info = run_both(ctx, p, spl=777)
    assert_same(a, ref, info, p)


def test_first_passage_mode(ctx):
    for p in (quick(), double()):
        dev, ref, info = run_both(ctx, p, lanes=32, mode=1, step_cap=200_000)
        np.testing.assert_array_equal(dev["counts"], ref["counts"])
        np.testing.assert_array_equal(dev["sums"], ref["sums"])
        np.testing.assert_array_equal(dev["x_final"], ref["x_final"])
        c = dev["counts"]
        done = c[L.C_FPT2] == 1
        cens = (c[L.C_FLAGS] & L.FLAG_CENSORED) != 0
        assert np.all(done ^ cens)


def test_job_id_and_seed_select_streams(ctx):
    p = quick(steps=30_000, freq=10)
    a, _, _ = run_both(ctx, p, seed=1, job_id=0)
    b, _, _ = run_both(ctx, p, seed=1, job_id=1)
    c, _, _ = run_both(ctx, p, seed=2, job_id=0)
    assert not np.array_equal(a["x_final"], b["x_final"])
    assert not np.array_equal(a["x_final"], c["x_final"])


def test_fp64_batch_jobs_side_by_side_equal_each_alone(ctx):
    # A batch runs its FP64 plain jobs on two streams at once; each job's
    # results equal the same job run alone, bit for bit, and its MSD too.
    ps = [quick(steps=40_000, freq=20), quick(steps=60_000, freq=20, tau=1e-3), double(steps=40_000, freq=20)]
    for p in ps:
        p.random_seed = 1234
    lanes = [600, 300, 900]
    jobs = [ldp.Job(ctx, p, lanes=n, job_id=i) for i, (p, n) in enumerate(zip(ps, lanes))]
    ldp.submit_batch(ctx, jobs)
    got = []
    for j in jobs:
        j.wait()
        r = j.results()
        r["lags"], r["msd"] = j.msd()
        got.append(r)
        j.close()
    for i, (p, n) in enumerate(zip(ps, lanes)):
        with ldp.Job(ctx, p, lanes=n, job_id=i) as job:
            job.run()
            alone = job.results()
            alone["lags"], alone["msd"] = job.msd()
        for k in ("counts", "sums", "x_final", "frames_x", "msd"):
            np.testing.assert_array_equal(got[i][k], alone[k], err_msg=f"job {i} {k}")


@pytest.mark.parametrize("precision", [ldp.PREC_FP64_PLAIN, ldp.PREC_FP32_BATCHED])
def test_rank_slice_job_equals_its_slice_of_the_run(ctx, precision):
    # A job of ranks 2..3 of a 4-rank run (first_rank 2) draws the streams
    # of those ranks' trajectories: it equals the whole run's slice bit for
    # bit, on both paths (the FP64 one also against the oracle's slice).
    p = quick(steps=60_000, freq=20, uniform_initial_states=1)
    p.number_of_runs, p.random_seed = 2, 1234
    lanes = 64
    with ldp.Job(ctx, p, lanes=lanes, ranks=4, precision=precision, job_id=3) as whole:
        whole.run()
        rw = whole.results()
    with ldp.Job(ctx, p, lanes=lanes, ranks=2, first_rank=2, precision=precision, job_id=3) as part:
        part.run()
        rp = part.results()
    sl = slice(2 * 2 * lanes, 4 * 2 * lanes)
    for k in ("counts", "sums", "x_final", "state0", "v0"):
        np.testing.assert_array_equal(rp[k], rw[k][..., sl], err_msg=k)
    np.testing.assert_array_equal(rp["frames_x"], rw["frames_x"][:, sl])
    if precision == ldp.PREC_FP64_PLAIN:
        ref = O.run(p, 1234, lanes=lanes, ranks=4, traj_begin=sl.start, traj_end=sl.stop, job_id=3,
                    tick_cap=rp["ticks"].shape[1] if "ticks" in rp else 0)
        np.testing.assert_array_equal(rp["counts"], ref["counts"])
        np.testing.assert_array_equal(rp["x_final"], ref["x_final"])


@pytest.mark.parametrize("ntraj", [8192, 9000])
def test_group_mode_of_large_jobs_equals_one_trajectory_per_thread(ctx_thread, ctx_group, ntraj):
    # Group mode takes four producer warps up to 8192 trajectories and two
    # above; both equal the thread-per-trajectory kernel bit for bit (the
    # oracle would take minutes at this size).
    p = quick(steps=24_000, freq=20, tau=1e-3)
    p.random_seed = 77
    out = []
    for c in (ctx_thread, ctx_group):
        with ldp.Job(c, p, lanes=ntraj // 8, ranks=8) as job:
            job.run()
            r = job.results()
            r["msd0"] = job.msd_traj()
            out.append(r)
    a, b = out
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert (a["counts"][L.C_STEPS] == 24_000).all()
