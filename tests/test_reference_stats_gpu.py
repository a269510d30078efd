"""Statistical parity with the reference's own code on every model type.

The reference ships golden outputs for one model only (single barrier,
overdamped).  For the double-barrier model and for underdamped runs the
checker is the reference's own code, built here (oracle/_ref: the AVX-512
build with the MPI and MKL-VSL stand-ins) and run on the host cores beside
the FP64 device path on the same .inp parameters.  Their random streams
differ (MT19937 banks against per-trajectory Philox), so the comparison is
statistical, on equally long trajectories:

* the distribution of per-trajectory mean first-passage times (FPT2 on both
  models; FPT and TPT on the single barrier; the .dat files the reference
  writes against ldp_job_traj_means): two-sample Kolmogorov-Smirnov,
  p > 0.01;
* the mean of those per-trajectory means (the MFPT the reference reports):
  inside the 99.7 % interval of the difference (z = 3: about a dozen
  comparisons share the run);
* the MSD at lags of 1, 10 and 100 frames and the fraction of steps in
  barrier state 1: inside the same interval, with the spread estimated from
  the device trajectories.
"""
import os
import sys

import numpy as np
import pytest
from scipy import stats

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "inp")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import refrun  # noqa: E402

pytestmark = pytest.mark.gpu

NSTEPS, FREQ = 600_000, 500      # 1201 frames (the lag grid keeps 1000 origins)
NDEV = 65536
Z = 3.0


def kinds():
    return ["single_over", "single_under", "double_over", "double_under"]


def setup(kind):
    """Device parameters and the reference's .inp text for one model type:
    the sample geometries with barriers low enough for a few renewal events
    per trajectory (TAU 1e-2, dt 1e-4)."""
    dbl, over = kind.startswith("double"), kind.endswith("over")
    if dbl:
        base = os.path.join(GOLDEN, "CuIDB_double__2.0_7.2_m1.0_1.00e-05.inp")
        heights = {"BARRIERHEIGHTS0": "1.2 0.5", "BARRIERHEIGHTS1": "1.5 0.5"}
    else:
        base = os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp")
        heights = {"BARRIERHEIGHTS": "1.5 0.5"}
    common = {"OUTPUTBASE": "r", "OVERDAMPED": "true" if over else "false", "TAU": "0.01",
              "NUMBEROFSTEPS": str(NSTEPS), "NUMBEROFPREVIOUSSTEPS": "0", "FREQSAVE": str(FREQ),
              "WAITINGTIME": "false", "WRITEX": "false", "READRESTART": "false", "WRITERESTART": "false",
              "PRINTTIMER": "false"}
    common.update(heights)
    p = ldp.params_from_inp(base, ldp.MODEL_DOUBLE if dbl else ldp.MODEL_SINGLE)
    if dbl:
        p.barrier_heights[0][0], p.barrier_heights[0][1] = 1.2, 0.5
        p.barrier_heights[1][0], p.barrier_heights[1][1] = 1.5, 0.5
    else:
        p.barrier_heights[0][0], p.barrier_heights[0][1] = 1.5, 0.5
    p.overdamped = int(over)
    p.tau, p.number_of_steps, p.freq_save, p.random_seed = 0.01, NSTEPS, FREQ, 20241204
    p.waiting_time, p.write_x = 0, 0
    return dbl, base, common, p


def interval_ok(name, a, sa, na, b, sb, nb):
    se = np.sqrt(sa * sa / na + sb * sb / nb)
    print(f"  {name}: reference {a:.6g} (n={na}) device {b:.6g} (n={nb}) diff {(b - a) / se:+.2f} SE")
    return abs(b - a) <= Z * se


@pytest.mark.skipif(not refrun.available("single") or not refrun.available("double"),
                    reason="reference build absent (make -C oracle ref)")
@pytest.mark.parametrize("kind", kinds())
def test_device_fp64_matches_the_reference_build(ctx, kind):
    dbl, base, common, p = setup(kind)
    nproc = min(os.cpu_count() or 1, 32)
    lanes = refrun.lanes(True)
    trials = max(1, -(-1024 // (nproc * lanes)))           # >= 1024 reference trajectories
    inps = [refrun.inp_text(base, dict(common, NUMBEROFRUNS=str(trials), RANDOMSEED=str(777 + i)))
            for i in range(nproc)]
    with refrun.Runs(refrun.exe("double" if dbl else "single"), inps, timeout=900) as ref:
        assert ref.ok(), ref.errors
        stats_names = [("firstPassageTime2", L.E_FPT2)]
        if not dbl:
            stats_names += [("firstPassageTime", L.E_FPT), ("transitionPathTime", L.E_TPT)]
        rdat = {n: ref.dat("r", n) for n, _ in stats_names}
        rmsd = np.stack([ref.msd("r", i)[:, 1] for i in range(nproc)])    # per process: mean over its lanes
        rsc = np.array([ref.state_counts("r", i) for i in range(nproc)], dtype=np.float64)
    with ldp.Job(ctx, p, lanes=NDEV) as job:
        job.run()
        means = job.means()
        lags, msd = job.msd()
        m0 = job.msd_traj()
        c = job.results(frames=False, ticks=False)["counts"]
    nref = nproc * trials * lanes
    print(f"{kind}: {nref} reference trajectories on {nproc} processes, {NDEV} device trajectories")
    ok = True
    for name, row in stats_names:
        r, d = rdat[name], means[row]
        assert r.shape == (nref,)
        ks = stats.ks_2samp(r, d)
        print(f"  {name} per-trajectory means: KS p = {ks.pvalue:.3f}")
        ok &= ks.pvalue > 0.01
        ok &= interval_ok(name + " mean", r.mean(), r.std(), len(r), d.mean(), d.std(), len(d))
    # MSD: the reference's per-process curves are means over trials x lanes
    for lag in (1, 10, 100):
        i = int(np.searchsorted(lags, lag))
        assert lags[i] == lag
        sd = m0[i].std()
        ok &= interval_ok(f"MSD lag {lag}", rmsd[:, i].mean(), sd, nref, msd[i], sd, NDEV)
    f_ref = rsc[:, 1].sum() / rsc.sum()
    fd = c[L.C_STATE1] / (c[L.C_STATE0] + c[L.C_STATE1])
    ok &= interval_ok("state-1 fraction", f_ref, fd.std(), nref, fd.mean(), fd.std(), NDEV)
    assert ok
