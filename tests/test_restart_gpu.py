"""Restart files on the FP64 plain path (WriteRestartFile / ReadRestartFile,
src/langevinDynamicsSingleBarrier.h:1048-1202).

* The per-event lists the files hold equal the CPU oracle's, bit for bit.
* A run chained through restart files equals the uninterrupted run bit for
  bit: counts, sums, frames, event lists, waiting ticks, MSD.
* A file without this library's exact-resume block (as the reference writes
  it) resumes: the reference's own quick_test checkpoint continues on the
  device with its statistics carried on.
"""
import lzma
import os
import struct

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L
import pyoracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu
CAP = 4096


def quick(steps, freq=200, **kw):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed = steps, freq, 1234
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def double(steps, freq=200, **kw):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "inp", "CuIDB_double__2.0_7.2_m1.0_1.00e-05.inp"),
                            ldp.MODEL_DOUBLE)
    p.number_of_steps, p.freq_save, p.random_seed = steps, freq, 1234
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def job_results(job):
    r = job.results()
    r["lags"], r["msd"] = job.msd()
    r["msd0"] = job.msd_traj()
    return r


@pytest.mark.parametrize("model", ["single", "double"])
def test_event_lists_match_the_oracle(ctx, model):
    p = quick(600_000) if model == "single" else double(600_000)
    with ldp.Job(ctx, p, lanes=8, ranks=2, event_cap=CAP, tick_cap=CAP) as job:
        job.run()
        dev = job.results(frames=False)
        info = job.info
    ref = O.run(p, 1234, lanes=8, ranks=2, tick_cap=info.tick_cap, event_cap=CAP, frames=False)
    np.testing.assert_array_equal(dev["counts"], ref["counts"])
    np.testing.assert_array_equal(dev["sums"], ref["sums"])
    np.testing.assert_array_equal(dev["events"], ref["events"])
    np.testing.assert_array_equal(dev["event_states"], ref["event_states"])
    c = dev["counts"]
    lists = [(L.E_FPT2, L.C_FPT2, L.S_FPT2)] + [(L.E_CG0 + j, L.C_CG0 + j, L.S_CG0 + j) for j in range(p.n_cg)]
    if model == "single":
        lists += [(L.E_FPT, L.C_FPT, L.S_FPT), (L.E_TPT, L.C_TPT, L.S_TPT), (L.E_TPT2, L.C_TPT2, L.S_TPT2)]
        assert c[L.C_FPT].sum() > 0
        st = dev["event_states"]
        for t in range(info.ntraj):
            k = c[L.C_FPT, t]
            assert (st[t, :k] & 1).sum() == c[L.C_INST1, t] and (st[t, :k] >> 1).sum() == c[L.C_INIT1, t]
    for e, cf, sf in lists:
        for t in range(info.ntraj):
            k = c[cf, t]
            assert np.all(dev["events"][e, t, k:] == 0.0)
            s = 0.0
            for x in dev["events"][e, t, :k]:
                s += x                       # event order, as the device sums
            assert s == dev["sums"][sf, t]


def strip_exact_resume(path):
    data = open(path, "rb").read()
    cut = data.rfind(struct.pack("<ii", 9990, 0x5844504C))
    assert cut > 0
    open(path, "wb").write(data[: cut + 4])


CASES = {
    "single_over": lambda steps, **kw: quick(steps, write_x=1, **kw),
    "single_under": lambda steps, **kw: quick(steps, overdamped=0, write_x=1, **kw),
    "double_over": lambda steps, **kw: double(steps, **kw),
    "double_under_eq": lambda steps, **kw: double(steps, overdamped=0, eq=1, **kw),
}


@pytest.mark.parametrize("case", list(CASES))
def test_chained_run_equals_the_uninterrupted_run(ctx, tmp_path, case):
    N, M = 300_000, 300_000
    mk = CASES[case]
    kw = dict(lanes=8, ranks=2, event_cap=CAP, tick_cap=CAP)
    with ldp.Job(ctx, mk(N + M), **kw) as job:
        job.run()
        a = job_results(job)
    base = str(tmp_path / "chain")
    with ldp.Job(ctx, mk(N), **kw) as job:
        job.run()
        job.save_restart(base)
    s = ldp.restart_inspect(mk(N), base + "_00001_00000.restart")
    assert s["steps"] == N and s["lanes"] == 8 and s["rank"] == 1 and s["has_exact_resume"]
    with ldp.Job(ctx, mk(M, number_of_previous_steps=N), **kw) as job:
        job.restore(base)
        assert job.info.steps_before == N
        job.run()
        b = job_results(job)
    assert a["counts"][L.C_FPT2].sum() > 0
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_resume_without_the_exact_block_continues_the_statistics(ctx, tmp_path):
    N, M = 300_000, 300_000
    kw = dict(lanes=8, ranks=1, event_cap=CAP, tick_cap=CAP)
    base = str(tmp_path / "plain")
    with ldp.Job(ctx, quick(N, write_x=1), **kw) as job:
        job.run()
        first = job.results()
        job.save_restart(base)
    strip_exact_resume(base + "_00000_00000.restart")
    assert not ldp.restart_inspect(quick(N, write_x=1), base + "_00000_00000.restart")["has_exact_resume"]
    with ldp.Job(ctx, quick(M, write_x=1, number_of_previous_steps=N), **kw) as job:
        job.restore(base)
        job.run()
        b = job.results()
    c0, c1 = first["counts"], b["counts"]
    assert np.all(c1[L.C_STEPS] == N + M)
    assert np.all(c1[L.C_STATE0] + c1[L.C_STATE1] == N + M + 1)
    for f in (L.C_FPT, L.C_FPT2, L.C_TPT, L.C_WT):
        assert np.all(c1[f] >= c0[f])
    nf0 = N // 200 + 1
    for k in ("frames_x", "frames_f", "frames_state"):
        np.testing.assert_array_equal(b[k][:nf0], first[k][:nf0], err_msg=k)
    ev = b["events"][L.E_FPT2]
    for t in range(8):
        np.testing.assert_array_equal(ev[t, :c0[L.C_FPT2, t]], first["events"][L.E_FPT2, t, :c0[L.C_FPT2, t]])


def test_restart_errors(ctx, tmp_path):
    base = str(tmp_path / "e")
    with ldp.Job(ctx, quick(300_000), lanes=8, event_cap=CAP) as job:
        job.run()
        x0 = job.results(frames=False)["x_final"][0]
        job.save_restart(base)
    # a damaged file: lane 0's position replaced by NaN
    data = open(base + "_00000_00000.restart", "rb").read()
    at = data.find(struct.pack("<d", x0))
    assert at > 0
    bad = str(tmp_path / "bad")
    open(bad + "_00000_00000.restart", "wb").write(data[:at] + struct.pack("<d", float("nan")) + data[at + 8:])
    with ldp.Job(ctx, quick(300_000, number_of_previous_steps=300_000), lanes=8, event_cap=CAP) as job:
        with pytest.raises(ldp.LdpError, match="corrupted"):
            job.restore(bad)
    # step count must match NUMBEROFPREVIOUSSTEPS
    with ldp.Job(ctx, quick(300_000, number_of_previous_steps=200_000), lanes=8, event_cap=CAP) as job:
        with pytest.raises(ldp.LdpError, match="NUMBEROFPREVIOUSSTEPS"):
            job.restore(base)
    # parameters must match the file's (ReadRestartFile's checks)
    with ldp.Job(ctx, quick(300_000, number_of_previous_steps=300_000, tau=2e-5), lanes=8, event_cap=CAP) as job:
        with pytest.raises(ldp.LdpError, match="inconsistent tau0"):
            job.restore(base)
    with ldp.Job(ctx, quick(300_000, number_of_previous_steps=300_000), lanes=4, event_cap=CAP) as job:
        with pytest.raises(ldp.LdpError, match="simd"):
            job.restore(base)
    # a continuation without its files cannot start
    with ldp.Job(ctx, quick(300_000, number_of_previous_steps=300_000), lanes=8) as job:
        with pytest.raises(ldp.LdpError, match="restore"):
            job.submit()
    # writing needs the event lists
    with ldp.Job(ctx, quick(300_000), lanes=8) as job:
        job.run()
        with pytest.raises(ldp.LdpError, match="event_cap"):
            job.save_restart(base)
    # and full ones
    with ldp.Job(ctx, quick(600_000), lanes=8, event_cap=1) as job:
        job.run()
        assert np.any(job.results(frames=False)["counts"][L.C_FLAGS] & L.FLAG_EVENT_OVERFLOW)
        with pytest.raises(ldp.LdpError, match="more events"):
            job.save_restart(base)


def test_the_reference_checkpoint_continues_on_the_device(ctx, tmp_path):
    # Rank 0 of the reference's quick_test run: 4 lanes after 3e9 steps.
    base = str(tmp_path / "ref")
    with lzma.open(os.path.join(GOLDEN, "quick_test_rank0.restart.xz"), "rb") as f:
        open(base + "_00000_00000.restart", "wb").write(f.read())
    S0, M = 3_000_000_000, 6_000_000           # 20 more frames at FREQSAVE 300000
    p = ldp.params_from_inp(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.number_of_previous_steps, p.random_seed = M, S0, 1234
    before = ldp.restart_inspect(p, base + "_00000_00000.restart")
    with ldp.Job(ctx, p, lanes=4, ranks=1, event_cap=-1) as job:
        job.restore(base)
        job.run()
        r = job.results()
        lags, msd = job.msd()
        job.save_restart(str(tmp_path / "next"))
    c0, c = before["counts"], r["counts"]
    assert np.all(c[L.C_STEPS] == S0 + M)
    assert np.all(c[L.C_STATE0] + c[L.C_STATE1] == S0 + M + 1)
    # about 14 FPT events per lane in 6e6 steps (7110 in 3e9); the device
    # lists continue the file's and the sums continue its sums
    new = c[L.C_FPT] - c0[L.C_FPT]
    assert new.sum() > 10 and np.all(new < 80)
    for t in range(4):
        s = 0.0
        for x in r["events"][L.E_FPT, t, :c0[L.C_FPT, t]]:
            s += x
        assert s == before["sums"][L.S_FPT, t]
        for x in r["events"][L.E_FPT, t, c0[L.C_FPT, t]:c[L.C_FPT, t]]:
            s += x
        assert s == r["sums"][L.S_FPT, t]
    assert r["frames_x"].shape[0] == 10021
    assert np.all(np.isfinite(msd)) and msd[-1] > msd[1] > 0
    after = ldp.restart_inspect(p, str(tmp_path / "next_00000_00000.restart"))
    assert after["steps"] == S0 + M and after["frames"] == 10021 and after["has_exact_resume"]
    np.testing.assert_array_equal(after["counts"], c[:, :4])


def test_drop_in_executable_chains_through_restart_files(tmp_path):
    # `exe -i run.inp` with WRITERESTART, then with READRESTART and
    # NUMBEROFPREVIOUSSTEPS: the per-trajectory results (.dat) equal those of
    # one uninterrupted run byte for byte.
    import re
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "langevindynamicsforpcp_b200", "bin", "langevinDynamicsSingleBarrier")
    text = open(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp")).read()

    def inp(path, **kv):
        t = text
        for k, v in kv.items():
            t, n = re.subn(rf"^{k}\s+.*$", f"{k} {v}", t, flags=re.M)
            assert n == 1, k
        open(path, "w").write(t)

    common = dict(FREQSAVE=200, WRITEX="false", RANDOMSEED=77, PRINTTIMER="false", OUTPUTBASE="out")
    N, M = 300_000, 300_000
    one, two = tmp_path / "straight", tmp_path / "chained"
    one.mkdir()
    two.mkdir()
    inp(one / "run.inp", NUMBEROFSTEPS=N + M, WRITERESTART="false", **common)
    inp(two / "a.inp", NUMBEROFSTEPS=N, WRITERESTART="true", OUTPUTRESTART="ck", **common)
    inp(two / "b.inp", NUMBEROFSTEPS=M, NUMBEROFPREVIOUSSTEPS=N, READRESTART="true", INPUTRESTART="ck",
        WRITERESTART="false", **common)
    args = ["-n", "2", "--lanes", "4"]
    subprocess.run([exe, "-i", "run.inp", *args], cwd=one, check=True, capture_output=True, timeout=600)
    subprocess.run([exe, "-i", "a.inp", *args], cwd=two, check=True, capture_output=True, timeout=600)
    assert (two / "ck_00001_00000.restart").exists()
    subprocess.run([exe, "-i", "b.inp", *args], cwd=two, check=True, capture_output=True, timeout=600)
    dats = sorted(p.name for p in one.glob("out_*.dat"))
    assert "out_firstPassageTime.dat" in dats and len(dats) >= 5
    for name in dats:
        assert (one / name).read_bytes() == (two / name).read_bytes(), name
