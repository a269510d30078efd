"""Restart files in the reference's layout, host side (no GPU).

The fixture is rank 0's .restart file of the reference's own quick_test run
(sample_input/quick_test/executed_job, written by WriteRestartFile,
src/langevinDynamicsSingleBarrier.h:1048-1136): read and written again it
must come out byte for byte, and the per-lane statistics a job restored from
it starts with must be the reference's per-trajectory results of that run.
"""
import json
import lzma
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def quick():
    return ldp.params_from_inp(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))


@pytest.fixture(scope="module")
def ref_file(tmp_path_factory):
    path = tmp_path_factory.mktemp("restart") / "ref_00000_00000.restart"
    with lzma.open(os.path.join(GOLDEN, "quick_test_rank0.restart.xz"), "rb") as f:
        path.write_bytes(f.read())
    return str(path)


def test_reference_file_round_trips_byte_for_byte(ref_file, tmp_path):
    out = tmp_path / "copy.restart"
    ldp.restart_rewrite(quick(), ref_file, str(out))
    assert out.read_bytes() == open(ref_file, "rb").read()


def test_reference_file_statistics_are_the_reference_results(ref_file):
    s = ldp.restart_inspect(quick(), ref_file)
    assert (s["lanes"], s["rank"], s["steps"], s["frames"]) == (4, 0, 3_000_000_000, 10001)
    assert not s["has_exact_resume"]
    c, m = s["counts"], s["sums"]
    assert list(c[L.C_FPT]) == [7110, 7268, 7096, 7083]
    assert np.all(c[L.C_STATE0] + c[L.C_STATE1] == 3_000_000_001)     # step 0 included
    assert np.all(c[L.C_STEPS] == 3_000_000_000)
    assert np.all(c[L.C_INIT0] + c[L.C_INIT1] == c[L.C_FPT])
    assert np.all(c[L.C_INST0] + c[L.C_INST1] == c[L.C_FPT])
    with open(os.path.join(GOLDEN, "quick_test.json")) as f:
        g = json.load(f)
    # Per-lane means = the reference's per-trajectory means of rank 0 (its
    # first four trajectories in the .dat files).
    for name, cf, sf in (("firstPassageTime", L.C_FPT, L.S_FPT), ("firstPassageTime2", L.C_FPT2, L.S_FPT2),
                         ("transitionPathTime", L.C_TPT, L.S_TPT), ("transitionPathTime2", L.C_TPT2, L.S_TPT2)):
        np.testing.assert_allclose(m[sf] / c[cf], g[name]["per_traj"][:4], rtol=1e-12, err_msg=name)
    for j, e in enumerate(g["firstPassageTimeCG2"]):
        ok = c[L.C_CG0 + j] > 0
        want = np.array(e["per_traj"][:4])
        np.testing.assert_allclose((m[L.S_CG0 + j][ok] / c[L.C_CG0 + j][ok]), want[ok], rtol=1e-12)


def test_layout_mismatch_and_damage_are_errors(ref_file, tmp_path):
    p = quick()
    p.tpt = 0                    # a run without TPT writes no TPT block
    with pytest.raises(ldp.LdpError, match="truncated|corrupted|layout"):
        ldp.restart_inspect(p, ref_file)
    data = open(ref_file, "rb").read()
    cut = tmp_path / "cut.restart"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(ldp.LdpError, match="truncated"):
        ldp.restart_inspect(quick(), str(cut))
    bad = tmp_path / "bad.restart"
    bad.write_bytes(b"\x00" * 64)
    with pytest.raises(ldp.LdpError, match="signature"):
        ldp.restart_inspect(quick(), str(bad))
    with pytest.raises(ldp.LdpError) as e:
        ldp.restart_inspect(quick(), str(tmp_path / "missing.restart"))
    assert e.value.status == 9   # LDP_ERR_RESTART
