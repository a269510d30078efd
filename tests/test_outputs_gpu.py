"""Output files against the reference's own outputs of the same data.

The four .restart files of the reference's quick_test run hold every lane's
state after 3e9 steps.  Restored with no further steps, a job's output
files (LangevinEquationRunnerMPI::Run's post-analysis and writers,
src/langevinDynamicsSingleBarrier.h:3452-3970) must equal the files the
reference wrote at the end of that run: the .dat files byte for byte, the
.log files line for line after the parameter header (whose seed and step
lines describe this run), the MSD to the 7 digits it prints (its sums over
origins run in another order).
"""
import lzma
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
OUTS = os.path.join(GOLDEN, "quick_test_outputs")
pytestmark = pytest.mark.gpu


def body(path):
    """Lines after the PrintParameter header (which ends with the restart
    lines and a separator)."""
    lines = open(path).read().splitlines()
    for i, line in enumerate(lines):
        if line.startswith("# Output restart (base)"):
            return lines[i + 2:]
    raise AssertionError(f"no parameter header in {path}")


@pytest.fixture(scope="module")
def outputs(ctx, tmp_path_factory):
    d = tmp_path_factory.mktemp("outputs")
    base = str(d / "ref")
    for rank in range(4):
        with lzma.open(os.path.join(GOLDEN, f"quick_test_rank{rank}.restart.xz"), "rb") as f:
            open(f"{base}_{rank:05d}_00000.restart", "wb").write(f.read())
    p = ldp.params_from_inp(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.number_of_previous_steps = 0, 3_000_000_000
    out = d / "out"
    out.mkdir()
    with ldp.Job(ctx, p, lanes=4, ranks=4) as job:
        job.restore(base)
        job.run()
        job.write_outputs(str(out))
    return out


NAMES = sorted(n for n in os.listdir(OUTS) if not n.endswith("_time.log") and not n.endswith(".xz"))


@pytest.mark.parametrize("name", NAMES)
def test_output_file_equals_the_reference(outputs, name):
    ours, ref = outputs / name, os.path.join(OUTS, name)
    assert ours.exists(), name
    if name.endswith(".dat"):
        assert ours.read_bytes() == open(ref, "rb").read()
        return
    a, b = body(ours), body(ref)
    assert len(a) == len(b)
    if name.endswith("_msd.log"):
        x = np.array([[float(v) for v in line.split()] for line in a])
        y = np.array([[float(v) for v in line.split()] for line in b])
        np.testing.assert_array_equal(x[:, 0], y[:, 0])
        np.testing.assert_allclose(x[:, 1], y[:, 1], rtol=1e-6)
        return
    for la, lb in zip(a, b):
        assert la == lb


def test_trajectory_dump_equals_the_reference(outputs):
    # WRITEX dump of trial 0, lane 1, rank 2 (Run, S.h:3514-3554): frames of
    # x, v, F, barrier, PE, KE and state, then the waiting-time event ticks.
    name = "m1.0_t1.00e-05_0_trajectory_0000000000_0000000001_0000000002.log"
    with lzma.open(os.path.join(OUTS, name + ".xz"), "rt") as f:
        ref = f.read().splitlines()
    ours = (outputs / name).read_text().splitlines()
    cut = lambda lines: lines[next(i for i, l in enumerate(lines) if l.startswith("# Output restart (base)")) + 2:]
    a, b = cut(ours), cut(ref)
    assert len(a) == len(b) == 17309 - 71
    for la, lb in zip(a, b):
        assert la == lb
