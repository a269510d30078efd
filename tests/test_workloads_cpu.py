"""The synthetic workloads match the configurations they stand in for.

There is no dataset: the bench, the parameter scan and the serving stream
generate their parameter sets from seeded draws.  These tests pin the
shapes and ranges of those draws (host code only, no GPU):

* precision (bench.py): 16 single-barrier jobs x 65536 trajectories = 2^20,
  dt 1e-5, barrier height H in {2, 3, 4, 5} with the high state 3.6 H, flip
  rate k log-uniform in [1e-2, 1e2] (TAU = 1/k), 300000 steps, frames every
  100 steps;
* parameter scan: a 4 x 4 x 4 grid, H in linspace(3.5, 6.5, 4), k in
  logspace(-2, 2, 4), gamma in logspace(-1, 1, 4), overdamped and
  underdamped on a checkerboard (32 each), 2^[12, 18] trajectories per set;
* serving: jobs of all four types (single/double x over/underdamped),
  2^[10, 18] trajectories, k in [1e-2, 1e2], gamma in [0.1, 10].
"""
import os
import sys

import numpy as np

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import scan, serve

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_precision_workload():
    ps = bench.workload_params(ldp)
    assert len(ps) == bench.NJOBS == 16 and bench.NJOBS * bench.NTRAJ == 2 ** 20
    for p in ps:
        h_hi, h_lo = p.barrier_heights[0][0], p.barrier_heights[0][1]
        assert h_lo in (2.0, 3.0, 4.0, 5.0) and abs(h_hi - 3.6 * h_lo) < 1e-12
        assert 1e-2 <= 1.0 / p.tau <= 1e2
        assert p.model == ldp.MODEL_SINGLE and p.overdamped == 1
        assert (p.timestep, p.number_of_steps, p.freq_save) == (1e-5, 300000, 100)
    # the draws differ between jobs (one parameter set per job)
    assert len({(p.barrier_heights[0][1], p.tau) for p in ps}) > 8


def test_parameter_scan_grid():
    sets = scan.scan_grid()
    assert len(sets) == 64
    labels = [l for _, _, l in sets]
    np.testing.assert_allclose(sorted({l["H"] for l in labels}), np.linspace(3.5, 6.5, 4))
    np.testing.assert_allclose(sorted({l["k"] for l in labels}), np.logspace(-2, 2, 4))
    np.testing.assert_allclose(sorted({l["gamma"] for l in labels}), np.logspace(-1, 1, 4))
    assert sum(l["overdamped"] for l in labels) == 32
    for p, n, l in sets:
        assert 2 ** 12 <= n <= 2 ** 18
        assert p.overdamped == int(l["overdamped"])
        assert abs(p.tau - 1.0 / l["k"]) < 1e-9 * p.tau and abs(p.gamma - l["gamma"]) < 1e-12
        assert p.barrier_heights[0][1] == l["H"]


def test_serving_stream():
    work = serve.serving_workload(400)
    labels = [l for _, _, l in work]
    kinds = {(l["double"], l["overdamped"]) for l in labels}
    assert kinds == {(a, b) for a in (False, True) for b in (False, True)}
    for p, n, l in work:
        assert 2 ** 10 <= n <= 2 ** 18 and l["ntraj"] == n
        assert 1e-2 <= l["k"] <= 1e2 and 0.1 <= l["gamma"] <= 10
        assert p.model == (ldp.MODEL_DOUBLE if l["double"] else ldp.MODEL_SINGLE)
        assert p.overdamped == int(l["overdamped"])
    sizes = np.log2([n for _, n, _ in work])
    assert sizes.min() < 11 and sizes.max() > 17   # the whole range is drawn
