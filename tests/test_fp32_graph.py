"""A batch run as one CUDA graph (ldp_submit_batch_graph) against the same
batch submitted launch by launch (ldp_submit_batch).

The scan grid (64 parameter sets, overdamped and underdamped on alternate
grid points, uneven trajectory counts) is run both ways at small trajectory
counts.  Every random draw is keyed by (seed, job, trajectory, step), so the
two runs must agree bit for bit: per-trajectory counts and duration sums,
final positions and the MSD.
"""
import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import scan

pytestmark = pytest.mark.gpu


def run(ctx, sets, graph):
    jobs, ms = scan.run_scan(ctx, sets, graph=graph)
    out = []
    for j in jobs:
        r = j.results(frames=False, ticks=False)
        lags, msd = j.msd()
        out.append((r["counts"], r["sums"], r["x_final"], msd, j.info.nframe))
        j.close()
    return out


def test_graph_batch_equals_launch_by_launch_batch():
    sets = scan.scan_grid(steps=24000, exp_lo=7, exp_hi=10)
    with ldp.Context(0) as ctx:
        a = run(ctx, sets, graph=True)
        b = run(ctx, sets, graph=False)
        c = run(ctx, sets, graph=True)   # a second graph on the same queues
    for (ca, sa, xa, ma, _), (cb, sb, xb, mb, _), (cc, sc, xc, mc, _) in zip(a, b, c):
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(sa, sb)
        np.testing.assert_array_equal(xa, xb)
        np.testing.assert_array_equal(ma, mb)
        np.testing.assert_array_equal(ca, cc)
        np.testing.assert_array_equal(ma, mc)
    # the runs did work: every trajectory ran its steps
    from langevindynamicsforpcp_b200 import _lib as L
    assert all((ca[L.C_STEPS] == 24000).all() for ca, *_ in a)


def test_graph_batch_rejects_fp64_jobs():
    p = scan.scan_grid(steps=24000, exp_lo=4, exp_hi=5)[0][0]
    with ldp.Context(0) as ctx:
        j = ldp.Job(ctx, p, lanes=8, precision=ldp.PREC_FP64_PLAIN)
        with pytest.raises(ldp.LdpError):
            ldp.submit_batch(ctx, [j], graph=True)
        j.close()
