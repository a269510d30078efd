"""The allocation-free entry point, ldp_integrate_fp64_noalloc.

It serves callers that cannot allocate device memory: the caller hands in
its own device buffers for the outputs and the library keeps its working
state in a fixed device array.  These tests call it through the C ABI with
buffers the test allocates, two calls in a row (different trajectories, same
scratch array), and check each result against the allocating path
(ldp_job_create / ldp_submit, FP64 plain) at the tolerance of the other FP64
parity tests: bit for bit.  One case spreads trajectories over more cells
than their cell-table ring holds, so that evictions happen, and compares the
two paths at the same ring size.  The file is collected last on purpose.
"""
import ctypes as C
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


def params(steps=60_000, freq=20, seed=4321):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed = steps, freq, seed
    p.waiting_time, p.write_x = 0, 0
    return p


def evicting(steps, period):
    # Short period and slow asymmetric flips: trajectories cross many cells
    # and re-enter barriers after their pending flips (lazy catch-up).
    p = params(steps=steps, freq=50, seed=77)
    p.tau, p.eq, p.eq_constant, p.periodic_length, p.x0 = 1e-2, 0, 2.0, period, -period / 2
    p.barrier_half_width[0] = period / 4
    p.barrier_heights[0][0], p.barrier_heights[0][1] = 0.5, 0.2
    return p


def opts(lanes, ranks, job_id, slots=256):
    o = L.JobOpts()
    L.lib().ldp_job_opts_default(C.byref(o))
    o.lanes, o.ranks, o.job_id, o.table_slots = lanes, ranks, job_id, slots
    return o


def allocating(p, lanes, ranks, job_id, slots=256):
    with ldp.Context(0) as ctx, ldp.Job(ctx, p, lanes=lanes, ranks=ranks, job_id=job_id, table_slots=slots) as job:
        job.run()
        return job.results()


def noalloc(p, lanes, ranks, job_id, slots=256):
    import torch
    torch.cuda.set_device(0)
    n = lanes * ranks * p.number_of_runs
    nf = p.number_of_steps // p.freq_save + 1
    counts = torch.full((L.NCOUNT, n), -1, dtype=torch.int64, device="cuda")
    sums = torch.full((L.NSUM, n), float("nan"), dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    fx = torch.zeros((nf, n), dtype=torch.float64, device="cuda")
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = L.lib().ldp_integrate_fp64_noalloc(C.byref(p), C.byref(opts(lanes, ranks, job_id, slots)),
                                            counts.data_ptr(), sums.data_ptr(), x.data_ptr(), fx.data_ptr(),
                                            stream, err, 256)
    assert st == 0, err.value.decode()
    torch.cuda.synchronize()
    return {"counts": counts.cpu().numpy(), "sums": sums.cpu().numpy(), "x_final": x.cpu().numpy(),
            "frames_x": fx.cpu().numpy()}


def assert_same(got, ref):
    np.testing.assert_array_equal(got["counts"], ref["counts"])
    np.testing.assert_array_equal(got["sums"], ref["sums"])
    np.testing.assert_array_equal(got["x_final"], ref["x_final"])
    np.testing.assert_array_equal(got["frames_x"], ref["frames_x"])


def test_noalloc_matches_allocating_path_twice_in_a_row():
    # Two calls back to back share the scratch array; each must equal the
    # allocating path for its own trajectories.
    for lanes, ranks, job_id, steps in ((64, 4, 3, 60_000), (128, 1, 9, 40_000)):
        p = params(steps=steps)
        assert_same(noalloc(p, lanes, ranks, job_id), allocating(p, lanes, ranks, job_id))


def test_noalloc_matches_allocating_path_with_ring_evictions():
    # A 16-slot ring evicts within a few thousand steps at period 0.2; the
    # default 256-slot ring evicts at period 0.02.  Both paths use the same
    # ring size, so evictions (and the catch-ups after them) agree.
    for slots, period, steps in ((16, 0.2, 100_000), (256, 0.02, 200_000)):
        p = evicting(steps, period)
        ref = allocating(p, 32, 2, 5, slots)
        assert ref["counts"][L.C_EVICT].sum() > 0
        assert_same(noalloc(p, 32, 2, 5, slots), ref)


def test_noalloc_rejects_too_many_trajectories_and_too_large_rings():
    p = params()
    err = C.create_string_buffer(256)
    o = opts(L.NOALLOC_MAX_TRAJ + 1, 1, 0)
    st = L.lib().ldp_integrate_fp64_noalloc(C.byref(p), C.byref(o), 1, 1, 1, None, None, err, 256)
    assert st == 1
    assert b"this entry point takes 1 to 4096" in err.value
    o = opts(8, 1, 0, slots=2 * L.NOALLOC_MAX_SLOTS)
    st = L.lib().ldp_integrate_fp64_noalloc(C.byref(p), C.byref(o), 1, 1, 1, None, None, err, 256)
    assert st == 7
    assert b"a power of two from 16 to 256" in err.value
