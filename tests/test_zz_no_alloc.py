"""The allocation-free entry point, ldp_integrate_fp64_noalloc.

It serves callers that cannot allocate device memory: the caller hands in
its own device buffers for the outputs and the library keeps its working
state in a fixed device array.  This test calls it through the C ABI with
buffers the test allocates, twice in a row (different trajectories, same
scratch array), and checks each result against the allocating path
(ldp_job_create / ldp_submit, FP64 plain) at the tolerance of the other FP64
parity tests: bit for bit.  The file is collected last on purpose.
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


def opts(lanes, ranks, job_id):
    o = L.JobOpts()
    L.lib().ldp_job_opts_default(C.byref(o))
    o.lanes, o.ranks, o.job_id = lanes, ranks, job_id
    return o


def allocating(p, lanes, ranks, job_id):
    with ldp.Context(0) as ctx, ldp.Job(ctx, p, lanes=lanes, ranks=ranks, job_id=job_id) as job:
        job.run()
        return job.results()


def noalloc(p, lanes, ranks, job_id):
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
    st = L.lib().ldp_integrate_fp64_noalloc(C.byref(p), C.byref(opts(lanes, ranks, job_id)), counts.data_ptr(),
                                            sums.data_ptr(), x.data_ptr(), fx.data_ptr(), stream, err, 256)
    assert st == 0, err.value.decode()
    torch.cuda.synchronize()
    return {"counts": counts.cpu().numpy(), "sums": sums.cpu().numpy(), "x_final": x.cpu().numpy(),
            "frames_x": fx.cpu().numpy()}


def test_noalloc_matches_allocating_path_twice_in_a_row():
    # Two calls back to back share the scratch array; each must equal the
    # allocating path for its own trajectories.
    for lanes, ranks, job_id, steps in ((64, 4, 3, 60_000), (128, 1, 9, 40_000)):
        p = params(steps=steps)
        ref = allocating(p, lanes, ranks, job_id)
        got = noalloc(p, lanes, ranks, job_id)
        np.testing.assert_array_equal(got["counts"], ref["counts"])
        np.testing.assert_array_equal(got["sums"], ref["sums"])
        np.testing.assert_array_equal(got["x_final"], ref["x_final"])
        np.testing.assert_array_equal(got["frames_x"], ref["frames_x"])


def test_noalloc_rejects_too_many_trajectories():
    p = params()
    err = C.create_string_buffer(256)
    o = opts(L.NOALLOC_MAX_TRAJ + 1, 1, 0)
    st = L.lib().ldp_integrate_fp64_noalloc(C.byref(p), C.byref(o), 1, 1, 1, None, None, err, 256)
    assert st == 1
    assert b"this entry point takes 1 to 4096" in err.value
