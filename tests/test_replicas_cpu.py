"""Replicas over ranks (the bench's N-GPU path), on CPU with two gloo ranks.

Each rank integrates its own replica (job ids offset by rank), with the CPU
oracle standing in for a GPU; nothing is exchanged but the timing, which is
the maximum over ranks.
"""
import os
import socket
import sys
import time

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INP = os.path.join(ROOT, "tests", "golden", "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp")


def quick():
    import langevindynamicsforpcp_b200 as ldp
    p = ldp.params_from_inp(INP)
    p.number_of_steps, p.freq_save = 20_000, 20
    return p


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    from langevindynamicsforpcp_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    t = time.perf_counter()
    r = O.run(quick(), 1234, lanes=4, job_id=rep.job_id_base, frames=False)
    mine = time.perf_counter() - t + 0.5 * rank      # rank 1 reports the longer time
    rep.barrier()
    slowest = rep.max_over_ranks(mine)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), x=r["x_final"], counts=r["counts"], mine=mine,
             slowest=slowest, base=rep.job_id_base)
    rep.close()


def test_two_replicas_integrate_their_own_trajectories_and_report_the_slowest(tmp_path):
    mp.start_processes(worker, args=(2, free_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    a, b = np.load(tmp_path / "rank0.npz"), np.load(tmp_path / "rank1.npz")
    assert int(a["base"]) == 0 and int(b["base"]) == 1000
    assert not np.array_equal(a["x"], b["x"])                   # different streams
    assert float(a["slowest"]) == float(b["slowest"]) == max(float(a["mine"]), float(b["mine"]))
    # a replica is the job with its job id, whichever rank runs it
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    alone = O.run(quick(), 1234, lanes=4, job_id=1000, frames=False)
    np.testing.assert_array_equal(alone["x_final"], b["x"])
    np.testing.assert_array_equal(alone["counts"], b["counts"])


def test_one_rank_needs_no_process_group(monkeypatch):
    from langevindynamicsforpcp_b200.replicas import Replicas
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setenv("RANK", "0")
    rep = Replicas("gloo")
    assert rep.dist is None and rep.job_id_base == 0 and rep.max_over_ranks(2.5) == 2.5
    rep.barrier()
    rep.close()
