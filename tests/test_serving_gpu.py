"""The serving loop (ldp_server_*): continuous batching of jobs of all four
model types arriving over time, admission by device-memory footprint.

Every random draw is keyed by (seed, job id, trajectory, step), so a job's
results must be the same alone and in the mix: the test runs a staggered
stream of mixed jobs through the server and compares each job, bit for bit,
with the same job run alone through ldp_submit.  A second test gives the
server a memory budget that holds about two jobs and checks that the bytes
admitted never exceed it while every job still completes, and that the
space of released jobs is whole again afterwards.
"""
import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import serve
from langevindynamicsforpcp_b200 import _lib as L

pytestmark = pytest.mark.gpu


def results(job):
    r = job.results(frames=False, ticks=False)
    _, msd = job.msd()
    return r["counts"], r["sums"], r["x_final"], msd


def test_results_same_alone_and_in_the_stream():
    work = serve.serving_workload(24, exp_lo=6, exp_hi=10, steps=24000)
    assert {(l["double"], l["overdamped"]) for _, _, l in work} == {(a, b) for a in (0, 1) for b in (0, 1)}
    got = {}
    with ldp.Context(0) as ctx:
        with serve.Server(ctx) as srv:
            arrivals = np.arange(len(work)) * 0.004   # a new job every 4 ms
            lat = serve.run_stream(srv, work, arrivals, on_done=lambda i, j: got.__setitem__(i, results(j)),
                                   timeout_s=120)
        assert np.all(np.isfinite(lat)) and np.all(lat > 0)
        for i, (p, n, _) in enumerate(work):
            with ldp.Job(ctx, p, lanes=n, precision=ldp.PREC_FP32_BATCHED, job_id=i) as j:
                j.run()
                ref = results(j)
            for a, b in zip(got[i], ref):
                np.testing.assert_array_equal(a, b)
            assert (got[i][0][L.C_STEPS] == 24000).all()


def test_admission_respects_the_memory_budget():
    work = serve.serving_workload(10, seed=99, exp_lo=9, exp_hi=11, steps=24000)
    with ldp.Context(0) as ctx:
        sizes = []
        for p, n, _ in work:
            with ldp.Job(ctx, p, lanes=n, precision=ldp.PREC_FP32_BATCHED) as j:
                sizes.append(j.info.device_bytes)
        budget = int(2.2 * max(sizes))
        with serve.Server(ctx, hbm_budget=budget) as srv:
            tickets = [srv.submit(p, n, job_id=i) for i, (p, n, _) in enumerate(work)]
            peak, done = 0, set()
            for _ in range(200000):
                srv.step()
                info = srv.info()
                peak = max(peak, info["hbm_in_use"])
                assert info["hbm_in_use"] <= budget
                ended = srv.ended()
                for t in tickets:   # the ended list names exactly the jobs that became done
                    if t not in done and srv.poll(t)[0] == L.SRV_DONE:
                        assert t in ended
                        done.add(t)
                        srv.release(t)
                assert set(ended) <= done
                if len(done) == len(tickets):
                    break
            assert len(done) == len(tickets)
            assert srv.ended() == []
            assert peak >= min(sizes)
            # Arenas live in the server's region: released jobs give their
            # space back and freed neighbours merge, so a job of about twice
            # the largest one above (the region holds 2.2x) is placed.
            assert srv.info()["hbm_in_use"] == 0
            big = max(range(len(work)), key=lambda i: sizes[i])
            p, n, _ = work[big]
            t = srv.submit(p, 2 * n, job_id=100)
            for _ in range(200000):
                srv.step()
                if srv.poll(t)[0] == L.SRV_DONE:
                    break
            assert srv.poll(t)[0] == L.SRV_DONE
            assert sizes[big] < srv.info()["hbm_in_use"] <= budget
            srv.release(t)
