"""Per-trajectory mean event times computed on the device
(ldp_job_traj_means): each equals the sum of its list divided by the count,
the reference's STATISTICS::AVERAGE, bit for bit; 0 for an empty list."""
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "inp")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [ldp.PREC_FP64_PLAIN, ldp.PREC_FP32_BATCHED])
def test_means_are_sums_over_counts(ctx, precision):
    p = ldp.params_from_inp(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))
    p.number_of_steps, p.freq_save, p.random_seed = 600_000, 200, 1234
    with ldp.Job(ctx, p, lanes=256, ranks=2, precision=precision) as job:
        job.run()
        m = job.means()
        r = job.results(frames=False, ticks=False)
    c, s = r["counts"], r["sums"]
    fields = [(L.C_FPT, L.S_FPT), (L.C_FPT2, L.S_FPT2), (L.C_TPT, L.S_TPT), (L.C_TPT2, L.S_TPT2)]
    fields += [(L.C_CG0 + j, L.S_CG0 + j) for j in range(p.n_cg)]
    assert m.shape == (len(fields), 512)
    for row, (cf, sf) in enumerate(fields):
        want = np.zeros(512)
        ok = c[cf] > 0
        want[ok] = s[sf][ok] / c[cf][ok]
        np.testing.assert_array_equal(m[row], want, err_msg=str(row))
    assert (c[L.C_FPT] > 0).any()
