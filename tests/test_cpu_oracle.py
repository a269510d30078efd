"""CPU tests of the oracle: Philox known answers, the FP64 elementary
functions, the MSD lag grid and the oracle's bookkeeping against the
reference's shipped quick_test outputs (tests/golden)."""
import json
import math
import os

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L
import pyoracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden():
    with open(os.path.join(GOLDEN, "quick_test.json")) as f:
        return json.load(f)


def quick_params():
    return ldp.params_from_inp(os.path.join(GOLDEN, "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp"))


def test_philox_known_answers():
    # Known-answer vectors of Philox4x32-10 published with Random123
    # (Salmon et al., SC'11).
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_fp64_elementary_functions_accuracy():
    rng = np.random.default_rng(7)
    for w in rng.integers(0, 2**32, 20000):
        u = (float(w) + 1.0) * 2.0**-32
        if u != 1.0:
            assert abs(O.log(u) - math.log(u)) <= 4e-16 * abs(math.log(u))
        t = float(w) * 2.0**-32
        s, c = O.sincos2pi(t)
        assert abs(s - math.sin(2 * math.pi * t)) < 2e-15
        assert abs(c - math.cos(2 * math.pi * t)) < 2e-15
    assert O.log(1.0) == 0.0
    for x in np.concatenate([-rng.uniform(0, 1e-7, 5000), -rng.uniform(0, 70, 5000), [-1e-300, -80.0]]):
        assert abs(O.expm1(x) - math.expm1(x)) <= 4e-16 * abs(math.expm1(x)) + 1e-300


def test_prob_threshold():
    assert O.lib().ldpo_prob_to_u64(0.0) == 0
    assert O.lib().ldpo_prob_to_u64(0.5) == 2**63
    assert O.lib().ldpo_prob_to_u64(1.0) == 2**64 - 1


def test_lag_grid_matches_golden_msd_times():
    p = quick_params()
    lags = O.lags(p)
    g = golden()
    ts = p.timestep * p.freq_save
    times = np.array([r[0] for r in g["msd"]])
    assert len(lags) == len(times) == 127
    np.testing.assert_allclose(lags * ts, times, rtol=1e-6)


def test_frame_and_step_counts():
    p = quick_params()
    assert O.lib().ldpo_nframe(p) == 10001
    assert O.lib().ldpo_effective_steps(p) == 3_000_000_000
    p.number_of_steps = 1000
    p.freq_save = 300
    assert O.lib().ldpo_effective_steps(p) == 900     # whole FREQSAVE groups only
    p.freq_save = 7
    assert O.lib().ldpo_effective_steps(p) == 1000    # flat loop below 10


def test_oracle_state_counts_include_step_zero():
    p = quick_params()
    p.number_of_steps, p.freq_save = 30_000, 30
    r = O.run(p, 1234, lanes=4)
    c = r["counts"]
    assert np.all(c[L.C_STATE0] + c[L.C_STATE1] == 30_001)   # golden stateCount sums to n*(steps+1)
    assert np.all(c[L.C_STEPS] == 30_000)
    g = golden()
    assert sum(g["stateCount"]) == 16 * (3_000_000_000 + 1)


def test_oracle_is_deterministic_and_range_splittable():
    p = quick_params()
    p.number_of_steps, p.freq_save = 20_000, 20
    a = O.run(p, 99, lanes=4, ranks=2)
    b = O.run(p, 99, lanes=4, ranks=2, traj_begin=3, traj_end=8)
    np.testing.assert_array_equal(a["counts"][:, 3:], b["counts"])
    np.testing.assert_array_equal(a["x_final"][3:], b["x_final"])


def test_oracle_event_bookkeeping_consistency():
    # Every FPT event records one initial and one instantaneous barrier state;
    # waiting ticks are bounded by the well-crossing count.
    p = quick_params()
    p.number_of_steps, p.freq_save = 400_000, 400
    r = O.run(p, 5, lanes=4, tick_cap=4096)
    c = r["counts"]
    assert np.all(c[L.C_INIT0] + c[L.C_INIT1] == c[L.C_FPT])
    assert np.all(c[L.C_INST0] + c[L.C_INST1] == c[L.C_FPT])
    assert np.all(c[L.C_TPT] == c[L.C_FPT])        # both close on the same barrier crossings
    ticks = r["ticks"]
    for t in range(4):
        k = ticks[t, :c[L.C_WT, t]]
        assert np.all(np.diff(k) > 0)


@pytest.mark.parametrize("name", sorted(os.listdir(os.path.join(GOLDEN, "inp"))))
def test_every_sample_input_parses(name):
    model = ldp.MODEL_DOUBLE if "double" in name else ldp.MODEL_SINGLE
    p = ldp.params_from_inp(os.path.join(GOLDEN, "inp", name), model)
    assert p.number_of_steps > 0 and p.timestep > 0
    assert p.model == model


def free_barrier_params(eq, K, tau, nsteps):
    """Zero barrier heights (no force: the cells a trajectory visits do not
    depend on the barrier states), every barrier in state 0 at step 0, fast
    diffusion (a cell change every few hundred steps, revisits common)."""
    p = quick_params()
    bh = p.barrier_heights
    for i in range(len(bh)):
        for j in range(len(bh[i])):
            bh[i][j] = 0.0
    p.temperature = 400.0
    p.tau, p.eq, p.eq_constant = tau, int(eq), K
    p.initial_state, p.randomize_states, p.uniform_initial_states = 0, 0, 1
    p.number_of_steps, p.freq_save = nsteps, nsteps // 10
    p.write_x = p.waiting_time = p.tpt = 0
    p.fptcg = p.n_cg = 0
    return p


def expected_state1_steps(eq, K, tau, dt, n):
    """Mean steps in state 1 over steps 0..n of a two-state chain started in
    state 0, flip probabilities a (0->1) and b (1->0) per step: the state at
    step k is 1 with probability pi1 (1 - lam^k), lam = 1 - a - b."""
    if eq:
        lam, pi1 = np.exp(-2.0 * dt / tau), 0.5
    else:
        lam, pi1 = np.exp(-(K + 1.0) * dt / tau), K / (1.0 + K)
    return pi1 * ((n + 1) - (1.0 - lam ** (n + 1)) / (1.0 - lam))


@pytest.mark.parametrize("eq,K,tau", [(True, 1.0, 1.0), (False, 3.0, 2.0)])
def test_unobserved_barriers_follow_the_two_state_chain(eq, K, tau):
    # Each barrier flips as an independent two-state chain whether or not the
    # trajectory is in its cell: the current barrier on its pending flip
    # steps, a barrier left and re-entered by its kept pending flip or the
    # closed-form catch-up.  With no force the observed barrier's state at
    # step k is 1 with probability pi1 (1 - lam^k) whatever cells were
    # visited, so the mean time in state 1 has a closed form.
    n = 10_000
    p = free_barrier_params(eq, K, tau, n)
    r = O.run(p, 4321, lanes=8192, frames=False)
    c = r["counts"]
    assert np.all(r["state0"] == 0)
    assert np.all(c[L.C_EVICT] == 0)
    assert c[L.C_FPT2].mean() > 15          # many well-to-well passages each
    s1 = c[L.C_STATE1].astype(np.float64)
    want = expected_state1_steps(eq, K, tau, p.timestep, n)
    se = s1.std() / np.sqrt(len(s1))
    print(f"state-1 steps: {s1.mean():.1f} +- {se:.1f}, chain {want:.1f}")
    assert abs(s1.mean() - want) < 4 * se
    assert se < 0.006 * want
