"""CPU tests of the oracle: pinned against the reference's own known-answer
tests (ddecal/test/unit/tSolvers.cc with the SolverTester fixture) and
against the committed golden fixtures."""
import os

import numpy as np
import pytest

from oracle import oracle_ffi as of
from tests import helpers as H

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _check_dual(sol, inp, tol_percent):
    rel = tol_percent / 100.0
    worst = 0.0
    for cb in range(sol.shape[0]):
        for p in range(2):
            s, t = sol[cb, :, :, p], inp[:, :, p]
            a, b = np.abs(s) ** 2, np.abs(t) ** 2
            worst = max(worst, np.max(np.abs(a - b) / np.minimum(a, b)))
            a, b = (s * np.conj(s[:1])).real, (t * np.conj(t[:1])).real
            worst = max(worst, np.max(np.abs(a - b) /
                                      np.maximum(np.minimum(np.abs(a), np.abs(b)), 1e-300)))
    assert worst <= rel, worst


@pytest.mark.parametrize("ncorr", [4, 2])
def test_kat_iterative_diagonal_dd_intervals(built, ncorr):
    """tSolvers.cc iterative_diagonal_dd_intervals (MC2x2F) and
    iterative_duo_diagonal_dd_intervals (MC2x2FDiag): accuracy 1e-8, step 0.2,
    max 100 iterations, 4 threads, CheckDualResults(1e-2)."""
    prob, inp, init = of.solver_tester_problem(True, True, ncorr)
    st = of.settings(max_iterations=100, accuracy=1e-8, step_size=0.2)
    sol = init.copy()
    res, mags = of.solve(prob, sol, st, precision=32, n_threads=4)
    assert res.iterations <= 101
    _check_dual(sol, inp, 1e-2)


@pytest.mark.parametrize("ncorr", [4, 2, 1])
def test_kat_iterative_scalar_dd_intervals(built, ncorr):
    """tSolvers.cc iterative_{,duo_,uni_}scalar_dd_intervals:
    CheckScalarResults(1e-3)."""
    prob, inp, init = of.solver_tester_problem(False, True, ncorr)
    st = of.settings(max_iterations=100, accuracy=1e-8, step_size=0.2)
    sol = init.copy()
    res, _ = of.solve(prob, sol, st, precision=32, n_threads=4)
    assert res.iterations <= 101
    for cb in range(sol.shape[0]):
        s, t = sol[cb, :, :, 0], inp[:, :, 0]
        np.testing.assert_allclose(np.abs(s) ** 2, np.abs(t) ** 2, rtol=1e-5)
        a, b = s * np.conj(s[:1]), t * np.conj(t[:1])
        assert np.max(np.abs(a - b)) < 1e-3 * np.sqrt(2)


def test_kat_min_iterations(built):
    """tSolvers.cc min_iterations: SetMinIterations(10), SetAccuracy(1e8)."""
    prob, inp, init = of.solver_tester_problem(False, False, 4)
    st = of.settings(max_iterations=100, min_iterations=10, accuracy=1e8)
    res, _ = of.solve(prob, init.copy(), st, precision=32, n_threads=4)
    assert res.iterations == 10


def test_fp32_and_fp64_oracle_agree(built):
    obs = H.small_observation(n_stations=10, n_directions=3, n_channels=8,
                              n_cb=2, n_times=2, seed=31)
    prob = H.problem_from_observation(obs)
    st = of.settings(max_iterations=40, accuracy=1e-5)
    a = H.unit_solutions(prob)
    b = a.copy()
    ra, _ = of.solve(prob, a, st, precision=32, n_threads=3)
    rb, _ = of.solve(prob, b, st, precision=64, n_threads=1)
    assert ra.iterations == rb.iterations
    assert H.max_rel_diff(a, b) < 1e-4


def test_thread_count_does_not_change_result_beyond_fp32(built):
    obs = H.small_observation(n_stations=10, n_directions=2, n_channels=8,
                              n_cb=2, n_times=2, seed=33)
    prob = H.problem_from_observation(obs)
    st = of.settings(max_iterations=30, accuracy=1e-5)
    outs = []
    for nt in (1, 2, 8):
        s = H.unit_solutions(prob)
        of.solve(prob, s, st, precision=32, n_threads=nt)
        outs.append(s)
    for o in outs[1:]:
        assert H.max_rel_diff(o, outs[0]) < 1e-5


def _load_golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} missing")
    return dict(np.load(path, allow_pickle=False))


@pytest.mark.parametrize("name", ["small_diag_duo.npz", "small_scalar_full.npz",
                                  "solver_tester_pass.npz"])
def test_golden_fixtures(built, name):
    """Regression fixtures written by tests/golden/make_golden.py."""
    g = _load_golden(name)
    ncb = int(g["n_cb"])
    if "data0" in g:
        prob = dict(n_antennas=int(g["n_antennas"]),
                    n_correlations=int(g["n_correlations"]),
                    n_pol=int(g["n_pol"]),
                    n_solutions_per_direction=list(g["nspd"]),
                    data=[g[f"data{i}"] for i in range(ncb)],
                    model=[g[f"model{i}"] for i in range(ncb)],
                    antenna_pairs=[g[f"ap{i}"] for i in range(ncb)],
                    solution_map=[g[f"sm{i}"] for i in range(ncb)])
    else:  # SolverTester inputs are regenerated (deterministic mt19937)
        prob, _, _ = of.solver_tester_problem(True, True,
                                              int(g["n_correlations"]))
    if "next64" in g:
        nxt = of.perform_iteration(prob, g["sol0"], precision=64)
        np.testing.assert_allclose(nxt, g["next64"], rtol=1e-12, atol=1e-300)
    if "solved64" in g:
        st = of.settings(max_iterations=int(g["max_iterations"]),
                         accuracy=float(g["accuracy"]))
        s = g["sol0"].copy()
        r, mags = of.solve(prob, s, st, precision=64, n_threads=1)
        assert r.iterations == int(g["iterations"])
        np.testing.assert_allclose(s, g["solved64"], rtol=1e-10)
