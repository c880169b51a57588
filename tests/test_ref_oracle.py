"""CPU tests pinning the restated oracle (oracle/ddecal_oracle.cc) to the
reference itself: DP3's own IterativeDiagonalSolver / IterativeScalarSolver /
SolverBase / SolveData compiled here from the reference sources
(oracle/_ref/libddecal_ref.so, oracle/ref_ffi.py).

Both run with at most one thread per channel block, so each has a fixed FP32
summation order (SolverBase::NSubThreads() = 1, SolverBase.cc:416-420); they
differ only in that order (the restatement folds the add-back into one pass
per visibility, the reference copies the residual per direction,
IterativeDiagonalSolver.cc:100-127). Bar: identical iteration counts and a
maximum relative difference <= 1e-6 after phase referencing to antenna 0.
"""
import types

import numpy as np
import pytest

from dp3_b200 import synth
from oracle import oracle_ffi as of
from oracle import ref_ffi as rf
from tests import helpers as H

pytestmark = pytest.mark.skipif(not rf.available(), reason="reference-code oracle not built")

RTOL_PIN = 1e-6

SOLVER_KINDS = [(True, 2), (True, 4), (False, 1), (False, 2), (False, 4)]


def regular_tester_inputs(prob):
    """The SolverTester problem (regular SolveData layout: time -> baseline
    -> channel, 4 even channel blocks) as the reference's regular
    constructor inputs: a config and the baseline antenna lists."""
    ap = prob["antenna_pairs"][0].reshape(of.TESTER_N_TIMES, of.TESTER_N_BASELINES, -1, 2)
    assert (ap == ap[:1, :, :1]).all()
    cfg = types.SimpleNamespace(n_stations=of.TESTER_N_ANTENNAS, n_times=of.TESTER_N_TIMES,
                                n_baselines=of.TESTER_N_BASELINES,
                                cb_channels=[ap.shape[2]] * len(prob["data"]),
                                nspd=prob["n_solutions_per_direction"])
    return cfg, ap[0, :, 0, 0], ap[0, :, 0, 1]


def _ref_solve_problem(cfg, a1, a2, prob, sol, n_threads=1, **st):
    return rf.solve(cfg, a1, a2, prob["data"], prob["model"], prob["n_correlations"],
                    prob["n_pol"], sol, rf.settings(**st), n_threads=n_threads)


@pytest.mark.parametrize("diagonal,ncorr", SOLVER_KINDS)
@pytest.mark.parametrize("dd", [False, True])
def test_solver_tester_fixture_matches_reference(built, diagonal, ncorr, dd):
    """tSolvers.cc's SolverTester problem (restated fixture), accuracy 1e-8,
    step 0.2, max 100 iterations, for every solver and data kind."""
    prob, inp, init = of.solver_tester_problem(diagonal, dd, ncorr)
    cfg, a1, a2 = regular_tester_inputs(prob)
    st = dict(max_iterations=100, accuracy=1e-8, step_size=0.2)
    # one thread per channel block: blocks in parallel, each block's sums in
    # a fixed order (NSubThreads() = 1 in both)
    a = init.copy()
    r, _ = of.solve(prob, a, of.settings(**st), precision=32, n_threads=4)
    b = init.copy()
    rr = _ref_solve_problem(cfg, a1, a2, prob, b, n_threads=4, **st)
    assert r.iterations == rr.iterations
    assert H.max_rel_diff(a, b) < RTOL_PIN


def test_benchmark_c0_matches_reference(built):
    """Benchmark config c0 at full size: unit start, tolerance 1e-5, max 50."""
    cfg = synth.benchmark_configs()[0]
    obs = synth.observe(cfg)
    prob = H.problem_from_observation(obs)
    st = dict(max_iterations=cfg.max_iterations, accuracy=cfg.tolerance,
              step_size=cfg.step_size)
    a = H.unit_solutions(prob)
    r, _ = of.solve(prob, a, of.settings(**st), precision=32, n_threads=1)
    b = H.unit_solutions(prob)
    rr = _ref_solve_problem(cfg, obs.antenna1, obs.antenna2, prob, b, **st)
    assert r.iterations == rr.iterations
    assert H.max_rel_diff(a, b) < RTOL_PIN


@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (1, 1), (2, 1), (4, 1)])
@pytest.mark.parametrize("case", ["converging", "phase_only", "min_iterations",
                                  "dd", "dd_beyond_times", "flagged_antenna"])
def test_small_cases_match_reference(built, ncorr, npol, case):
    nspd = {"dd": [2, 1, 2], "dd_beyond_times": [2, 1, 6]}.get(case)
    obs = H.small_observation(n_stations=10, n_directions=3, n_channels=8, n_cb=2,
                              n_times=4, nspd=nspd, seed=21)
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.02)
    if case == "flagged_antenna":  # antenna 4 without data: NaN solutions, repaired
        for cb in range(len(prob["data"])):
            ap = prob["antenna_pairs"][cb]
            bad = (ap[:, 0] == 4) | (ap[:, 1] == 4)
            prob["data"][cb][bad] = 0
            prob["model"][cb][:, bad] = 0
    st = dict(max_iterations=60, accuracy=1e-5, step_size=0.2,
              phase_only=case == "phase_only",
              min_iterations=40 if case == "min_iterations" else 0)
    start = H.perturbed_start(obs, prob, scale=0.05)
    if case == "phase_only":
        start = start / np.abs(start)
    a = start.copy()
    r, _ = of.solve(prob, a, of.settings(**st), precision=32, n_threads=1)
    b = start.copy()
    rr = _ref_solve_problem(obs.cfg, obs.antenna1, obs.antenna2, prob, b, **st)
    assert r.iterations == rr.iterations
    n_used = int(np.minimum(obs.cfg.nspd, obs.cfg.n_times).sum())
    assert H.max_rel_diff(a[:, :, :n_used], b[:, :, :n_used]) < RTOL_PIN


def test_stall_detection_matches_reference(built):
    """An accuracy FP32 cannot reach (1e-14): the step magnitudes plateau at
    the FP32 noise floor and DetectStall (SolverBase.cc:63-86) stops the
    solve; both stop at the same iteration."""
    obs = H.small_observation(n_stations=10, n_directions=3, n_channels=8, n_cb=2,
                              n_times=3, seed=21)
    prob = H.problem_from_observation(obs)
    st = dict(max_iterations=3000, accuracy=1e-14, step_size=0.5)
    a = H.unit_solutions(prob)
    r, _ = of.solve(prob, a, of.settings(**st), precision=32, n_threads=1)
    b = H.unit_solutions(prob)
    rr = _ref_solve_problem(obs.cfg, obs.antenna1, obs.antenna2, prob, b, **st)
    assert r.has_stalled and r.iterations < 3000
    assert r.iterations == rr.iterations
    assert H.max_rel_diff(a, b) < RTOL_PIN


@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 1)])
def test_one_pass_matches_fp64_oracle(built, ncorr, npol):
    """The reference's PerformIteration output (through Solve with one
    iteration of step 1) against the FP64 oracle's pass: the FP32 reference
    is within 1e-4 per element of the FP64 answer on this case."""
    obs = H.small_observation(n_stations=9, n_directions=3, n_channels=12, n_cb=3,
                              n_times=4, nspd=[2, 1, 2], seed=11)
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.05)
    sol0 = H.perturbed_start(obs, prob)
    ref64 = of.perform_iteration(prob, sol0, precision=64)
    got = rf.perform_iteration(obs.cfg, obs.antenna1, obs.antenna2, prob["data"],
                               prob["model"], ncorr, npol, sol0)
    err = np.abs(got - ref64) / np.maximum(np.abs(ref64), 1e-12)
    assert np.nanmax(err) < 1e-4
