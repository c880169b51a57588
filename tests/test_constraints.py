"""Host constraints between device passes (SolverBase::ApplyConstraints,
ddecal/gain_solvers/SolverBase.cc:160-190, driven as in
IterativeDiagonalSolver.cc:38-97): the mirror's host loop.

CPU: with the oracle's pass in place of the GPU's, the host loop with a
constraint that changes nothing reproduces the oracle's own solve (iteration
count, step magnitudes, solutions), and AntennaConstraint leaves each set of
antennas with equal solutions. GPU: the same loop over the GPU pass matches
the oracle-driven loop (identical iteration counts, 1e-4 after antenna-0
phase referencing) and, with no-op constraints, the device-only solve."""
import numpy as np
import pytest

from dp3_b200.solvers import AntennaConstraint, Constraint
from oracle import oracle_ffi as of
from tests import helpers as H

RTOL = 1e-4


class NoOp(Constraint):
    def Apply(self, solutions, time):
        pass


def _problem(seed=3):
    obs = H.small_observation(n_stations=10, n_directions=2, n_channels=8, n_cb=2,
                              n_times=2, seed=seed)
    return obs, H.problem_from_observation(obs)


def _oracle_perform(prob):
    return lambda sol: of.perform_iteration(prob, sol, precision=32, n_threads=4)


@pytest.mark.parametrize("npol", [2, 1])
def test_host_loop_with_noop_constraint_reproduces_oracle_solve(npol):
    obs, prob = _problem()
    prob = H.problem_from_observation(obs, 2, npol)
    st = of.settings(max_iterations=40, accuracy=1e-5, step_size=0.2)
    ref = H.unit_solutions(prob)
    r, mags = of.solve(prob, ref, st, precision=32, n_threads=4)
    solver = H.make_solver(prob, max_iterations=40, accuracy=1e-5, step_size=0.2)
    solver.AddConstraint(NoOp())
    got = H.unit_solutions(prob)
    res = solver._solve_with_constraints(_oracle_perform(prob), got, 0.0, None)
    assert res.iterations == r.iterations
    np.testing.assert_allclose(res.step_magnitudes, mags[:len(res.step_magnitudes)],
                               rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-12)


def test_antenna_constraint_equalises_sets():
    obs, prob = _problem(seed=4)
    solver = H.make_solver(prob, max_iterations=15)
    solver.AddConstraint(AntennaConstraint([[0, 1, 2], [5, 7]]))
    got = H.unit_solutions(prob)
    solver._solve_with_constraints(_oracle_perform(prob), got, 0.0, None)
    for ants in ([0, 1, 2], [5, 7]):
        for a in ants[1:]:
            np.testing.assert_allclose(got[:, a], got[:, ants[0]], rtol=1e-12)


@pytest.mark.gpu
def test_gpu_host_loop_matches_oracle_loop(built):
    obs, prob = _problem(seed=5)
    sd = obs.solve_data()
    ref_solver = H.make_solver(prob, max_iterations=30)
    ref_solver.AddConstraint(AntennaConstraint([[0, 1, 2]]))
    ref = H.unit_solutions(prob)
    r = ref_solver._solve_with_constraints(_oracle_perform(prob), ref, 0.0, None)
    solver = H.make_solver(prob, max_iterations=30)
    solver.AddConstraint(AntennaConstraint([[0, 1, 2]]))
    got = H.unit_solutions(prob)
    res = solver.Solve(sd, got, 0.0)
    assert res.iterations == r.iterations
    assert H.max_rel_diff(got, ref) < RTOL


@pytest.mark.gpu
def test_gpu_host_loop_noop_matches_device_loop(built):
    obs, prob = _problem(seed=6)
    sd = obs.solve_data()
    dev = H.make_solver(prob, max_iterations=40)
    a = H.unit_solutions(prob)
    ra = dev.Solve(sd, a, 0.0)
    host = H.make_solver(prob, max_iterations=40)
    host.AddConstraint(NoOp())
    b = H.unit_solutions(prob)
    rb = host.Solve(sd, b, 0.0)
    assert ra.iterations == rb.iterations
    assert H.max_rel_diff(b, a) < RTOL
