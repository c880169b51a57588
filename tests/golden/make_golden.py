"""Writes the regression fixtures of tests/test_oracle.py.

The fixtures are outputs of the FP64 oracle (oracle/ddecal_oracle.cc) on
small seeded inputs; the oracle itself is pinned to the reference's own
known-answer tests (SolverTester recipe, tSolvers.cc) in test_oracle.py.
Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle_ffi as of  # noqa: E402
from tests import helpers as H  # noqa: E402


def _save(name, prob, sol0, max_iterations=20, accuracy=1e-5, with_inputs=True):
    out = dict(n_cb=len(prob["data"]), n_antennas=prob["n_antennas"],
               n_correlations=prob["n_correlations"], n_pol=prob["n_pol"],
               nspd=np.asarray(prob["n_solutions_per_direction"], np.uint32),
               sol0=sol0)
    if with_inputs:
        for i in range(len(prob["data"])):
            out[f"data{i}"] = prob["data"][i]
            out[f"model{i}"] = prob["model"][i]
            out[f"ap{i}"] = prob["antenna_pairs"][i]
            out[f"sm{i}"] = prob["solution_map"][i]
    out["next64"] = of.perform_iteration(prob, sol0, precision=64)
    if with_inputs:
        st = of.settings(max_iterations=max_iterations, accuracy=accuracy)
        s = sol0.copy()
        r, _ = of.solve(prob, s, st, precision=64, n_threads=1)
        out["solved64"] = s
        out["iterations"] = r.iterations
        out["max_iterations"] = max_iterations
        out["accuracy"] = accuracy
    np.savez_compressed(os.path.join(HERE, name), **out)


def main():
    of.build()
    obs = H.small_observation(n_stations=8, n_directions=2, n_channels=8,
                              n_cb=2, n_times=2, seed=41, nspd=[1, 2])
    prob = H.problem_from_observation(obs, 2, 2)
    _save("small_diag_duo.npz", prob, H.unit_solutions(prob))
    obs = H.small_observation(n_stations=7, n_directions=3, n_channels=6,
                              n_cb=3, n_times=2, seed=43)
    prob = H.problem_from_observation(obs, 4, 1, leakage=0.05, seed=2)
    _save("small_scalar_full.npz", prob, H.unit_solutions(prob))
    prob, inp, init = of.solver_tester_problem(True, True, 4)
    _save("solver_tester_pass.npz", prob, init, with_inputs=False)


if __name__ == "__main__":
    main()
