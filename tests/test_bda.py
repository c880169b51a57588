"""Baseline-dependently averaged (BDA) intervals.

DDECal packs BDA data through its second SolveData constructor
(ddecal/gain_solvers/SolveData.cc:190-300), restated in oracle/bda_oracle.py:
rows of differing channel counts are split over the channel blocks by their
own channel count, autocorrelations are dropped and solution indices come from
nearest-neighbour binning of each row's mid time. The product solves the
result through the generic per-visibility entry point, so the GPU tests check
that path on such data (runs of every length, empty channel-block splits,
shuffled row order) against the FP64 and FP32 oracles with the tolerances of
tests/test_gpu_parity.py: 1e-4 relative per element for one pass, identical
iteration counts and 1e-4 after phase referencing for full solves.
"""
import numpy as np
import pytest

from oracle import bda_oracle as bda
from oracle import oracle_ffi as of
from tests import helpers as H

RTOL_PASS = 1e-4
RTOL_SOLVE = 1e-4


def _factors(n_bl, seed):
    rng = np.random.default_rng(seed)
    return rng.choice([1, 2, 3, 6], n_bl), rng.choice([1, 2, 3, 4, 6], n_bl)


def bda_problem(obs, ncorr=2, npol=2, seed=0, shuffle=True, leakage=0.0,
                antenna2=None, unit_factors=False):
    cfg = obs.cfg
    if unit_factors:
        tf = ff = np.ones(cfg.n_baselines, int)
    else:
        tf, ff = _factors(cfg.n_baselines, seed)
        tf[0] = ff[0] = 1
    rng = np.random.default_rng(seed + 1) if shuffle else None
    rows, duration = bda.bda_rows(obs, tf, ff, rng)
    # The solvers take SolutionIndex(d, 0) as direction d's lowest index
    # (SolveData.h:72-80): an unaveraged cross-correlation row at the
    # interval start goes first.
    first = next(i for i, r in enumerate(rows)
                 if r["baseline"] == 0 and r["time"] == 0.5 * bda.TIME_STEP_S)
    rows.insert(0, rows.pop(first))
    a2 = obs.antenna2 if antenna2 is None else antenna2
    blocks, n_sol = bda.bda_solve_data(rows, duration, obs.antenna1, a2,
                                       cfg.n_channel_blocks, list(cfg.nspd))
    data = [H.to_ncorr(b["data"], ncorr) for b in blocks]
    model = [H.to_ncorr(b["model"], ncorr) for b in blocks]
    if ncorr == 4 and leakage > 0:
        r = np.random.default_rng(seed + 2)
        for d, m in zip(data, model):
            m[..., 1:3, :] += leakage * r.standard_normal(m[..., 1:3, :].shape).astype(np.float32)
            d[..., 1:3, :] += leakage * r.standard_normal(d[..., 1:3, :].shape).astype(np.float32)
    prob = dict(n_antennas=cfg.n_stations, n_correlations=ncorr, n_pol=npol,
                n_solutions_per_direction=list(n_sol), data=data, model=model,
                antenna_pairs=[b["antenna_pairs"] for b in blocks],
                solution_map=[b["solution_map"] for b in blocks])
    return prob, rows


def _obs(seed=31, nspd=(1, 2, 3)):
    return H.small_observation(n_stations=9, n_directions=3, n_channels=12,
                               n_cb=3, n_times=6, seed=seed, nspd=list(nspd))


def test_bda_packing_unit_factors_matches_regular():
    """Unaveraged rows in time-major order pack to exactly the regular
    constructor's visibilities; with solution counts that divide the time
    count the nearest-neighbour binning gives the regular solution map."""
    obs = _obs(nspd=(1, 2, 3))
    prob, _ = bda_problem(obs, shuffle=False, unit_factors=True)
    ref = H.problem_from_observation(obs)
    for cb in range(obs.cfg.n_channel_blocks):
        np.testing.assert_array_equal(prob["data"][cb], ref["data"][cb])
        np.testing.assert_array_equal(prob["model"][cb], ref["model"][cb])
        np.testing.assert_array_equal(prob["antenna_pairs"][cb], ref["antenna_pairs"][cb])
        np.testing.assert_array_equal(prob["solution_map"][cb], ref["solution_map"][cb])


def test_bda_packing_counts_and_bins():
    """Averaged rows: per-block visibility counts follow the per-row channel
    split, autocorrelation rows are dropped, and every solution index lies in
    its direction's range; solution counts are limited by the row count."""
    obs = _obs(nspd=(1, 2, 3))
    cfg = obs.cfg
    a2 = obs.antenna2.copy()
    a2[0] = obs.antenna1[0]  # baseline 0 becomes an autocorrelation
    prob, rows = bda_problem(obs, antenna2=a2, seed=4)
    n_cb = cfg.n_channel_blocks
    want = np.zeros(n_cb, int)
    for r in rows:
        if r["baseline"] == 0:
            continue
        n = r["n_channels"]
        for cb in range(n_cb):
            want[cb] += (cb + 1) * n // n_cb - cb * n // n_cb
    assert [len(d) for d in prob["data"]] == list(want)
    assert all(want > 0)
    ap = np.concatenate(prob["antenna_pairs"])
    assert np.all(ap[:, 0] != ap[:, 1])
    start = np.concatenate([[0], np.cumsum(prob["n_solutions_per_direction"])[:-1]])
    for sm in prob["solution_map"]:
        for d, n in enumerate(prob["n_solutions_per_direction"]):
            assert np.all((sm[d] >= start[d]) & (sm[d] < start[d] + n))
    assert bda.limit_n_solutions([5, 1, 40], 7) == [5, 1, 7]


def test_bda_oracle_pass_is_finite():
    obs = _obs()
    prob, _ = bda_problem(obs)
    sol0 = H.perturbed_start(obs, prob, scale=0.2)
    out = of.perform_iteration(prob, sol0, precision=64)
    assert out.shape == sol0.shape and np.all(np.isfinite(out))


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (1, 1), (4, 2), (2, 1)])
@pytest.mark.parametrize("seed", [0, 7])
def test_bda_perform_iteration_matches_fp64_oracle(built, ncorr, npol, seed):
    obs = _obs(seed=31 + seed)
    prob, _ = bda_problem(obs, ncorr, npol, seed=seed, leakage=0.05)
    sol0 = H.perturbed_start(obs, prob, scale=0.2)
    ref = of.perform_iteration(prob, sol0, precision=64)
    solver = H.make_solver(prob)
    got = solver.PerformIteration(H.solve_data_from_problem(prob), sol0)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (1, 1)])
def test_bda_solve_matches_oracle(built, ncorr, npol):
    obs = _obs(seed=41)
    prob, _ = bda_problem(obs, ncorr, npol, seed=3)
    sol0 = H.perturbed_start(obs, prob, scale=0.05)
    st = of.settings(max_iterations=50, accuracy=1e-5)
    ref32 = sol0.copy()
    r32, _ = of.solve(prob, ref32, st, precision=32, n_threads=4)
    ref64 = sol0.copy()
    r64, m64 = of.solve(prob, ref64, st, precision=64, n_threads=4)
    solver = H.make_solver(prob, max_iterations=50, accuracy=1e-5)
    got = sol0.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations == r32.iterations == r64.iterations
    assert H.max_rel_diff(got, ref32) < RTOL_SOLVE
    assert H.max_rel_diff(got, ref64) < RTOL_SOLVE
    np.testing.assert_allclose(res.step_magnitudes, m64, rtol=1e-3, atol=1e-12)
