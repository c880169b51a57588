"""Shared helpers of the test suite (problem builders and comparisons)."""
import numpy as np

from dp3_b200 import synth
from dp3_b200.solvers import (IterativeDiagonalSolver, IterativeScalarSolver,
                              SolveData)


def to_ncorr(arr_2corr, ncorr):
    """Converts XX/YY arrays [..., 2, 2] to 1 (mean of XX, YY) or 4
    correlations (XY = YX = 0), the ToSpecificMatrix conversions of
    ddecal/gain_solvers/SolveData.cc:18-31 applied to diagonal data."""
    if ncorr == 2:
        return np.ascontiguousarray(arr_2corr)
    if ncorr == 1:
        c = arr_2corr[..., 0, :] + arr_2corr[..., 1, :]
        return np.ascontiguousarray((0.5 * c)[..., None, :].astype(np.float32))
    shp = arr_2corr.shape[:-2] + (4, 2)
    out = np.zeros(shp, np.float32)
    out[..., 0, :] = arr_2corr[..., 0, :]
    out[..., 3, :] = arr_2corr[..., 1, :]
    return out


def problem_from_observation(obs, ncorr=2, npol=2, leakage=0.0, seed=0):
    """Oracle problem dict of an Observation. With ncorr == 4 and leakage > 0
    the off-diagonal correlations get random model/data content."""
    ap, sm = obs.generic_arrays()
    data = [to_ncorr(d, ncorr) for d in obs.data]
    model = [to_ncorr(m, ncorr) for m in obs.model]
    if ncorr == 4 and leakage > 0:
        rng = np.random.default_rng(seed)
        for d, m in zip(data, model):
            m[..., 1:3, :] += leakage * rng.standard_normal(m[..., 1:3, :].shape).astype(np.float32)
            d[..., 1:3, :] += leakage * rng.standard_normal(d[..., 1:3, :].shape).astype(np.float32)
    return dict(n_antennas=obs.cfg.n_stations, n_correlations=ncorr, n_pol=npol,
                n_solutions_per_direction=list(obs.cfg.nspd), data=data,
                model=model, antenna_pairs=ap, solution_map=sm)


def solve_data_from_problem(problem):
    return SolveData.from_arrays(problem["data"], problem["model"],
                                 problem["antenna_pairs"],
                                 problem["solution_map"],
                                 problem["n_correlations"])


def make_solver(problem, max_iterations=50, accuracy=1e-5, step_size=0.2,
                detect_stalling=True, phase_only=False, min_iterations=0):
    cls = IterativeDiagonalSolver if problem["n_pol"] == 2 else IterativeScalarSolver
    s = cls()
    s.SetMaxIterations(max_iterations)
    s.SetMinIterations(min_iterations)
    s.SetAccuracy(accuracy)
    s.SetStepSize(step_size)
    s.SetDetectStalling(detect_stalling, 0.1)
    s.SetPhaseOnly(phase_only)
    s.Initialize(problem["n_antennas"], problem["n_solutions_per_direction"],
                 len(problem["data"]))
    return s


def perturbed_start(obs, problem, scale=0.3, seed=3):
    """Initial solutions: true gain at the block's first channel times a
    random perturbation, so one pass does real work."""
    cfg = obs.cfg
    rng = np.random.default_rng(seed)
    ncb = cfg.n_channel_blocks
    n_sub = sum(problem["n_solutions_per_direction"])
    npol = problem["n_pol"]
    starts = np.cumsum([0] + list(cfg.cb_channels))[:-1]
    sol = np.ones((ncb, cfg.n_stations, n_sub, npol), np.complex128)
    d_of_sub = np.repeat(np.arange(cfg.n_directions),
                         problem["n_solutions_per_direction"])
    for cb in range(ncb):
        g = obs.true_gains[starts[cb]]  # [st, dir, 2]
        for s in range(n_sub):
            gg = g[:, d_of_sub[s], :npol]
            pert = 1 + scale * (rng.standard_normal(gg.shape)
                                + 1j * rng.standard_normal(gg.shape))
            sol[cb, :, s, :] = gg * pert
    return sol


def unit_solutions(problem):
    n_sub = sum(problem["n_solutions_per_direction"])
    return np.ones((len(problem["data"]), problem["n_antennas"], n_sub,
                    problem["n_pol"]), np.complex128)


def phase_referenced(sol):
    """Solutions [cb, ant, sub, pol] referenced to antenna 0's phase."""
    ref = sol[:, :1, :, :]
    ph = np.where(np.abs(ref) > 0, ref / np.abs(ref), 1.0)
    return sol * np.conj(ph)


def max_rel_diff(a, b):
    """max |a - b| / max(|b|, tiny) over all finite elements, after phase
    referencing to antenna 0."""
    ar, br = phase_referenced(a), phase_referenced(b)
    denom = np.maximum(np.abs(br), 1e-30)
    d = np.abs(ar - br) / denom
    return float(np.nanmax(d))


def small_observation(**kw):
    cfg = synth.small_config(**kw)
    return synth.observe(cfg)
