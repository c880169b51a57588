"""Device-side constraints (ddsolve_add_smoothness_constraint,
ddsolve_add_antenna_constraint, ddsolve_add_reference_antenna_constraint)
against the reference's own solver with DP3's own constraint classes
(oracle/_ref: SmoothnessConstraint.cc, AntennaConstraint.h and
Constraint::ApplyReferenceAntenna compiled from the reference sources),
applied by DP3's SolverBase::ApplyConstraints between Step and
AssignSolutions (IterativeDiagonalSolver.cc:77-83).

GPU: the whole constrained loop runs on the device (one CUDA graph); the
iteration count equals the reference's and the solutions agree to 1e-4
relative after phase referencing to antenna 0 (the parity tolerance), on
the pipelined path (2 and 4 correlations) and on the streaming path
(1 correlation), diagonal and scalar. CPU: the reference-oracle side of the
new constraint options.
"""
import numpy as np
import pytest

from dp3_b200 import synth
from oracle import ref_ffi as rf
from tests import helpers as H

RTOL = 1e-4


def _cb_frequencies(cfg):
    freqs = synth.frequencies(cfg)
    edges = np.cumsum([0] + list(cfg.cb_channels))
    return np.array([freqs[lo:hi].mean() for lo, hi in zip(edges[:-1], edges[1:])])


def _observation(nspd=None, seed=23):
    return H.small_observation(n_stations=10, n_directions=3, n_channels=16, n_cb=8,
                               n_times=4, nspd=nspd, seed=seed)


def _case(name, obs, n_sub):
    """Constraint set of a test case: keyword arguments of rf.solve."""
    cfg = obs.cfg
    n_ant, n_cb = cfg.n_stations, len(cfg.cb_channels)
    rng = np.random.default_rng(5)
    weights = rng.uniform(0.5, 2.0, n_ant * n_cb)
    if name == "smoothness":
        return dict(smoothness=dict(bandwidth_hz=10e6))
    if name == "smoothness_factors":
        return dict(smoothness=dict(bandwidth_hz=8e6, bandwidth_ref_frequency_hz=130e6,
                                    spectral_exponent=-1.0, weights=weights,
                                    antenna_factors=rng.uniform(0.7, 1.5, n_ant),
                                    dd_factors=rng.uniform(0.5, 2.0, n_sub)))
    if name == "sub_weights":
        return dict(smoothness=dict(bandwidth_hz=12e6, kernel_truncation=False,
                                    sub_solution_weights=rng.uniform(0.5, 2.0,
                                                                     (n_sub, n_ant * n_cb))))
    if name == "antenna":
        return dict(antenna_sets=[[0, 1, 2, 3], [7, 5]])
    if name == "reference":
        return dict(reference_antenna=True)
    if name == "all":
        return dict(antenna_sets=[[1, 2, 3]], smoothness=dict(bandwidth_hz=10e6, weights=weights),
                    reference_antenna=True)
    raise ValueError(name)


def _add_to_context(ctx, case, cb_freqs):
    """The same constraints on the device, in the reference's order
    (antenna, smoothness, reference antenna: the order the oracle adds them)."""
    if case.get("antenna_sets"):
        ctx.add_antenna_constraint(case["antenna_sets"])
    s = case.get("smoothness")
    if s:
        n = len(cb_freqs)
        w = s.get("weights")
        if w is None and s.get("sub_solution_weights") is None:
            w = np.ones(ctx.n_antennas * n)
        ctx.add_smoothness_constraint(
            cb_freqs, s["bandwidth_hz"], weights=w,
            bandwidth_ref_frequency_hz=s.get("bandwidth_ref_frequency_hz", 0.0),
            spectral_exponent=s.get("spectral_exponent", -1.0),
            kernel_truncation=s.get("kernel_truncation", True),
            sub_solution_weights=s.get("sub_solution_weights"),
            antenna_factors=s.get("antenna_factors"), dd_factors=s.get("dd_factors"))
    if case.get("reference_antenna"):
        ctx.add_reference_antenna_constraint()


def test_reference_oracle_constraint_options(built):
    """The reference oracle with the phase-referencing constraint leaves the
    reference antenna at exactly 1, and the antenna-factor / dd-factor /
    sub-solution-weight options of the smoothness constraint run."""
    obs = _observation()
    prob = H.problem_from_observation(obs)
    n_sub = sum(obs.cfg.nspd)
    st = rf.settings(max_iterations=20, accuracy=1e-5)
    for name in ("reference", "smoothness_factors", "sub_weights"):
        sol = H.perturbed_start(obs, prob, scale=0.05)
        r = rf.solve(obs.cfg, obs.antenna1, obs.antenna2, prob["data"], prob["model"], 2, 2,
                     sol, st, cb_frequencies=_cb_frequencies(obs.cfg), **_case(name, obs, n_sub))
        assert r.iterations >= 1 and np.all(np.isfinite(sol))
        if name == "reference":
            np.testing.assert_array_equal(sol[:, 0], 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (1, 1), (2, 1)])
@pytest.mark.parametrize("name", ["smoothness", "smoothness_factors", "sub_weights",
                                  "antenna", "reference", "all"])
def test_device_constraints_match_reference(built, ncorr, npol, name):
    from dp3_b200 import ddsolve
    obs = _observation(nspd=[2, 1, 2] if name == "all" else None)
    cfg = obs.cfg
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.02)
    n_sub = sum(cfg.nspd)
    case = _case(name, obs, n_sub)
    cb_freqs = _cb_frequencies(cfg)
    st = rf.settings(max_iterations=80, accuracy=1e-5)
    start = H.perturbed_start(obs, prob, scale=0.05)
    ref = start.copy()
    rr = rf.solve(cfg, obs.antenna1, obs.antenna2, prob["data"], prob["model"], ncorr, npol,
                  ref, st, cb_frequencies=cb_freqs, **case)

    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, ncorr, npol)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, prob["data"][cb],
                                      prob["model"][cb], obs.antenna1, obs.antenna2)
    ds = ddsolve.default_settings()
    ds.max_iterations, ds.accuracy = st.max_iterations, st.accuracy
    ctx.set_settings(ds)
    _add_to_context(ctx, case, cb_freqs)
    got = start.copy()
    mags = np.full(st.max_iterations, np.nan)
    res = ctx.solve(got, mags)
    assert ctx.last_launch_count() > res.iterations  # constraint kernels in the loop
    ctx.close()
    assert res.iterations == rr.iterations
    assert H.max_rel_diff(got, ref) < RTOL
    if name == "antenna":  # the last constraint applied: the sets share one solution
        for s in case["antenna_sets"]:
            s = sorted(s)
            np.testing.assert_allclose(got[:, s[1:]], np.repeat(got[:, s[:1]], len(s) - 1, 1),
                                       rtol=1e-12)


@pytest.mark.gpu
def test_device_constraints_cleared_and_unsupported_batch(built):
    """Clearing the constraints gives the unconstrained solve again; a
    batched context refuses device constraints."""
    from dp3_b200 import ddsolve
    obs = _observation()
    cfg = obs.cfg
    prob = H.problem_from_observation(obs)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                      obs.model[cb], obs.antenna1, obs.antenna2)
    start = H.perturbed_start(obs, prob, scale=0.05)
    plain = start.copy()
    r0 = ctx.solve(plain)
    ctx.add_antenna_constraint([[0, 1]])
    cons = start.copy()
    ctx.solve(cons)
    np.testing.assert_array_equal(cons[:, 0], cons[:, 1])
    ctx.clear_constraints()
    again = start.copy()
    r1 = ctx.solve(again)
    assert r1.iterations == r0.iterations
    np.testing.assert_array_equal(again, plain)
    ctx.add_antenna_constraint([[0, 1]])
    ctx.set_intervals([0, 4, cfg.n_channel_blocks])
    with pytest.raises(RuntimeError, match="single-interval"):
        ctx.solve_batch(start.copy())
    ctx.close()
