"""Full-Jones solver (2x2 gains on 4-correlation data; n_pol = 4 contexts)
against the reference's own IterativeFullJonesSolver (oracle/_ref, compiled
from ddecal/gain_solvers/IterativeFullJonesSolver.cc).

Full-Jones solutions are fixed only up to a unitary matrix per direction
(J -> J U leaves J_a M J_b^H unchanged): solutions are compared as J_a J_0^-1
(gauge invariant), the way phase referencing to antenna 0 serves the diagonal
solvers.

CPU: the reference oracle's solution of a noiseless interval reproduces the
data (a known-answer check of the oracle and of the test data). GPU: the
full-Jones path (fj_pass_kernel / fj_finalize_kernel) against the reference:
identical iteration counts and solutions within 1e-4 relative,
with and without DD solution intervals, a damped and a phase-only step, one
pass (ddsolve_perform_iteration) against the reference's first iteration,
and the non-finite repair of a flagged antenna.
"""
import numpy as np
import pytest

from dp3_b200 import synth
from oracle import ref_ffi as rf
from tests import helpers as H

RTOL = 1e-4


def full_jones_problem(n_stations=8, n_directions=2, n_channels=8, n_cb=2, n_times=3,
                       nspd=None, noise=0.0, seed=11):
    """A regular interval with 4-correlation models (random cross terms) and
    data = sum_d J_a M_d J_b^H + noise for random 2x2 gains J per (channel
    block, antenna, sub-solution): (obs, problem dict, true solutions
    [n_cb, n_ant, n_sub, 4])."""
    obs = H.small_observation(n_stations=n_stations, n_directions=n_directions,
                              n_channels=n_channels, n_cb=n_cb, n_times=n_times, nspd=nspd,
                              seed=seed)
    cfg = obs.cfg
    rng = np.random.default_rng(seed)
    n_sub = sum(cfg.nspd)
    truth = np.zeros((n_cb, cfg.n_stations, n_sub, 4), np.complex128)
    for cb in range(n_cb):
        diag = np.exp(0.1 * rng.standard_normal((cfg.n_stations, n_sub, 2))
                      + 1j * rng.uniform(-np.pi, np.pi, (cfg.n_stations, n_sub, 2)))
        cross = 0.1 * (rng.standard_normal((cfg.n_stations, n_sub, 2))
                       + 1j * rng.standard_normal((cfg.n_stations, n_sub, 2)))
        truth[cb, :, :, 0], truth[cb, :, :, 3] = diag[..., 0], diag[..., 1]
        truth[cb, :, :, 1], truth[cb, :, :, 2] = cross[..., 0], cross[..., 1]
    starts = np.cumsum([0] + list(cfg.nspd))[:-1]
    data, model = [], []
    for cb, nc in enumerate(cfg.cb_channels):
        m2 = obs.model[cb]  # [dir, n_vis, 2, 2] XX / YY
        n_vis = m2.shape[1]
        m = np.zeros((cfg.n_directions, n_vis, 2, 2), np.complex128)
        m[..., 0, 0] = m2[..., 0, 0] + 1j * m2[..., 0, 1]
        m[..., 1, 1] = m2[..., 1, 0] + 1j * m2[..., 1, 1]
        lk = 0.05 * (rng.standard_normal((cfg.n_directions, n_vis, 2))
                     + 1j * rng.standard_normal((cfg.n_directions, n_vis, 2)))
        m[..., 0, 1], m[..., 1, 0] = lk[..., 0], lk[..., 1]
        m = m.astype(np.complex64).astype(np.complex128)
        d = noise * (rng.standard_normal((n_vis, 2, 2)) + 1j * rng.standard_normal((n_vis, 2, 2)))
        v = np.arange(n_vis)
        t = v // (cfg.n_baselines * nc)
        bl = (v // nc) % cfg.n_baselines
        a1, a2 = np.asarray(obs.antenna1)[bl], np.asarray(obs.antenna2)[bl]
        for di in range(cfg.n_directions):
            n_s = cfg.nspd[di]
            sub = starts[di] + (t * min(n_s, cfg.n_times)) // cfg.n_times
            ja = truth[cb, a1, sub].reshape(n_vis, 2, 2)
            jb = truth[cb, a2, sub].reshape(n_vis, 2, 2)
            d += ja @ m[di] @ np.conj(np.swapaxes(jb, 1, 2))
        data.append(np.ascontiguousarray(
            np.stack([d.real, d.imag], -1).reshape(n_vis, 4, 2), np.float32))
        model.append(np.ascontiguousarray(
            np.stack([m.real, m.imag], -1).reshape(cfg.n_directions, n_vis, 4, 2), np.float32))
    prob = dict(n_antennas=cfg.n_stations, n_correlations=4, n_pol=4,
                n_solutions_per_direction=list(cfg.nspd), data=data, model=model)
    return obs, prob, truth


def perturbed(truth, scale=0.05, seed=3):
    rng = np.random.default_rng(seed)
    return truth + scale * (rng.standard_normal(truth.shape)
                            + 1j * rng.standard_normal(truth.shape))


def ref_solve(obs, prob, sol, st):
    return rf.solve(obs.cfg, obs.antenna1, obs.antenna2, prob["data"], prob["model"], 4, 4,
                    sol, st)


def gpu_context(obs, prob, st):
    from dp3_b200 import ddsolve
    cfg = obs.cfg
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 4, 4)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, prob["data"][cb],
                                      prob["model"][cb], obs.antenna1, obs.antenna2)
    ds = ddsolve.default_settings()
    ds.max_iterations, ds.accuracy, ds.step_size = st.max_iterations, st.accuracy, st.step_size
    ds.phase_only, ds.detect_stalling = st.phase_only, st.detect_stalling
    ctx.set_settings(ds)
    return ctx


def gauge_fixed(sol):
    """J_a J_0^-1 per (channel block, sub-solution): invariant under J -> J U."""
    j = sol.reshape(sol.shape[:3] + (2, 2))
    inv0 = np.linalg.inv(j[:, :1])
    return (j @ inv0).reshape(sol.shape)


def rel_diff(a, b):
    a, b = gauge_fixed(a), gauge_fixed(b)
    return float(np.nanmax(np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * np.nanmax(np.abs(b)))))


def residual_rms(obs, prob, sol):
    """rms |D - sum_d J_a M_d J_b^H| / rms |D| over the interval (invariant
    under the per-direction unitary gauge of full-Jones solutions)."""
    cfg = obs.cfg
    starts = np.cumsum([0] + list(cfg.nspd))[:-1]
    num = den = 0.0
    for cb, nc in enumerate(cfg.cb_channels):
        d = prob["data"][cb]
        n_vis = d.shape[0]
        res = (d[..., 0] + 1j * d[..., 1]).reshape(n_vis, 2, 2).astype(np.complex128)
        den += np.sum(np.abs(res) ** 2)
        v = np.arange(n_vis)
        t = v // (cfg.n_baselines * nc)
        bl = (v // nc) % cfg.n_baselines
        a1, a2 = np.asarray(obs.antenna1)[bl], np.asarray(obs.antenna2)[bl]
        for di in range(cfg.n_directions):
            m = prob["model"][cb][di]
            m = (m[..., 0] + 1j * m[..., 1]).reshape(n_vis, 2, 2)
            sub = starts[di] + (t * min(cfg.nspd[di], cfg.n_times)) // cfg.n_times
            ja = sol[cb, a1, sub].reshape(n_vis, 2, 2)
            jb = sol[cb, a2, sub].reshape(n_vis, 2, 2)
            res = res - ja @ m @ np.conj(np.swapaxes(jb, 1, 2))
        num += np.sum(np.abs(res) ** 2)
    return float(np.sqrt(num / den))


def test_reference_full_jones_recovers_true_gains(built):
    """A noiseless interval: the reference's solution reproduces the data
    (its gains equal the true ones up to the unitary gauge of each
    direction, under which J_a M J_b^H is invariant)."""
    obs, prob, truth = full_jones_problem()
    assert residual_rms(obs, prob, truth) < 1e-6
    st = rf.settings(max_iterations=500, accuracy=1e-9, step_size=0.5)
    sol = perturbed(truth, 0.05)
    start_rms = residual_rms(obs, prob, sol)
    r = ref_solve(obs, prob, sol, st)
    assert r.iterations >= 2
    assert residual_rms(obs, prob, sol) < 1e-2 * start_rms


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["plain", "dd", "phase_only", "three_dirs", "six_dirs_dd",
                                  "nine_dirs"])
def test_full_jones_matches_reference(built, case):
    """Full solves against the reference; six and nine directions take the
    chunked pass (directions in launches of four)."""
    kw = dict(nspd=[2, 1]) if case == "dd" else {}
    if case == "three_dirs":
        kw = dict(n_directions=3)
    if case == "six_dirs_dd":
        kw = dict(n_directions=6, nspd=[1, 2, 1, 3, 1, 2])
    if case == "nine_dirs":
        kw = dict(n_directions=9, n_stations=10)
    obs, prob, truth = full_jones_problem(noise=0.01, **kw)
    st = rf.settings(max_iterations=80, accuracy=1e-5, phase_only=case == "phase_only")
    start = perturbed(truth, 0.05)
    if case == "phase_only":
        start = start / np.abs(start)
    ref = start.copy()
    rr = ref_solve(obs, prob, ref, st)
    ctx = gpu_context(obs, prob, st)
    got = start.copy()
    res = ctx.solve(got)
    ctx.close()
    assert res.iterations == rr.iterations
    assert rel_diff(got, ref) < RTOL


@pytest.mark.gpu
@pytest.mark.parametrize("n_directions", [2, 7])
def test_full_jones_one_pass_matches_reference_first_iteration(built, n_directions):
    """ddsolve_perform_iteration (the undamped next solutions) stepped by
    hand equals the reference's first iteration (max_iterations = 1)."""
    obs, prob, truth = full_jones_problem(noise=0.01, n_directions=n_directions)
    st = rf.settings(max_iterations=1, accuracy=1e-12, step_size=1.0)
    start = perturbed(truth, 0.1)
    ref = start.copy()
    ref_solve(obs, prob, ref, st)
    ctx = gpu_context(obs, prob, st)
    nxt = ctx.perform_iteration(start)
    ctx.close()
    assert rel_diff(nxt, ref) < RTOL


@pytest.mark.gpu
def test_full_jones_flagged_antenna(built):
    """An antenna whose data is all zero: its normal equations are singular
    (NaN solutions, as the reference's failed Invert), repaired by
    MakeSolutionsFinite4Pol at the next iteration; iteration count and the
    other antennas as the reference."""
    obs, prob, truth = full_jones_problem(noise=0.01)
    cfg = obs.cfg
    bad = 3
    a1, a2 = np.asarray(obs.antenna1), np.asarray(obs.antenna2)
    for cb, nc in enumerate(cfg.cb_channels):
        n_vis = prob["data"][cb].shape[0]
        bl = (np.arange(n_vis) // nc) % cfg.n_baselines
        hit = (a1[bl] == bad) | (a2[bl] == bad)
        prob["data"][cb][hit] = 0.0
        prob["model"][cb][:, hit] = 0.0
    st = rf.settings(max_iterations=40, accuracy=1e-5)
    start = perturbed(truth, 0.05)
    ref = start.copy()
    rr = ref_solve(obs, prob, ref, st)
    ctx = gpu_context(obs, prob, st)
    got = start.copy()
    res = ctx.solve(got)
    ctx.close()
    assert res.iterations == rr.iterations
    keep = np.arange(cfg.n_stations) != bad
    assert rel_diff(got[:, keep], ref[:, keep]) < RTOL
    np.testing.assert_allclose(got[:, bad], ref[:, bad], rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("nspd", [None, [2, 1]])
def test_full_jones_adapter_matches_dp3(built, nspd):
    """The DP3 adapter's full-Jones instance (IterativeFullJonesSolverB200)
    against DP3's own IterativeFullJonesSolver on the same SolveData, both set
    up through DP3's SolverBase (tests/adapter)."""
    from tests import test_dp3_adapter as A
    obs, prob, truth = full_jones_problem(noise=0.01, nspd=nspd)
    st = rf.settings(max_iterations=80, accuracy=1e-5)
    start = perturbed(truth, 0.05)
    a, b = start.copy(), start.copy()
    rd, _ = A.run(obs, prob, a, st, use_b200=False)
    rg, _ = A.run(obs, prob, b, st, use_b200=True)
    assert rg.iterations == rd.iterations
    assert rel_diff(b, a) < RTOL
