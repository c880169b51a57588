"""GPU parity of the CUDA solver against the CPU oracle, through the C ABI.

Tolerances (the parity contract of this path):
  * one direction-iterative pass (next_solutions before the step): relative
    difference <= 1e-4 per element vs the FP64 oracle;
  * full solves: identical iteration counts and max relative difference
    <= 1e-4 after phase-referencing to antenna 0, vs the oracle run with the
    reference's own FP32 arithmetic, and vs the FP64 oracle.
"""
import numpy as np
import pytest

from dp3_b200 import synth
from dp3_b200.solvers import SolveData
from oracle import oracle_ffi as of
from tests import helpers as H

pytestmark = pytest.mark.gpu

RTOL_PASS = 1e-4
RTOL_SOLVE = 1e-4

COMBOS = [(2, 2), (4, 2), (1, 1), (2, 1), (4, 1)]


_perturbed_start = H.perturbed_start


@pytest.mark.parametrize("ncorr,npol", COMBOS)
@pytest.mark.parametrize("regular", [True, False])
@pytest.mark.parametrize("dd", [False, True])
def test_perform_iteration_matches_fp64_oracle(built, ncorr, npol, regular, dd):
    nspd = [2, 1, 2] if dd else None
    obs = H.small_observation(n_stations=9, n_directions=3, n_channels=12,
                              n_cb=3, n_times=4, nspd=nspd, seed=11)
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.05)
    sol0 = _perturbed_start(obs, prob)
    ref = of.perform_iteration(prob, sol0, precision=64)
    solver = H.make_solver(prob)
    if regular:
        cfg = obs.cfg
        sd = SolveData.regular(prob["data"], prob["model"], cfg.n_times,
                               cfg.n_baselines, cfg.cb_channels, obs.antenna1,
                               obs.antenna2, ncorr)
    else:
        sd = H.solve_data_from_problem(prob)
    got = solver.PerformIteration(sd, sol0)
    assert got.shape == ref.shape
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)


@pytest.mark.parametrize("ncorr,npol", COMBOS)
def test_solve_matches_oracle(built, ncorr, npol):
    obs = H.small_observation(n_stations=10, n_directions=3, n_channels=8,
                              n_cb=2, n_times=3, seed=21)
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.02)
    sol0 = _perturbed_start(obs, prob, scale=0.05)
    st = of.settings(max_iterations=50, accuracy=1e-5)
    ref32 = sol0.copy()
    r32, m32 = of.solve(prob, ref32, st, precision=32, n_threads=4)
    ref64 = sol0.copy()
    r64, m64 = of.solve(prob, ref64, st, precision=64, n_threads=4)
    solver = H.make_solver(prob, max_iterations=50, accuracy=1e-5)
    got = sol0.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations == r32.iterations == r64.iterations
    assert H.max_rel_diff(got, ref32) < RTOL_SOLVE
    assert H.max_rel_diff(got, ref64) < RTOL_SOLVE
    np.testing.assert_allclose(res.step_magnitudes, m64, rtol=1e-3, atol=1e-12)


@pytest.mark.parametrize("cfg_index", [0, 4])
def test_benchmark_config_parity(built, cfg_index):
    """Benchmark configs c0 (full size) and c4 (full size): unit start,
    tolerance 1e-5, max 50 iterations."""
    cfg = synth.benchmark_configs()[cfg_index]
    obs = synth.observe(cfg)
    prob = H.problem_from_observation(obs)
    st = of.settings(max_iterations=cfg.max_iterations, accuracy=cfg.tolerance,
                     step_size=cfg.step_size)
    ref = H.unit_solutions(prob)
    r, mags = of.solve(prob, ref, st, precision=32, n_threads=8)
    solver = H.make_solver(prob, cfg.max_iterations, cfg.tolerance, cfg.step_size)
    got = H.unit_solutions(prob)
    res = solver.Solve(obs.solve_data(), got, 0.0)
    assert res.iterations == r.iterations
    assert H.max_rel_diff(got, ref) < RTOL_SOLVE


def test_converging_solve_same_iteration_count(built):
    """A case that converges before max iterations: counts must match."""
    obs = H.small_observation(n_stations=12, n_directions=2, n_channels=8,
                              n_cb=2, n_times=2, seed=5)
    prob = H.problem_from_observation(obs)
    sol0 = _perturbed_start(obs, prob, scale=0.01)
    st = of.settings(max_iterations=100, accuracy=1e-5)
    ref = sol0.copy()
    r, _ = of.solve(prob, ref, st, precision=32, n_threads=2)
    assert r.has_converged and r.iterations < 100
    solver = H.make_solver(prob, max_iterations=100, accuracy=1e-5)
    got = sol0.copy()
    res = solver.Solve(obs.solve_data(), got, 0.0)
    assert res.has_converged
    assert res.iterations == r.iterations
    assert H.max_rel_diff(got, ref) < RTOL_SOLVE


@pytest.mark.parametrize("ncorr", [4, 2])
def test_solver_tester_diagonal_dd(built, ncorr):
    """tSolvers.cc iterative_diagonal_dd_intervals / iterative_duo_diagonal_dd_
    intervals: CheckDualResults(1e-2) against the true gains and
    iterations <= max + 1; plus parity with the oracle on the same data."""
    prob, inp, init = of.solver_tester_problem(True, True, ncorr)
    solver = H.make_solver(prob, max_iterations=100, accuracy=1e-8)
    got = init.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations <= 101
    _check_dual_results(got, inp, 1e-2)
    st = of.settings(max_iterations=100, accuracy=1e-8)
    ref = init.copy()
    r, _ = of.solve(prob, ref, st, precision=32, n_threads=8)
    assert H.max_rel_diff(got, ref) < RTOL_SOLVE
    # The fixture's accuracy (1e-8) lies below the noise floor of the
    # reference's FP32 accumulators (step magnitudes plateau near 7e-8 for
    # the XX/YY case), so the iteration count is compared with the FP64
    # oracle, which the compensated GPU sums follow.
    ref64 = init.copy()
    r64, _ = of.solve(prob, ref64, st, precision=64, n_threads=8)
    assert res.iterations == r64.iterations
    assert H.max_rel_diff(got, ref64) < RTOL_SOLVE


@pytest.mark.parametrize("ncorr", [4, 2, 1])
def test_solver_tester_scalar_dd(built, ncorr):
    """tSolvers.cc iterative_{,duo_,uni_}scalar_dd_intervals:
    CheckScalarResults(1e-3)."""
    prob, inp, init = of.solver_tester_problem(False, True, ncorr)
    solver = H.make_solver(prob, max_iterations=100, accuracy=1e-8)
    got = init.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations <= 101
    _check_scalar_results(got, inp, 1e-3)


def _check_dual_results(sol, inp, tol_percent):
    # SolverTester::CheckDualResults (SolverTester.cc:409-439); BOOST_CHECK_CLOSE
    # is relative in percent.
    rel = tol_percent / 100.0
    for cb in range(sol.shape[0]):
        for p in range(2):
            s = sol[cb, :, :, p]
            t = inp[:, :, p]
            np.testing.assert_allclose(np.abs(s) ** 2, np.abs(t) ** 2, rtol=rel)
            np.testing.assert_allclose((s * np.conj(s[:1])).real,
                                       (t * np.conj(t[:1])).real, rtol=rel,
                                       atol=1e-12)


def _check_scalar_results(sol, inp, tol):
    # SolverTester::CheckScalarResults (SolverTester.cc:382-407)
    for cb in range(sol.shape[0]):
        s = sol[cb, :, :, 0]
        t = inp[:, :, 0]
        np.testing.assert_allclose(np.abs(s) ** 2, np.abs(t) ** 2,
                                   rtol=tol / 100.0)
        a = s * np.conj(s[:1])
        b = t * np.conj(t[:1])
        assert np.max(np.abs(a.real - b.real)) < tol
        assert np.max(np.abs(a.imag - b.imag)) < tol


def test_min_iterations(built):
    """tSolvers.cc min_iterations: accuracy 1e8 stops right at the minimum."""
    prob, inp, init = of.solver_tester_problem(False, False, 4)
    solver = H.make_solver(prob, max_iterations=100, accuracy=1e8,
                           min_iterations=10)
    got = init.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations == 10


def test_flagged_antenna_nan_repair(built):
    """An antenna whose visibilities are all zero (flagged by AssignAndWeight)
    gets den == 0 -> NaN, repaired by MakeSolutionsFinite2Pol, exactly as the
    oracle does."""
    obs = H.small_observation(n_stations=8, n_directions=2, n_channels=4,
                              n_cb=2, n_times=2, seed=9)
    prob = H.problem_from_observation(obs)
    for cb in range(len(prob["data"])):
        ap = prob["antenna_pairs"][cb]
        bad = (ap[:, 0] == 3) | (ap[:, 1] == 3)
        prob["data"][cb][bad] = 0
        prob["model"][cb][:, bad] = 0
    st = of.settings(max_iterations=20, accuracy=1e-5)
    sol0 = H.unit_solutions(prob)
    ref = sol0.copy()
    r, _ = of.solve(prob, ref, st, precision=64, n_threads=1)
    solver = H.make_solver(prob, max_iterations=20)
    got = sol0.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations == r.iterations
    np.testing.assert_allclose(got[:, 3], ref[:, 3], rtol=1e-6)
    ok = np.arange(8) != 3
    assert H.max_rel_diff(got[:, ok], ref[:, ok]) < RTOL_SOLVE


def test_phase_only(built):
    obs = H.small_observation(n_stations=8, n_directions=2, n_channels=4,
                              n_cb=2, n_times=2, seed=13)
    prob = H.problem_from_observation(obs)
    st = of.settings(max_iterations=30, accuracy=1e-5, phase_only=True)
    sol0 = H.unit_solutions(prob)
    ref = sol0.copy()
    r, _ = of.solve(prob, ref, st, precision=64, n_threads=1)
    solver = H.make_solver(prob, max_iterations=30, phase_only=True)
    got = sol0.copy()
    res = solver.Solve(H.solve_data_from_problem(prob), got, 0.0)
    assert res.iterations == r.iterations
    np.testing.assert_allclose(np.abs(got), 1.0, rtol=1e-12)
    assert H.max_rel_diff(got, ref) < RTOL_SOLVE


@pytest.mark.parametrize("n_dir", [7, 12, 23])
def test_many_directions_lane_groups(built, n_dir):
    """Direction counts that need several lanes per run (direction groups)."""
    obs = H.small_observation(n_stations=7, n_directions=n_dir, n_channels=4,
                              n_cb=2, n_times=2, seed=17, n_sources=2)
    prob = H.problem_from_observation(obs)
    sol0 = _perturbed_start(obs, prob, scale=0.2)
    ref = of.perform_iteration(prob, sol0, precision=64)
    for ng in (0, 1, 2, 4, 8):
        solver = H.make_solver(prob)
        solver.SetTuning(direction_groups=ng)
        try:
            got = solver.PerformIteration(obs.solve_data(), sol0)
        except RuntimeError as e:
            assert "unsupported" in str(e) or "too many" in str(e)
            continue
        err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
        assert np.nanmax(err) < RTOL_PASS, (ng, np.nanmax(err))


def test_irregular_layout_matches_regular(built):
    """A BDA-like irregular SolveData (visibilities dropped and runs of
    varying length, shuffled time order) through the generic entry point."""
    obs = H.small_observation(n_stations=9, n_directions=3, n_channels=12,
                              n_cb=2, n_times=4, seed=23, nspd=[1, 2, 4])
    prob = H.problem_from_observation(obs)
    rng = np.random.default_rng(1)
    for cb in range(len(prob["data"])):
        n = prob["data"][cb].shape[0]
        keep = np.sort(rng.choice(n, size=int(0.7 * n), replace=False))
        perm = keep
        prob["data"][cb] = np.ascontiguousarray(prob["data"][cb][perm])
        prob["model"][cb] = np.ascontiguousarray(prob["model"][cb][:, perm])
        prob["antenna_pairs"][cb] = np.ascontiguousarray(prob["antenna_pairs"][cb][perm])
        prob["solution_map"][cb] = np.ascontiguousarray(prob["solution_map"][cb][:, perm])
    sol0 = _perturbed_start(obs, prob, scale=0.2)
    ref = of.perform_iteration(prob, sol0, precision=64)
    solver = H.make_solver(prob)
    got = solver.PerformIteration(H.solve_data_from_problem(prob), sol0)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS


def test_slab_time_split_equivalence(built):
    """Folding several time steps into one slab or not gives the same pass."""
    obs = H.small_observation(n_stations=10, n_directions=2, n_channels=6,
                              n_cb=2, n_times=6, seed=29)
    prob = H.problem_from_observation(obs)
    sol0 = _perturbed_start(obs, prob, scale=0.2)
    outs = []
    for mt in (0, 1, 2, 4):
        solver = H.make_solver(prob)
        solver.SetTuning(max_slab_times=mt)
        outs.append(solver.PerformIteration(obs.solve_data(), sol0))
    for o in outs[1:]:
        np.testing.assert_allclose(o, outs[0], rtol=1e-5)


def test_scale_invariance_full_size_c1(built):
    """Size-independent property at the full c1 size: scaling data and model
    by alpha leaves next_solutions unchanged; also checks one full-size pass
    against the FP64 oracle."""
    cfg = synth.benchmark_configs()[1]
    obs = synth.observe(cfg)
    prob = H.problem_from_observation(obs)
    sol0 = _perturbed_start(obs, prob, scale=0.1)
    solver = H.make_solver(prob)
    got = solver.PerformIteration(obs.solve_data(), sol0)
    ref = of.perform_iteration(prob, sol0, precision=64)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS
    alpha = np.float32(3.0)
    sd = obs.solve_data()
    for b in sd.channel_blocks:
        b.data = b.data * alpha
        b.model = b.model * alpha
    got2 = solver.PerformIteration(sd, sol0)
    np.testing.assert_allclose(got2, got, rtol=1e-5)


@pytest.mark.parametrize("npol", [2, 1])
def test_full_size_large_array_pass(built, npol):
    """The 512-station configuration at full size (130816 baselines, 5
    directions, 64 channels in 16 blocks, 2 timesteps, 16.7 M visibilities):
    one pass of the diagonal (npol 2) and of the scalar (npol 1) solver
    against the FP64 oracle."""
    cfg = synth.benchmark_configs()[3]
    obs = synth.observe(cfg)
    prob = H.problem_from_observation(obs, 2, npol)
    sol0 = _perturbed_start(obs, prob, scale=0.1)
    solver = H.make_solver(prob)
    got = solver.PerformIteration(obs.solve_data(), sol0)
    ref = of.perform_iteration(prob, sol0, precision=64)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))


def test_full_size_dd_interval_configuration(built):
    """One interval of the 40-direction configuration at full size (62
    stations, 40 directions with 8, 4, 2 or 1 solutions per 8-timestep
    interval, 120 channels in uneven blocks of 3-12 channels): one pass
    against the FP64 oracle, then a 10-iteration solve against the oracle
    with the reference's FP32 arithmetic."""
    cfg = synth.benchmark_configs()[2]
    obs = synth.observe(cfg)
    prob = H.problem_from_observation(obs)
    sol0 = _perturbed_start(obs, prob, scale=0.1)
    solver = H.make_solver(prob, max_iterations=10, accuracy=cfg.tolerance)
    got = solver.PerformIteration(obs.solve_data(), sol0)
    ref = of.perform_iteration(prob, sol0, precision=64)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)
    st = of.settings(max_iterations=10, accuracy=cfg.tolerance, step_size=cfg.step_size)
    ref32 = sol0.copy()
    r, _ = of.solve(prob, ref32, st, precision=32)
    got_s = sol0.copy()
    res = solver.Solve(obs.solve_data(), got_s, 0.0)
    assert res.iterations == r.iterations
    assert H.max_rel_diff(got_s, ref32) < RTOL_SOLVE


def test_autotune_keeps_results_and_caches(built):
    """The autotuner picks a plan variant whose pass equals the default one
    within the pass tolerance, and a second context of the same shape takes
    the cached choice."""
    from dp3_b200 import ddsolve
    import time
    obs = H.small_observation(n_stations=20, n_directions=5, n_channels=16, n_cb=4,
                              n_times=4, seed=13)
    cfg = obs.cfg
    prob = H.problem_from_observation(obs)
    sol0 = _perturbed_start(obs, prob, scale=0.1)

    def make():
        ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
        for cb, nc in enumerate(cfg.cb_channels):
            ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                          obs.model[cb], obs.antenna1, obs.antenna2)
        return ctx

    ctx = make()
    expect = ctx.perform_iteration(sol0)
    choice, ms = ctx.autotune(3)
    assert ms > 0
    assert ctx.tuning() == choice
    got = ctx.perform_iteration(sol0)
    err = np.abs(got - expect) / np.maximum(np.abs(expect), 1e-12)
    assert np.nanmax(err) < RTOL_PASS
    ctx.close()
    ctx2 = make()
    t0 = time.perf_counter()
    choice2, ms2 = ctx2.autotune(3)
    assert choice2 == choice and ms2 == ms
    ctx2.close()
    # every explicit variant gives the same pass
    for t in ({"use_pipe": 0, "direction_groups": 2}, {"use_pipe": 1, "model_powers": 1,
              "gain_buffers": 1, "stages": 3}, {"use_pipe": 1, "model_powers": 0}):
        c = make()
        c.set_plan_tuning(**t)
        got = c.perform_iteration(sol0)
        err = np.abs(got - expect) / np.maximum(np.abs(expect), 1e-12)
        assert np.nanmax(err) < RTOL_PASS, t
        c.close()


@pytest.mark.parametrize("use_pipe", [-1, 0])
def test_batched_intervals_match_separate_solves(built, use_pipe):
    """Three independent intervals in one context (ddsolve_set_intervals /
    ddsolve_solve_batch) give each interval the iteration count and the
    solutions of its own solve: intervals stop at different iterations and a
    stopped interval keeps its solutions while the others go on. Default plan
    (pipe_kernel, per-interval control in its fused finalisation) and the
    stream_kernel plan."""
    from dp3_b200 import ddsolve
    obs_list = [synth.observe(synth.small_config(n_stations=12, n_directions=3, n_channels=8,
                                                 n_cb=2, n_times=2, seed=seed))
                for seed in (21, 22, 23)]
    cfg = obs_list[0].cfg
    n_sub = sum(cfg.nspd)
    st = ddsolve.default_settings()
    st.max_iterations, st.accuracy, st.step_size = 150, 1e-5, 0.2
    singles = []
    for obs in obs_list:
        ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
        ctx.set_settings(st)
        for cb, nc in enumerate(cfg.cb_channels):
            ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                          obs.model[cb], obs.antenna1, obs.antenna2)
        sol = np.ones((cfg.n_channel_blocks, cfg.n_stations, n_sub, 2), np.complex128)
        mags = np.zeros(150)
        r = ctx.solve(sol, mags)
        singles.append((r, sol, mags))
        ctx.close()
    n_cb = cfg.n_channel_blocks
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, 3 * n_cb, 2, 2)
    ctx.set_settings(st)
    ctx.set_intervals([0, n_cb, 2 * n_cb, 3 * n_cb])
    ctx.set_plan_tuning(use_pipe=use_pipe)
    for g, obs in enumerate(obs_list):
        for cb, nc in enumerate(cfg.cb_channels):
            ctx.set_channel_block_regular(g * n_cb + cb, cfg.n_times, cfg.n_baselines, nc,
                                          obs.data[cb], obs.model[cb], obs.antenna1,
                                          obs.antenna2)
    sol = np.ones((3 * n_cb, cfg.n_stations, n_sub, 2), np.complex128)
    mags = np.zeros((3, 150))
    res = ctx.solve_batch(sol, mags)
    # which path ran: one pipe_kernel per iteration (plus make-finite, gain
    # tables and model powers once per solve), or three kernels per iteration
    max_it = max(r.iterations for r in res)
    if use_pipe == -1:
        assert ctx.last_launch_count() <= max_it + 3, (ctx.last_launch_count(), max_it)
    else:
        assert ctx.last_launch_count() >= 3 * (max_it - 1), (ctx.last_launch_count(), max_it)
    with pytest.raises(RuntimeError):
        ctx.solve(np.ones_like(sol))
    ctx.close()
    its = [r.iterations for r, _, _ in singles]
    assert len(set(its)) > 1, its  # the intervals stop at different iterations
    for g, (r, s1, m1) in enumerate(singles):
        assert res[g].iterations == r.iterations
        assert res[g].has_converged == r.has_converged
        assert H.max_rel_diff(sol[g * n_cb:(g + 1) * n_cb], s1) < RTOL_SOLVE
        n = min(r.iterations, 150)
        np.testing.assert_allclose(mags[g, :n], m1[:n], rtol=1e-3, atol=1e-12)


@pytest.mark.parametrize("n_dir,npol", [(13, 2), (16, 1), (40, 2)])
def test_lane_group_pipe_kernel(built, n_dir, npol):
    """More directions than one lane holds: pipe_kernel with four lanes per
    run (the residual summed across the run's lanes), against the FP64
    oracle for one pass and the FP32 oracle for a 20-iteration solve, and
    against the stream_kernel path."""
    obs = H.small_observation(n_stations=30, n_directions=n_dir, n_channels=8, n_cb=2,
                              n_times=2, seed=31 + n_dir, n_sources=2)
    prob = H.problem_from_observation(obs, 2, npol)
    sol0 = _perturbed_start(obs, prob, scale=0.1)
    solver = H.make_solver(prob, max_iterations=20)
    got = solver.PerformIteration(obs.solve_data(), sol0)
    assert solver._ctx.tuning()["use_pipe"] == -1
    ref = of.perform_iteration(prob, sol0, precision=64)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12)
    assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)
    v1 = H.make_solver(prob, max_iterations=20)
    v1.SetTuning(direction_groups=4)
    got_v1 = v1.PerformIteration(obs.solve_data(), sol0)
    np.testing.assert_allclose(got, got_v1, rtol=1e-4)
    st = of.settings(max_iterations=20, accuracy=1e-5, step_size=0.2)
    ref32 = sol0.copy()
    r, _ = of.solve(prob, ref32, st, precision=32)
    g = sol0.copy()
    res = solver.Solve(obs.solve_data(), g, 0.0)
    assert res.iterations == r.iterations
    assert H.max_rel_diff(g, ref32) < RTOL_SOLVE
