"""Tests of the DP3 adapter (dp3_b200/dp3/IterativeSolverB200.h), a C++
dp3::ddecal::SolverBase subclass that calls libddsolve_b200.so.

The harness (tests/adapter/, built from the reference tree) packs one regular
interval through DP3's own SolveData constructor and solves it with DP3's own
IterativeDiagonalSolver / IterativeScalarSolver or with the adapter, both set
up through DP3's SolverBase the way DDECal's SolverFactory does: the setters,
and DP3's AntennaConstraint / SmoothnessConstraint, which the adapter applies
through DP3's own SolverBase::ApplyConstraints between device passes.

CPU: the library loads and DP3's own path through the harness reproduces the
reference-code oracle bit for bit. GPU: the adapter against DP3's own solver
on the same inputs: identical iteration counts and <= 1e-4 relative after
phase referencing to antenna 0 (the parity tolerance), with and without
constraints, including a solve that DP3's stall detection stops.
"""
import ctypes
import multiprocessing
import os
import subprocess
from concurrent.futures import ProcessPoolExecutor
from concurrent.futures.process import BrokenProcessPool

import numpy as np
import pytest

from dp3_b200 import synth
from oracle import ref_ffi as rf
from tests import helpers as H

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "adapter", "_build", "libdp3_adapter_check.so")

pytestmark = pytest.mark.skipif(
    not (os.path.exists(LIB) or os.path.isdir(rf.REFERENCE)),
    reason="adapter harness not built and the reference tree is absent")

RTOL = 1e-4

_lib = None


def build():
    if os.path.isdir(rf.REFERENCE):
        subprocess.check_call(["make", "-C", os.path.join(HERE, "adapter"),
                               f"REF={rf.REFERENCE}"], stdout=subprocess.DEVNULL)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        L.adapter_solve.restype = ctypes.c_int
        L.adapter_solve.argtypes = [
            ctypes.POINTER(rf.Problem), ctypes.POINTER(rf.Settings), ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(rf.Constraints), ctypes.c_void_p,
            ctypes.POINTER(rf.Result), ctypes.c_void_p, ctypes.c_uint32]
        L.adapter_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def run(obs, prob, sol, st, use_b200, n_threads=1, antenna_sets=None, smoothness=None):
    """Solves `prob` (regular layout of `obs`) in place; returns (Result,
    step magnitudes from the adapter's statistics stream). The adapter runs
    in a child process (the GPU path of native code: a crash there fails the
    test instead of ending the test session)."""
    if not use_b200:
        return _run_here(obs, prob, sol, st, use_b200, n_threads, antenna_sets, smoothness)
    fields = tuple(getattr(st, f) for f, _ in rf.Settings._fields_)
    try:
        its, c_its, mags, out = _pool().submit(
            _run_child, obs, prob, sol, fields, int(use_b200), n_threads, antenna_sets,
            smoothness).result()
    except BrokenProcessPool:
        global _POOL
        _POOL = None
        raise RuntimeError("the adapter's child process crashed (see its stderr)")
    sol[...] = out
    res = rf.Result()
    res.iterations, res.constraint_iterations = its, c_its
    return res, mags


_POOL = None


def _pool():
    global _POOL
    if _POOL is None:
        _POOL = ProcessPoolExecutor(max_workers=1, mp_context=multiprocessing.get_context("spawn"))
    return _POOL


def _run_child(obs, prob, sol, fields, use_b200, n_threads, antenna_sets, smoothness):
    res, mags = _run_here(obs, prob, sol, rf.Settings(*fields), use_b200, n_threads,
                          antenna_sets, smoothness)
    return res.iterations, res.constraint_iterations, mags, sol


def _run_here(obs, prob, sol, st, use_b200, n_threads=1, antenna_sets=None, smoothness=None):
    cfg = obs.cfg
    n_cb = len(cfg.cb_channels)
    nspd = np.ascontiguousarray(cfg.nspd, np.uint32)
    a1 = np.ascontiguousarray(obs.antenna1, np.int32)
    a2 = np.ascontiguousarray(obs.antenna2, np.int32)
    data = [np.ascontiguousarray(d, np.float32) for d in prob["data"]]
    model = [np.ascontiguousarray(m, np.float32) for m in prob["model"]]
    dp = (ctypes.c_void_p * n_cb)(*[d.ctypes.data for d in data])
    mp = (ctypes.c_void_p * n_cb)(*[m.ctypes.data for m in model])
    p = rf.Problem(cfg.n_stations, cfg.n_times, cfg.n_baselines, sum(cfg.cb_channels), n_cb,
                   len(nspd), prob["n_correlations"],
                   nspd.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                   a1.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                   a2.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                   ctypes.cast(dp, ctypes.POINTER(ctypes.c_void_p)),
                   ctypes.cast(mp, ctypes.POINTER(ctypes.c_void_p)))
    keep = []
    cons = None
    if antenna_sets or smoothness:
        freqs = np.array([synth.frequencies(cfg)[lo:lo + n].mean() for lo, n in
                          zip(np.cumsum([0] + list(cfg.cb_channels))[:-1], cfg.cb_channels)])
        keep.append(freqs)
        cons = rf.Constraints()
        cons.channel_block_frequencies = freqs.ctypes.data
        if antenna_sets:
            sizes = np.array([len(s) for s in antenna_sets], np.uint32)
            members = np.concatenate([np.asarray(s, np.uint32) for s in antenna_sets])
            keep += [sizes, members]
            cons.n_antenna_sets = len(antenna_sets)
            cons.antenna_set_sizes = sizes.ctypes.data
            cons.antenna_set_members = members.ctypes.data
        if smoothness:
            cons.smoothness = 1
            cons.bandwidth_hz = smoothness
            cons.spectral_exponent = -1.0
            cons.kernel_truncation = 1
    mags = np.full(max(st.max_iterations, 1), np.nan)
    res = rf.Result()
    rc = lib().adapter_solve(ctypes.byref(p), ctypes.byref(st), rf.kind_of(
        prob["n_correlations"], prob["n_pol"]), int(use_b200), 0, n_threads,
        ctypes.byref(cons) if cons is not None else None, sol.ctypes.data, ctypes.byref(res),
        mags.ctypes.data, len(mags))
    if rc != 0:
        raise RuntimeError(lib().adapter_last_error().decode())
    return res, mags


def _small(ncorr, npol, seed=21, nspd=None, n_stations=10):
    obs = H.small_observation(n_stations=n_stations, n_directions=3, n_channels=8, n_cb=2,
                              n_times=4, nspd=nspd, seed=seed)
    return obs, H.problem_from_observation(obs, ncorr, npol, leakage=0.02)


def test_dp3_path_of_harness_matches_reference_oracle(built):
    """DP3's own solver through this harness == the reference-code oracle
    (the same compiled code and inputs): the harness packs and configures
    exactly as the oracle does. CPU only."""
    obs, prob = _small(2, 2)
    st = rf.settings(max_iterations=60, accuracy=1e-5)
    a = H.perturbed_start(obs, prob, scale=0.05)
    b = a.copy()
    ra, _ = run(obs, prob, a, st, use_b200=False)
    rb = rf.solve(obs.cfg, obs.antenna1, obs.antenna2, prob["data"], prob["model"], 2, 2, b, st)
    assert ra.iterations == rb.iterations
    np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (1, 1), (2, 1), (4, 1)])
@pytest.mark.parametrize("case", ["plain", "dd", "phase_only"])
def test_adapter_matches_dp3_solver(built, ncorr, npol, case):
    obs, prob = _small(ncorr, npol, nspd=[2, 1, 2] if case == "dd" else None)
    st = rf.settings(max_iterations=60, accuracy=1e-5, phase_only=case == "phase_only")
    start = H.perturbed_start(obs, prob, scale=0.05)
    if case == "phase_only":
        start = start / np.abs(start)
    a, b = start.copy(), start.copy()
    rd, _ = run(obs, prob, a, st, use_b200=False)
    rg, mags = run(obs, prob, b, st, use_b200=True)
    assert rg.iterations == rd.iterations
    assert H.max_rel_diff(b, a) < RTOL
    n_it = rg.iterations if rg.iterations <= st.max_iterations else st.max_iterations
    assert np.all(np.isfinite(mags[:n_it])) and np.all(np.isnan(mags[n_it:]))


@pytest.mark.gpu
def test_adapter_benchmark_c0(built):
    cfg = synth.benchmark_configs()[0]
    obs = synth.observe(cfg)
    prob = H.problem_from_observation(obs)
    st = rf.settings(max_iterations=cfg.max_iterations, accuracy=cfg.tolerance,
                     step_size=cfg.step_size)
    a, b = H.unit_solutions(prob), H.unit_solutions(prob)
    rd, _ = run(obs, prob, a, st, use_b200=False, n_threads=4)
    rg, _ = run(obs, prob, b, st, use_b200=True)
    assert rg.iterations == rd.iterations
    assert H.max_rel_diff(b, a) < RTOL


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (2, 1)])
@pytest.mark.parametrize("constraint", ["antenna", "smoothness", "both"])
@pytest.mark.parametrize("mode", [1, 2])
def test_adapter_with_dp3_constraints(built, ncorr, npol, constraint, mode):
    """DP3's AntennaConstraint (core antennas 0-3 share one solution) and
    SmoothnessConstraint (Gaussian kernel of 10 MHz over the channel
    blocks). Mode 1: DP3's constraint classes, applied by DP3's own
    SolverBase::ApplyConstraints between the adapter's device passes (the
    smoothness constraint keeps the loop on the host). Mode 2: the adapter's
    SmoothnessConstraintB200 in place of DP3's: every constraint has a
    device form and the whole constrained loop runs on the device."""
    obs = H.small_observation(n_stations=10, n_directions=3, n_channels=16, n_cb=8,
                              n_times=4, seed=23)
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.02)
    sets = [[0, 1, 2, 3]] if constraint in ("antenna", "both") else None
    smooth = 10e6 if constraint in ("smoothness", "both") else None
    st = rf.settings(max_iterations=80, accuracy=1e-5)
    start = H.perturbed_start(obs, prob, scale=0.05)
    a, b = start.copy(), start.copy()
    rd, _ = run(obs, prob, a, st, use_b200=False, antenna_sets=sets, smoothness=smooth)
    rg, _ = run(obs, prob, b, st, use_b200=mode, antenna_sets=sets, smoothness=smooth)
    assert rg.iterations == rd.iterations
    assert rg.constraint_iterations == rd.constraint_iterations
    assert H.max_rel_diff(b, a) < RTOL
    if sets:  # the constraint holds in the adapter's answer
        np.testing.assert_allclose(b[:, 1:4], np.repeat(b[:, :1], 3, axis=1), rtol=1e-12)


@pytest.mark.gpu
def test_adapter_stall_matches_dp3(built):
    """An accuracy FP32 cannot reach: DP3's DetectStall stops DP3's solver;
    the adapter evaluates DP3's own stopping rule over the device's step
    magnitudes and stops at the same iteration."""
    obs = H.small_observation(n_stations=10, n_directions=3, n_channels=8, n_cb=2,
                              n_times=3, seed=21)
    prob = H.problem_from_observation(obs)
    st = rf.settings(max_iterations=3000, accuracy=1e-14, step_size=0.5)
    a, b = H.unit_solutions(prob), H.unit_solutions(prob)
    rd, _ = run(obs, prob, a, st, use_b200=False)
    rg, _ = run(obs, prob, b, st, use_b200=True)
    assert rd.iterations < 3000
    assert rg.iterations == rd.iterations
    assert H.max_rel_diff(b, a) < RTOL


def _correct_subtract_child(n_pol, n_ant, n_cb, a1, a2, sol, data, model, subtract, keep):
    L = lib()
    L.adapter_correct_and_subtract.restype = ctypes.c_int
    u32 = ctypes.c_uint32
    n_dir, n_t, n_bl, n_ch, _ = model.shape
    data, model = data.copy(), model.copy()
    rc = L.adapter_correct_and_subtract(
        ctypes.c_int(n_pol), ctypes.c_int(0), u32(n_ant), u32(n_dir), u32(n_cb), u32(n_t),
        u32(n_bl), u32(n_ch), ctypes.c_void_p(a1.ctypes.data), ctypes.c_void_p(a2.ctypes.data),
        ctypes.c_void_p(sol.ctypes.data), ctypes.c_void_p(data.ctypes.data),
        ctypes.c_void_p(model.ctypes.data), ctypes.c_int(int(subtract)), ctypes.c_int(int(keep)))
    if rc != 0:
        raise RuntimeError(L.adapter_last_error().decode())
    return data, model


@pytest.mark.gpu
@pytest.mark.parametrize("n_pol", [1, 2, 4])
def test_adapter_correct_and_subtract(built, n_pol):
    """The adapter's CorrectAndSubtract (DDECal::CorrectAndSubtractModels on
    the GPU, one call per time step as DDECal holds its buffers) equals the
    restated step (oracle/subtract_oracle.py) bit for bit, data and kept
    models."""
    from oracle import subtract_oracle as so
    rng = np.random.default_rng(n_pol)
    n_st, n_t, n_ch, n_dir, n_cb = 7, 3, 10, 3, 3
    a1, a2 = (x.astype(np.uint32) for x in np.triu_indices(n_st, 0))
    cz = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s))  # noqa: E731
    data = cz(n_t, len(a1), n_ch, 4).astype(np.complex64)
    model = cz(n_dir, n_t, len(a1), n_ch, 4).astype(np.complex64)
    sol = np.ascontiguousarray(1.0 + 0.3 * cz(n_cb, n_st, n_dir, n_pol))
    try:
        got_d, got_m = _pool().submit(_correct_subtract_child, n_pol, n_st, n_cb, a1, a2, sol,
                                      data, model, True, True).result()
    except BrokenProcessPool:
        global _POOL
        _POOL = None
        raise RuntimeError("the adapter's child process crashed (see its stderr)")
    want_d, want_m = so.correct_and_subtract(data, model, sol, a1, a2, True, True)
    np.testing.assert_array_equal(got_d.view(np.uint32), want_d.view(np.uint32))
    np.testing.assert_array_equal(got_m.view(np.uint32), want_m.view(np.uint32))
