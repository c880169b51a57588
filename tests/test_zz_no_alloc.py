"""GPU test of the allocation-free entry point
ddsolve_perform_iteration_noalloc (include/ddsolve_b200.h).

That entry point serves callers that cannot let a library allocate device
memory (frameworks whose device memory all comes from their own pool,
processes with a fixed device budget): it keeps its accumulators in a static
array inside the library. Here the caller's device buffers are made with
torch. Two calls in a row are compared with the context-based
ddsolve_perform_iteration on the same inputs and with the FP64 oracle's
PerformIteration, within the pass tolerance of the parity suite (1e-4
relative per element). One case adds an autocorrelation baseline, which the
reference's SolveData drops (SolveData.cc:100,137), so the oracle never sees
it; one case gives a direction more solutions than the interval has time
steps, which SolveData limits to the number of time steps
(SolveData.cc:56-68,104-105).
This file is collected last so that a failure here leaves every other test
already run; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from dp3_b200 import ddsolve
from oracle import oracle_ffi as of
from tests import helpers as H

pytestmark = pytest.mark.gpu

RTOL_PASS = 1e-4


def _noalloc_fn():
    lib = ddsolve.lib()
    fn = lib.ddsolve_perform_iteration_noalloc
    vp = ctypes.c_void_p
    fn.argtypes = [ctypes.POINTER(ddsolve.Dims), ctypes.c_uint32, ctypes.c_uint32,
                   ctypes.POINTER(ctypes.c_uint32), vp, vp, vp, vp, vp, vp, vp]
    fn.restype = ctypes.c_int
    return fn


def _dims(n_ant, nspd, n_cb, ncorr, npol):
    arr = (ctypes.c_uint32 * len(nspd))(*nspd)
    return ddsolve.Dims(n_ant, len(nspd), n_cb, ncorr, npol,
                        ctypes.cast(arr, ctypes.POINTER(ctypes.c_uint32))), arr


def _with_autocorrelation(obs, prob, ncorr, seed=5):
    """Regular-layout inputs with one extra baseline (antenna 2, antenna 2)
    appended to every time step, with random data and model."""
    cfg = obs.cfg
    rng = np.random.default_rng(seed)
    data, model = [], []
    for cb, nc in enumerate(cfg.cb_channels):
        d = prob["data"][cb].reshape(cfg.n_times, cfg.n_baselines, nc, ncorr, 2)
        extra = rng.standard_normal((cfg.n_times, 1, nc, ncorr, 2)).astype(np.float32)
        data.append(np.concatenate([d, extra], axis=1).reshape(-1))
        m = prob["model"][cb].reshape(cfg.n_directions, cfg.n_times, cfg.n_baselines,
                                      nc, ncorr, 2)
        extra = rng.standard_normal((cfg.n_directions, cfg.n_times, 1, nc, ncorr,
                                     2)).astype(np.float32)
        model.append(np.concatenate([m, extra], axis=2).reshape(-1))
    a1 = np.append(obs.antenna1, np.uint32(2))
    a2 = np.append(obs.antenna2, np.uint32(2))
    return data, model, a1, a2, cfg.n_baselines + 1


@pytest.mark.parametrize("case", ["plain", "autocorrelation", "dd_beyond_times"])
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (2, 1), (4, 1), (1, 1)])
def test_noalloc_matches_context_and_oracle(built, ncorr, npol, case):
    import torch
    # dd_beyond_times: direction 2 asks for 6 solutions over 4 time steps;
    # SolveData limits it to 4, so sub-solutions 7 and 8 stay unused.
    nspd = [2, 1, 6] if case == "dd_beyond_times" else [2, 1, 2]
    obs = H.small_observation(n_stations=9, n_directions=3, n_channels=12,
                              n_cb=3, n_times=4, nspd=nspd, seed=51)
    cfg = obs.cfg
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.05)
    n_sub = sum(cfg.nspd)
    n_used = int(np.minimum(cfg.nspd, cfg.n_times).sum())
    shape = (cfg.n_channel_blocks, cfg.n_stations, n_sub, npol)
    starts = [H.perturbed_start(obs, prob, scale=0.3, seed=3),
              H.perturbed_start(obs, prob, scale=0.1, seed=4)]

    # Existing entry point (context, host buffers) and the FP64 oracle.
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks,
                          ncorr, npol)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc,
                                      prob["data"][cb], prob["model"][cb],
                                      obs.antenna1, obs.antenna2)
    expected = [ctx.perform_iteration(s) for s in starts]
    ctx.close()
    oracle = [of.perform_iteration(prob, s, precision=64) for s in starts]

    # Caller-owned device buffers.
    if case == "autocorrelation":
        data_l, model_l, a1_np, a2_np, n_bl = _with_autocorrelation(obs, prob, ncorr)
    else:
        data_l = [d.reshape(-1) for d in prob["data"]]
        model_l = [m.reshape(-1) for m in prob["model"]]
        a1_np, a2_np, n_bl = obs.antenna1, obs.antenna2, cfg.n_baselines
    dev = torch.device("cuda:0")
    data = torch.from_numpy(np.concatenate(data_l)).to(dev)
    model = torch.from_numpy(np.concatenate(model_l)).to(dev)
    a1 = torch.from_numpy(a1_np.view(np.int32)).to(dev)
    a2 = torch.from_numpy(a2_np.view(np.int32)).to(dev)
    sol = torch.empty(int(np.prod(shape)) * 2, dtype=torch.float64, device=dev)
    nxt = torch.empty_like(sol)
    dims, keep = _dims(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, ncorr, npol)
    cbc = (ctypes.c_uint32 * cfg.n_channel_blocks)(*cfg.cb_channels)
    fn = _noalloc_fn()
    stream = torch.cuda.current_stream(dev)
    for start, exp, ref in zip(starts, expected, oracle):  # two calls in a row
        sol.copy_(torch.from_numpy(start.view(np.float64).reshape(-1)))
        nxt.fill_(0.0)
        rc = fn(ctypes.byref(dims), cfg.n_times, n_bl, cbc,
                data.data_ptr(), model.data_ptr(), a1.data_ptr(), a2.data_ptr(),
                sol.data_ptr(), nxt.data_ptr(), stream.cuda_stream)
        assert rc == 0, ddsolve.lib().ddsolve_last_error(None)
        torch.cuda.synchronize()
        got = nxt.cpu().numpy().view(np.complex128).reshape(shape)[:, :, :n_used]
        for want in (exp[:, :, :n_used], ref[:, :, :n_used]):
            np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
            err = np.abs(got - want) / np.maximum(np.abs(want), 1e-12)
            assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)


def test_noalloc_rejects_sizes_beyond_limits(built):
    fn = _noalloc_fn()
    dims, keep = _dims(10, [1, 1], 2, 2, 2)
    dummy = ctypes.c_void_p(16)  # never dereferenced: rejected before launch
    cbc = (ctypes.c_uint32 * 2)(17, 4)  # 17 channels in a block
    rc = fn(ctypes.byref(dims), 2, 45, cbc, dummy, dummy, dummy, dummy, dummy,
            dummy, None)
    assert rc == 4
    assert b"channels per block" in ddsolve.lib().ddsolve_last_error(None)
    big, keep2 = _dims(60000, [8] * 40, 2, 2, 2)  # accumulators > 1 Mi floats
    cbc = (ctypes.c_uint32 * 2)(4, 4)
    rc = fn(ctypes.byref(big), 2, 45, cbc, dummy, dummy, dummy, dummy, dummy,
            dummy, None)
    assert rc == 4
    assert b"exceeds the static scratch" in ddsolve.lib().ddsolve_last_error(None)
    rc = fn(ctypes.byref(dims), 70000, 45, cbc, dummy, dummy, dummy, dummy, dummy,
            dummy, None)  # time steps beyond the launch grid's y limit
    assert rc == 4
    assert b"65535 time steps" in ddsolve.lib().ddsolve_last_error(None)
