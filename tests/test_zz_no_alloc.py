"""GPU test of the allocation-free entry point
ddsolve_perform_iteration_noalloc (include/ddsolve_b200.h).

That entry point serves callers that cannot let a library allocate device
memory (graph capture in progress, caller-owned memory pools, fixed device
memory budgets): it keeps its accumulators in a static array inside the
library. Here the caller's device buffers are made with torch, and two calls
in a row are compared with the context-based ddsolve_perform_iteration on the
same inputs, within the pass tolerance of the parity suite (1e-4 relative).
This file is collected last so that a failure here leaves every other test
already run; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from dp3_b200 import ddsolve
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


@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (2, 1)])
def test_noalloc_matches_context_entry_point(built, ncorr, npol):
    import torch
    obs = H.small_observation(n_stations=9, n_directions=3, n_channels=12,
                              n_cb=3, n_times=4, nspd=[2, 1, 2], seed=51)
    cfg = obs.cfg
    prob = H.problem_from_observation(obs, ncorr, npol, leakage=0.05)
    n_sub = sum(cfg.nspd)
    rng = np.random.default_rng(7)
    shape = (cfg.n_channel_blocks, cfg.n_stations, n_sub, npol)
    starts = [np.ones(shape, np.complex128),
              (1 + 0.3 * (rng.standard_normal(shape)
                          + 1j * rng.standard_normal(shape)))]

    # Existing entry point (context, host buffers).
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks,
                          ncorr, npol)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc,
                                      prob["data"][cb], prob["model"][cb],
                                      obs.antenna1, obs.antenna2)
    expected = [ctx.perform_iteration(s) for s in starts]
    ctx.close()

    # Caller-owned device buffers.
    dev = torch.device("cuda:0")
    data = torch.from_numpy(np.concatenate([d.reshape(-1) for d in prob["data"]])).to(dev)
    model = torch.from_numpy(np.concatenate([m.reshape(-1) for m in prob["model"]])).to(dev)
    a1 = torch.from_numpy(obs.antenna1.view(np.int32)).to(dev)
    a2 = torch.from_numpy(obs.antenna2.view(np.int32)).to(dev)
    sol = torch.empty(int(np.prod(shape)) * 2, dtype=torch.float64, device=dev)
    nxt = torch.empty_like(sol)
    dims, keep = _dims(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, ncorr, npol)
    cbc = (ctypes.c_uint32 * cfg.n_channel_blocks)(*cfg.cb_channels)
    fn = _noalloc_fn()
    stream = torch.cuda.current_stream(dev)
    for start, exp in zip(starts, expected):  # two calls in a row
        sol.copy_(torch.from_numpy(start.view(np.float64).reshape(-1)))
        nxt.fill_(0.0)
        rc = fn(ctypes.byref(dims), cfg.n_times, cfg.n_baselines, cbc,
                data.data_ptr(), model.data_ptr(), a1.data_ptr(), a2.data_ptr(),
                sol.data_ptr(), nxt.data_ptr(), stream.cuda_stream)
        assert rc == 0, ddsolve.lib().ddsolve_last_error(None)
        torch.cuda.synchronize()
        got = nxt.cpu().numpy().view(np.complex128).reshape(shape)
        err = np.abs(got - exp) / np.maximum(np.abs(exp), 1e-12)
        assert np.nanmax(err) < RTOL_PASS, np.nanmax(err)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(exp))


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
