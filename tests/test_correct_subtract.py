"""Tests of ddsolve_correct_and_subtract (include/ddsolve_b200.h): DDECal's
CorrectAndSubtractModels (steps/DDECal.cc:1004-1125), the step after the
solve, on the GPU.

CPU: the restated oracle (oracle/subtract_oracle.py) against a plain
complex128 matrix evaluation of G_1 M G_2^H, and its channel-block map.
GPU: for 1, 2 and 4 solution polarizations, with and without kept models,
host and device buffers, with autocorrelations: the GPU outputs equal the
oracle's bit for bit (both round every FP64 product and sum separately and
the float outputs once); with the model predicted on the GPU from the sky,
within 1e-5 of the oracle applied to the predict oracle's model (the models
differ by complex64 roundings). Direction-dependent intervals are refused,
as the reference throws.
"""
import ctypes

import numpy as np
import pytest

from dp3_b200 import ddsolve, synth
from oracle import predict_oracle as po
from oracle import subtract_oracle as so


def _interval(n_st=6, n_t=2, n_ch=7, n_dir=3, n_cb=2, npol=2, seed=0):
    rng = np.random.default_rng(seed)
    a1, a2 = np.triu_indices(n_st, 0)  # autocorrelations included
    n_bl = len(a1)
    cz = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s))  # noqa: E731
    data = cz(n_t, n_bl, n_ch, 4).astype(np.complex64)
    model = cz(n_dir, n_t, n_bl, n_ch, 4).astype(np.complex64)
    sol = 1.0 + 0.3 * cz(n_cb, n_st, n_dir, npol)
    return a1.astype(np.uint32), a2.astype(np.uint32), data, model, sol


def _naive(data, model, sol, a1, a2):
    n_dir, n_t, n_bl, n_ch, _ = model.shape
    npol = sol.shape[-1]
    cb = so.channel_block_of_channel(n_ch, sol.shape[0])
    out = data.astype(np.complex128)
    kept = np.zeros(model.shape, np.complex128)
    for d in range(n_dir):
        for b in range(n_bl):
            for c in range(n_ch):
                g1, g2 = sol[cb[c], a1[b], d], sol[cb[c], a2[b], d]
                m = model[d, :, b, c].astype(np.complex128).reshape(n_t, 2, 2)
                if npol == 4:
                    cm = g1.reshape(2, 2) @ m @ g2.reshape(2, 2).conj().T
                elif npol == 2:
                    cm = np.diag(g1) @ m @ np.diag(g2).conj()
                else:
                    cm = m * (g1[0] * np.conj(g2[0]))
                kept[d, :, b, c] = cm.reshape(n_t, 4)
                out[:, b, c] -= cm.reshape(n_t, 4)
    return out, kept


def test_channel_block_map_is_the_even_split():
    cb = so.channel_block_of_channel(10, 3)
    assert list(cb) == [0, 0, 0, 1, 1, 1, 2, 2, 2, 2]
    for n_ch, n_cb in [(7, 2), (120, 12), (13, 13), (240, 24)]:
        cb = so.channel_block_of_channel(n_ch, n_cb)
        for c in range(n_cb):
            assert np.all(cb[c * n_ch // n_cb:(c + 1) * n_ch // n_cb] == c)


@pytest.mark.parametrize("npol", [1, 2, 4])
def test_oracle_matches_matrix_products(npol):
    a1, a2, data, model, sol = _interval(npol=npol)
    out, kept = so.correct_and_subtract(data, model, sol, a1, a2, True, True)
    want_out, want_kept = _naive(data, model, sol, a1, a2)
    np.testing.assert_allclose(kept, want_kept, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(out, want_out, rtol=1e-6, atol=1e-5)
    out2, none = so.correct_and_subtract(data, model, sol, a1, a2, True, False)
    assert none is None
    np.testing.assert_array_equal(out2, out)


def _ctx(n_st, n_dir, n_cb, npol, nspd=None):
    ncorr = 4 if npol == 4 else 2
    return ddsolve.Context(n_st, nspd or [1] * n_dir, n_cb, ncorr, npol)


@pytest.mark.gpu
@pytest.mark.parametrize("npol", [1, 2, 4])
@pytest.mark.parametrize("subtract,keep", [(True, False), (True, True), (False, True)])
def test_gpu_equals_oracle_bitwise(built, npol, subtract, keep):
    a1, a2, data, model, sol = _interval(npol=npol, seed=npol)
    ctx = _ctx(6, 3, 2, npol)
    got_d, got_m = ctx.correct_and_subtract(a1, a2, sol, data=data, model=model,
                                            subtract=subtract, keep_model=keep)
    ctx.close()
    want_d, want_m = so.correct_and_subtract(data, model, sol, a1, a2, subtract, keep)
    if subtract:
        np.testing.assert_array_equal(got_d.view(np.uint32), want_d.view(np.uint32))
    else:
        assert got_d is None
    if keep:
        np.testing.assert_array_equal(got_m.view(np.uint32), want_m.view(np.uint32))
    else:
        assert got_m is None


@pytest.mark.gpu
@pytest.mark.parametrize("npol", [2, 4])
def test_gpu_device_buffers_in_place(built, npol):
    """Device-memory buffers through the C ABI, data and models corrected in
    place (data_out == data, models_out == models, one buffer per
    direction)."""
    import torch
    a1, a2, data, model, sol = _interval(n_st=9, n_t=3, n_ch=12, n_dir=4, n_cb=3, npol=npol,
                                         seed=7)
    want_d, want_m = so.correct_and_subtract(data, model, sol, a1, a2, True, True)
    ctx = _ctx(9, 4, 3, npol)
    dev = torch.device("cuda", 0)
    d_data = torch.from_numpy(data.view(np.float32).copy()).to(dev)
    # one separate device buffer per direction, as DDECal keeps them
    d_models = [torch.from_numpy(m.view(np.float32).copy()).to(dev) for m in model]
    d_sol = torch.from_numpy(sol.view(np.float64).copy()).to(dev)
    ptrs = (ctypes.c_void_p * len(d_models))(*[m.data_ptr() for m in d_models])
    ib = ddsolve.SubtractBuffers()
    ib.n_times, ib.n_baselines, ib.n_channels = data.shape[:3]
    ib.antenna1, ib.antenna2 = a1.ctypes.data, a2.ctypes.data
    ib.data, ib.models = d_data.data_ptr(), ctypes.cast(ptrs, ctypes.c_void_p).value
    torch.cuda.synchronize()
    rc = ddsolve.lib().ddsolve_correct_and_subtract(ctx._h, ctypes.byref(ib), d_sol.data_ptr(),
                                                    d_data.data_ptr(),
                                                    ctypes.cast(ptrs, ctypes.c_void_p))
    assert rc == 0, ddsolve.lib().ddsolve_last_error(ctx._h)
    ctx.close()
    got_d = d_data.cpu().numpy().view(np.complex64).reshape(data.shape)
    got_m = np.stack([m.cpu().numpy().view(np.complex64).reshape(model.shape[1:])
                      for m in d_models])
    np.testing.assert_array_equal(got_d.view(np.uint32), want_d.view(np.uint32))
    np.testing.assert_array_equal(got_m.view(np.uint32), want_m.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("npol", [1, 2])
def test_gpu_with_predicted_model(built, npol):
    """model = None: every direction's model (autocorrelations zero) predicted
    on the GPU from the sky, then corrected and subtracted."""
    cfg = synth.small_config(n_stations=7, n_directions=2, n_channels=8, n_cb=2, n_times=3,
                             seed=61)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    freqs = synth.frequencies(cfg)
    a1, a2, data, _, sol = _interval(n_st=7, n_t=3, n_ch=8, n_dir=2, n_cb=2, npol=npol)
    ctx = _ctx(7, 2, 2, npol)
    got_d, got_m = ctx.correct_and_subtract(a1, a2, sol, data=data, frequencies=freqs,
                                            station_uvw=uvw, sky=sky, keep_model=True)
    ctx.close()
    model = po.predict_raw(freqs, uvw, a1, a2, sky)
    want_d, want_m = so.correct_and_subtract(data, model, sol, a1, a2, True, True)
    scale = np.abs(want_m).max()
    assert np.abs(got_m - want_m).max() < 1e-5 * scale
    assert np.abs(got_d - want_d).max() < 1e-5 * scale
    auto = a1 == a2
    assert not got_m[:, :, auto].any()


@pytest.mark.gpu
def test_gpu_rejects_dd_intervals_and_bad_input(built):
    a1, a2, data, model, sol = _interval(n_dir=2)
    ctx = _ctx(6, 2, 2, 2, nspd=[1, 2])
    with pytest.raises(RuntimeError, match="direction dependent"):
        ctx.correct_and_subtract(a1, a2, np.ones((2, 6, 2, 2), np.complex128), data=data,
                                 model=model)
    ctx.close()
    ctx = _ctx(6, 2, 2, 2)
    bad = a2.copy()
    bad[3] = 40
    with pytest.raises(RuntimeError):
        ctx.correct_and_subtract(a1, bad, sol[:, :, :2], data=data, model=model[:2])
    with pytest.raises(RuntimeError):  # neither a model nor a sky
        ctx.correct_and_subtract(a1, a2, sol[:, :, :2], data=data)
    ctx.close()
