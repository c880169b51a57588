"""Tests of ddsolve_set_interval_buffers (include/ddsolve_b200.h): DDECal's
AssignAndWeight and regular SolveData packing done on the GPU from DP3's
raw per-interval buffers.

CPU: the weighting oracle (oracle/weigh_oracle.py, restated from
SolverTools.cc:81-167 and SolveData.cc:77-188) on known cases.
GPU: an interval with autocorrelations, random weights (some zero), random
flags, non-finite data and model values, in sqrt and linear weighting mode,
for every correlation / polarization kind: the GPU-weighted context's
PerformIteration equals, element for element, that of a context fed the
oracle's weighted and packed arrays through ddsolve_set_channel_block_regular
(the same FP32 products in the same order, so no tolerance); with the model
predicted on the GPU instead of uploaded, within 1e-5 (the model differs by
complex64 roundings).
"""
import numpy as np
import pytest

from dp3_b200 import ddsolve, synth
from oracle import predict_oracle as po
from oracle import weigh_oracle as wo


def _interval(n_st=7, n_t=3, n_ch=8, n_dir=2, seed=0):
    rng = np.random.default_rng(seed)
    a1, a2 = np.triu_indices(n_st, 0)  # autocorrelations included
    n_bl = len(a1)
    cz = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex64)  # noqa: E731
    data = cz(n_t, n_bl, n_ch, 4)
    model = cz(n_dir, n_t, n_bl, n_ch, 4)
    w = rng.uniform(0.0, 2.0, (n_t, n_bl, n_ch, 4)).astype(np.float32)
    w[rng.random(w.shape) < 0.1] = 0.0
    flags = (rng.random((n_t, n_bl, n_ch, 4)) < 0.05).astype(np.uint8)
    data[1, 3, 2, 1] = np.nan
    data[2, 5, 0, 3] = np.inf
    model[1, 0, 4, 6, 2] = np.nan
    model[0, 2, 9, 1, 0] = np.complex64(complex(np.inf, 0))
    return a1.astype(np.uint32), a2.astype(np.uint32), data, w, flags, model


def test_oracle_flags_and_weights():
    a1, a2, data, w, flags, model = _interval()
    d, m, a1x, a2x = wo.weigh_and_pack(data, w, flags, model, a1, a2, 2, 4)
    assert len(a1x) == 21 and (a1x != a2x).all()
    # visibility (t=1, first cross baseline (0, 1), channel 2) of block 0
    bl = 1  # baseline index of (0, 1) in buffer order
    want = data[1, bl, 2] * np.sqrt(w[1, bl, 2])
    if flags[1, bl, 2].any():
        want[:] = 0
    got = d[0].reshape(3, 21, 4, 4, 2)[1, 0, 2]
    np.testing.assert_array_equal(got[:, 0] + 1j * got[:, 1], want)
    # the NaN datum flags its whole visibility, data and models
    bx = int(np.flatnonzero((a1x == a1[3]) & (a2x == a2[3]))[0])
    assert not d[0].reshape(3, 21, 4, 4, 2)[1, bx, 2].any()
    assert not m[0].reshape(2, 3, 21, 4, 4, 2)[:, 1, bx, 2].any()


def _ctx(n_st, nspd, n_cb, ncorr, npol):
    return ddsolve.Context(n_st, nspd, n_cb, ncorr, npol)


def _start(n_cb, n_st, n_sub, npol, seed=3):
    rng = np.random.default_rng(seed)
    s = (rng.standard_normal((n_cb, n_st, n_sub, npol))
         + 1j * rng.standard_normal((n_cb, n_st, n_sub, npol)))
    return 1.0 + 0.2 * s


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (1, 1), (2, 1)])
@pytest.mark.parametrize("linear", [False, True])
def test_gpu_weighting_equals_oracle_packing(built, ncorr, npol, linear):
    n_st, n_t, n_ch, n_cb = 7, 3, 8, 2
    a1, a2, data, w, flags, model = _interval(n_st, n_t, n_ch)
    nspd = [1, 2]
    start = _start(n_cb, n_st, 3, npol)
    raw = _ctx(n_st, nspd, n_cb, ncorr, npol)
    raw.set_interval_buffers(a1, a2, data, w, flags=flags, model=model, linear_weighting=linear)
    got = raw.perform_iteration(start)
    raw.close()
    d, m, a1x, a2x = wo.weigh_and_pack(data, w, flags, model, a1, a2, n_cb, ncorr, linear)
    ref = _ctx(n_st, nspd, n_cb, ncorr, npol)
    for cb in range(n_cb):
        ref.set_channel_block_regular(cb, n_t, len(a1x), n_ch // n_cb, d[cb], m[cb], a1x, a2x)
    want = ref.perform_iteration(start)
    ref.close()
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 1)])
def test_gpu_weighting_with_gpu_predict(built, ncorr, npol):
    """model = None: the unweighted model predicted on the GPU from the sky,
    then weighted; against the oracle packing of the predict oracle's model."""
    cfg = synth.small_config(n_stations=7, n_directions=2, n_channels=8, n_cb=2, n_times=3,
                             seed=61)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    freqs = synth.frequencies(cfg)
    a1, a2, data, w, flags, _ = _interval(7, 3, 8)
    raw = _ctx(7, cfg.nspd, 2, ncorr, npol)
    raw.set_interval_buffers(a1, a2, data, w, flags=flags, frequencies=freqs,
                             station_uvw=uvw, sky=sky)
    start = _start(2, 7, 2, npol)
    got = raw.perform_iteration(start)
    raw.close()
    model = po.predict_raw(freqs, uvw, a1, a2, sky)
    d, m, a1x, a2x = wo.weigh_and_pack(data, w, flags, model, a1, a2, 2, ncorr)
    ref = _ctx(7, cfg.nspd, 2, ncorr, npol)
    for cb in range(2):
        ref.set_channel_block_regular(cb, 3, len(a1x), 4, d[cb], m[cb], a1x, a2x)
    want = ref.perform_iteration(start)
    ref.close()
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-12)
    assert np.nanmax(err) < 1e-5


@pytest.mark.gpu
def test_interval_buffers_reject_bad_input(built):
    a1, a2, data, w, flags, model = _interval()
    ctx = _ctx(7, [1, 2], 2, 2, 2)
    bad = a2.copy()
    bad[4] = 50
    with pytest.raises(RuntimeError):
        ctx.set_interval_buffers(a1, bad, data, w, model=model)
    with pytest.raises(RuntimeError):  # neither a model nor a sky
        ctx.set_interval_buffers(a1, a2, data, w)
    ctx.close()
