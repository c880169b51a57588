"""Tests of the GPU point-source predict (ddsolve_predict_regular,
ddsolve_set_channel_block_regular_sky in include/ddsolve_b200.h).

CPU: the predict oracle (oracle/predict_oracle.py, DP3's point-source
predict restated from base/Simulator.cc) against the model visibilities of
the synthetic generator (dp3_b200/csrc/synth.cc, the same phase equation with
a per-block phasor recurrence): one formula, two evaluations.
GPU: the predict kernel against the oracle for 1, 2 and 4 correlations (4
with polarized sources: Stokes Q, U, V), evenly and unevenly spaced
channels; at full size (62 stations, 10 directions x 20 sources, 240
channels) against the generator's model; and the solver fed by the GPU
predict against the solver fed the uploaded model.

Bound: FP64 evaluation, complex64 result, so element-wise |GPU - oracle| <=
2^-23 (sum over the direction's sources of |S|), i.e. a few units in the last
place of the largest possible model value (the sincos implementations
differ in the last FP64 bits; complex64 rounding dominates).
"""
import numpy as np
import pytest

from dp3_b200 import ddsolve, synth
from oracle import predict_oracle as po
from tests import helpers as H


def _bound(sky, d):
    return 2.0 ** -23 * np.abs(sky[d][1]).sum()


def _check(got, want, sky):
    for d in range(len(sky)):
        err = np.max(np.abs(got[d].astype(np.float64) - want[d].astype(np.float64)))
        assert err <= _bound(sky, d), (d, err, _bound(sky, d))


def _polarized_sky(cfg, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for lmn, st in synth.sky(cfg):
        st = st.copy()
        st[:, 1:] = 0.2 * st[:, :1] * rng.uniform(-1, 1, (st.shape[0], 3))
        out.append((lmn, st))
    return out


def _block_freqs(cfg, cb):
    f = synth.frequencies(cfg)
    c0 = int(np.sum(cfg.cb_channels[:cb]))
    return f[c0:c0 + cfg.cb_channels[cb]]


def test_oracle_matches_generator_model():
    cfg = synth.small_config(n_stations=9, n_directions=3, n_channels=12, n_cb=3, n_times=3,
                             seed=41)
    obs = synth.observe(cfg)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    for cb in range(cfg.n_channel_blocks):
        want = po.predict(_block_freqs(cfg, cb), uvw, obs.antenna1, obs.antenna2, sky, 2)
        _check(obs.model[cb].reshape(want.shape), want, sky)


@pytest.mark.gpu
@pytest.mark.parametrize("ncorr,npol", [(2, 2), (4, 2), (1, 1)])
@pytest.mark.parametrize("spacing", ["even", "uneven"])
def test_gpu_predict_matches_oracle(built, ncorr, npol, spacing):
    cfg = synth.small_config(n_stations=11, n_directions=3, n_channels=10, n_cb=1, n_times=3,
                             seed=43)
    sky = _polarized_sky(cfg) if ncorr == 4 else synth.sky(cfg)
    uvw = synth.station_uvw(cfg, start_time_s=1234.0)
    freqs = synth.frequencies(cfg)
    if spacing == "uneven":
        freqs = freqs + np.random.default_rng(1).uniform(-3e5, 3e5, freqs.shape)
    a1, a2 = np.triu_indices(cfg.n_stations, 1)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, 1, ncorr, npol)
    got = ctx.predict_regular(cfg.n_times, len(a1), freqs, uvw, a1, a2, sky)
    ctx.close()
    _check(got, po.predict(freqs, uvw, a1, a2, sky, ncorr), sky)


@pytest.mark.gpu
def test_gpu_predict_full_size_matches_generator(built):
    """62 stations, 10 directions x 20 sources, 240 channels in 24 blocks,
    8 time steps: every block against the generator's model."""
    cfg = synth.benchmark_configs()[1]
    obs = synth.observe(cfg)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
    for cb in range(cfg.n_channel_blocks):
        got = ctx.predict_regular(cfg.n_times, cfg.n_baselines, _block_freqs(cfg, cb), uvw,
                                  obs.antenna1, obs.antenna2, sky)
        _check(got, obs.model[cb].reshape(got.shape), sky)
    ctx.close()


@pytest.mark.gpu
def test_gpu_predict_into_device_memory(built):
    import torch
    cfg = synth.small_config(n_stations=8, n_directions=2, n_channels=6, n_cb=1, n_times=2,
                             seed=47)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    freqs = synth.frequencies(cfg)
    a1, a2 = np.triu_indices(cfg.n_stations, 1)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, 1, 2, 2)
    host = ctx.predict_regular(cfg.n_times, len(a1), freqs, uvw, a1, a2, sky)
    dev = torch.zeros(host.shape, dtype=torch.float32, device="cuda:0")
    ctx.predict_regular(cfg.n_times, len(a1), freqs, uvw, a1, a2, sky, out=dev)
    np.testing.assert_array_equal(dev.cpu().numpy(), host)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg_index", [0, 1])
def test_solve_with_gpu_predict_matches_uploaded_model(built, cfg_index):
    """The solver fed by the GPU predict (only the data uploaded) against the
    solver fed the generator's model: identical iteration counts and the
    parity tolerance 1e-4 after phase referencing."""
    cfg = synth.benchmark_configs()[cfg_index]
    obs = synth.observe(cfg)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    n_sub = sum(cfg.nspd)
    st = ddsolve.default_settings()
    st.max_iterations, st.accuracy, st.step_size = cfg.max_iterations, cfg.tolerance, 0.2
    sols = []
    for use_sky in (False, True):
        ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
        ctx.set_settings(st)
        for cb, nc in enumerate(cfg.cb_channels):
            if use_sky:
                ctx.set_channel_block_regular_sky(cb, cfg.n_times, cfg.n_baselines, obs.data[cb],
                                                  _block_freqs(cfg, cb), uvw, obs.antenna1,
                                                  obs.antenna2, sky)
            else:
                ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc,
                                              obs.data[cb], obs.model[cb], obs.antenna1,
                                              obs.antenna2)
        sol = np.ones((cfg.n_channel_blocks, cfg.n_stations, n_sub, 2), np.complex128)
        r = ctx.solve(sol)
        sols.append((r, sol))
        ctx.close()
    assert sols[0][0].iterations == sols[1][0].iterations
    assert H.max_rel_diff(sols[1][1], sols[0][1]) < 1e-4


@pytest.mark.gpu
def test_predict_rejects_bad_input(built):
    cfg = synth.small_config(n_stations=6, n_directions=2, n_channels=4, n_cb=1, n_times=2)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, 1, 2, 2)
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    a1, a2 = np.triu_indices(cfg.n_stations, 1)
    bad = a2.copy()
    bad[3] = 99
    with pytest.raises(RuntimeError):
        ctx.predict_regular(cfg.n_times, len(a1), synth.frequencies(cfg), uvw, a1, bad, sky)
    huge = [(np.zeros((5000, 3)), np.ones((5000, 4))), sky[1]]
    with pytest.raises(RuntimeError, match="unsupported|200 KiB"):
        ctx.predict_regular(cfg.n_times, len(a1), synth.frequencies(cfg), uvw, a1, a2, huge)
    ctx.close()
