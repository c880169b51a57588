"""CPU tests of the synthetic-observation generator."""
import numpy as np

from dp3_b200 import synth


def test_deterministic_and_threads_independent():
    cfg = synth.small_config(n_stations=6, n_directions=2, n_channels=6,
                             n_cb=2, n_times=2, seed=3)
    a = synth.observe(cfg)
    b = synth.observe(cfg)
    for x, y in zip(a.data + a.model, b.data + b.model):
        np.testing.assert_array_equal(x, y)


def test_data_equals_gain_corrupted_model_plus_noise():
    cfg = synth.small_config(n_stations=6, n_directions=3, n_channels=8,
                             n_cb=2, n_times=3, seed=4)
    cfg.noise_sigma_jy = 0.0
    obs = synth.observe(cfg)
    g = obs.true_gains
    ch0 = 0
    for cb, nc in enumerate(cfg.cb_channels):
        d = obs.data[cb].reshape(cfg.n_times, cfg.n_baselines, nc, 2, 2)
        m = obs.model[cb].reshape(cfg.n_directions, cfg.n_times,
                                  cfg.n_baselines, nc, 2, 2)
        dc = d[..., 0] + 1j * d[..., 1]
        mc = m[..., 0, 0] + 1j * m[..., 0, 1]
        for b in range(cfg.n_baselines):
            p, q = obs.antenna1[b], obs.antenna2[b]
            for c in range(nc):
                for pol in range(2):
                    exp = sum(g[ch0 + c, p, dd, pol] * mc[dd, :, b, c] *
                              np.conj(g[ch0 + c, q, dd, pol])
                              for dd in range(cfg.n_directions))
                    np.testing.assert_allclose(dc[:, b, c, pol], exp,
                                               rtol=2e-5, atol=2e-5)
        ch0 += nc


def test_model_phase_equation_single_source():
    """One unit source at the phase centre gives V = 1 on every baseline."""
    cfg = synth.small_config(n_stations=5, n_directions=1, n_channels=4,
                             n_cb=1, n_times=2, seed=5, n_sources=1)
    cfg.max_offset_deg = 0.0
    cfg.flux_min_jy = cfg.flux_max_jy = 1.0
    obs = synth.observe(cfg)
    m = obs.model[0]
    np.testing.assert_allclose(m[..., 0], 1.0, atol=1e-6)
    np.testing.assert_allclose(m[..., 1], 0.0, atol=1e-6)


def test_benchmark_config_shapes():
    cfgs = synth.benchmark_configs()
    assert [c.n_stations for c in cfgs] == [24, 62, 62, 512, 62]
    assert cfgs[0].n_baselines == 276 and cfgs[1].n_baselines == 1891
    assert cfgs[3].n_baselines == 130816
    assert cfgs[1].n_vis == 3630720 and cfgs[3].n_vis == 16744448
    assert sum(cfgs[2].cb_channels) == 120
    assert all(3 <= c <= 12 for c in cfgs[2].cb_channels)
    assert cfgs[0].cb_channels == [4, 4, 4, 4]


def test_generic_arrays_match_regular_constructor():
    cfg = synth.small_config(n_stations=5, n_directions=2, n_channels=6,
                             n_cb=2, n_times=4, seed=6, nspd=[2, 3])
    obs = synth.observe(cfg)
    ap, sm = obs.generic_arrays()
    nc = cfg.cb_channels[0]
    # visibility (t, b, c) -> index (t * n_bl + b) * nc + c
    t, b, c = 3, 7, 1
    v = (t * cfg.n_baselines + b) * nc + c
    assert tuple(ap[0][v]) == (obs.antenna1[b], obs.antenna2[b])
    # solution index = t * min(nsol, n_times) / n_times + start
    assert sm[0][0, v] == t * 2 // 4
    assert sm[0][1, v] == 2 + t * 3 // 4
