"""Tests of the learned warm start (include/ddwarm_b200.h, dp3_b200/warmstart.py).

CPU: the MLP oracle's gradient formulas against finite differences of its own
FP64 loss (the oracle has no reference counterpart to be pinned to), its BF16
rounding against known values, and the exported symbols.
GPU: every tensor-core product of the forward pass and of the loss gradient
checked layer by layer against the oracle fed the GPU's own input of that
layer (oracle/mlp_oracle.py check_trace: a BF16 output outside the interval
its FP32 accumulation allows is a bug, a neighbour rounding inside it is
counted), an end-to-end sanity check against the oracle's own chain, the GPU
feature and start computations against numpy, training, and
the iteration count the trained network saves on a sequence of solution
intervals, with the accuracy of the final solutions checked against a
tight-tolerance solve.
"""
import subprocess

import numpy as np
import pytest

from dp3_b200 import warmstart
from oracle import mlp_oracle as mo
from tests import helpers as H

GRAD_RTOL = 2e-2  # end-to-end sanity check only: Frobenius norm of the difference / of the oracle
PASS_RTOL = 1e-4  # final solutions


def _random_params(rng, n_in, hidden, n_out, scale=0.3):
    shapes = [(hidden, n_in), (hidden,), (hidden, hidden), (hidden,), (n_out, hidden), (n_out,)]
    return [rng.normal(0, scale / np.sqrt(s[-1]), s) if len(s) == 2 else rng.normal(0, 0.1, s)
            for s in shapes]


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n_in, hidden, n_out, n = 6, 10, 4, 9
    params = _random_params(rng, n_in, hidden, n_out, scale=1.0)
    x = rng.normal(size=(n, n_in))
    t = rng.normal(size=(n, n_out))
    loss, g = mo.loss_and_gradients(params, x, t, rounding=False)
    flat = np.concatenate([p.ravel() for p in params])

    def loss_at(v):
        return mo.loss_and_gradients(mo.unpack(v, n_in, hidden, n_out), x, t, rounding=False)[0]

    eps = 1e-6
    for i in rng.choice(flat.size, 40, replace=False):
        e = np.zeros_like(flat)
        e[i] = eps
        fd = (loss_at(flat + e) - loss_at(flat - e)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_known_values():
    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 0.0],
                 np.float32)
    # ties go to even mantissa: 1 + 2^-8 -> 1, 1 + 3 * 2^-8 -> 1 + 2^-6
    np.testing.assert_array_equal(mo.bf16(v), [1.0, 1.0, 1.0 + 2.0 ** -6, 1.0, -2.5, 0.0])


def test_library_exports_every_declared_symbol(built):
    out = subprocess.run(["nm", "-D", "--defined-only", warmstart.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    header = open(warmstart.LIB_PATH.replace("dp3_b200/libddwarm_b200.so",
                                             "include/ddwarm_b200.h")).read()
    for s in warmstart.EXPORTED_SYMBOLS:
        assert s in names, s
        assert s + "(" in header, s


def _np_features(sets, scale):
    """numpy statement of ddwarm_features (include/ddwarm_b200.h)."""
    n_cb, n_ant, n_sub, n_pol = sets[0].shape
    samp = lambda a: np.transpose(a, (1, 2, 0, 3)).reshape(n_ant * n_sub, n_cb * n_pol)
    base = samp(sets[0])
    parts = []
    for s_ in sets[1:]:
        with np.errstate(all="ignore"):
            r = np.log(samp(s_) / base)
        r[~np.isfinite(r)] = 0
        parts += [r.real, r.imag]
    return np.concatenate(parts, axis=1) * scale


@pytest.mark.gpu
def test_features_and_start_match_numpy(built):
    rng = np.random.default_rng(1)
    shape = (3, 5, 4, 2)
    sets = [np.exp(0.1 * (rng.normal(size=shape) + 1j * rng.normal(size=shape)))
            for _ in range(4)]
    sets[2][1, 2, 3, 0] = np.nan  # a flagged entry: its feature is 0
    lay = warmstart.Layout(3, 5, 4, 2, 20.0)
    st = warmstart.Stage(lay, 4, hidden=64, seed=2)
    x = st.features(sets)
    np.testing.assert_allclose(x, _np_features(sets, 20.0), rtol=1e-5, atol=1e-5)
    start = st.predict(sets)
    y = st.mlp.predict(x).astype(np.float64) / 20.0
    w = 6
    samp = lambda a: np.transpose(a, (1, 2, 0, 3)).reshape(20, w)
    expect = samp(sets[0]) * np.exp(y[:, :w] + 1j * y[:, w:])
    expect = np.transpose(expect.reshape(5, 4, 3, 2), (2, 0, 1, 3))
    np.testing.assert_allclose(start, expect, rtol=1e-6)
    # the same through device-resident sets and output
    import torch
    dev_sets = [torch.from_numpy(s_).cuda() for s_ in sets]
    np.testing.assert_allclose(st.predict(dev_sets).cpu().numpy(), start, rtol=1e-12)
    st.close()


def _assert_report(rep, max_flip_frac=0.01):
    """No element outside its layer-wise bound; neighbour roundings rare."""
    assert not rep["failures"], rep["failures"][:5]
    for k in [k for k in rep if k.endswith("_flips")]:
        frac = rep[k] / rep[k.replace("_flips", "_count")]
        assert frac <= max_flip_frac, (k, frac)


# (n_in, n_out, n, mlp seed, input seed); the first row is smoke()'s case
FORWARD_CASES = [(96, 48, 300, 3, 0), (96, 48, 300, 3, 96), (192, 48, 1000, 3, 1),
                 (40, 20, 128, 3, 2), (336, 48, 620, 3, 3), (144, 48, 4200, 3, 4)]


@pytest.mark.gpu
@pytest.mark.parametrize("n_in,n_out,n,mseed,seed", FORWARD_CASES)
def test_forward_matches_oracle_layerwise(built, n_in, n_out, n, mseed, seed):
    """Each product against the oracle fed the GPU's own layer input; the
    end-to-end difference from the oracle's own chain explained by the
    hidden-layer neighbour roundings (bounds in oracle/mlp_oracle.py)."""
    mlp = warmstart.MLP(n_in, n_out, hidden=256, seed=mseed)
    rep = mo.check_network(mlp, n, seed, with_target=False)
    mlp.close()
    _assert_report(rep)
    assert rep["y_vs_chain_outside"] == 0
    # predict() computes the same forward pass as the trace
    mlp = warmstart.MLP(n_in, n_out, hidden=256, seed=mseed)
    flat, x, _ = mo.check_case(mlp.shapes(), mlp.params(), n, seed)
    mlp.set_params(flat)
    np.testing.assert_array_equal(mlp.predict(x), mlp.trace(x)["y"])
    mlp.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(256, 5), (700, 6), (300, 0)])
def test_gradients_match_oracle_layerwise(built, n, seed):
    """dY, dZ2, dZ1 (BF16) and every weight / bias gradient and the loss
    against the oracle fed the GPU's own upstream values of that layer."""
    mlp = warmstart.MLP(96, 48, hidden=256, seed=5)
    rep = mo.check_network(mlp, n, seed, with_target=True)
    _assert_report(rep)
    # ddwarm_gradients is the same pass as the traced one
    flat, x, t = mo.check_case(mlp.shapes(), mlp.params(), n, seed)
    g, loss = mlp.gradients(x, t)
    tr = mlp.trace(x, t)
    np.testing.assert_array_equal(g, tr["grads"])
    assert loss == tr["loss"]
    mlp.close()


@pytest.mark.gpu
def test_gradients_close_to_oracle_chain(built):
    """End-to-end sanity check of the gradients against the oracle's own
    chain from x: GRAD_RTOL bounds the effect of BF16 neighbour roundings of
    the activations and dL/dZ (each a relative change of <= 2^-8) on the
    Frobenius norm of each gradient tensor."""
    n, n_in, n_out = 700, 96, 48
    mlp = warmstart.MLP(n_in, n_out, hidden=256, seed=5)
    flat, x, t = mo.check_case(mlp.shapes(), mlp.params(), n, 6)
    mlp.set_params(flat)
    g, loss = mlp.gradients(x, t)
    ref_loss, ref = mo.loss_and_gradients(mlp.unpack(mlp.params()), x, t)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for name, a, b in zip(("W1", "b1", "W2", "b2", "W3", "b3"), mlp.unpack(g),
                          mlp.unpack(ref)):
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < GRAD_RTOL, (name, rel)
    mlp.close()


@pytest.mark.gpu
def test_training_reduces_loss(built):
    rng = np.random.default_rng(11)
    n, n_in, n_out = 4096, 32, 16
    a = rng.normal(size=(n_in, n_out)) / np.sqrt(n_in)
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = np.tanh(x @ a).astype(np.float32)
    mlp = warmstart.MLP(n_in, n_out, hidden=128, seed=2)
    losses = mlp.train(x, t, epochs=30, batch=512, lr=2e-3, seed=4)
    assert losses[-1] < 0.1 * losses[0], losses
    mlp.close()


@pytest.mark.gpu
def test_perform_iterations_chains_single_passes(built):
    """ddsolve_perform_iterations equals the loop of single passes."""
    from dp3_b200 import ddsolve
    obs = H.small_observation(n_stations=9, n_directions=3, n_channels=8, n_cb=2,
                              n_times=2, seed=5)
    cfg = obs.cfg
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                      obs.model[cb], obs.antenna1, obs.antenna2)
    start = np.ones((cfg.n_channel_blocks, cfg.n_stations, sum(cfg.nspd), 2), np.complex128)
    chain = ctx.perform_iterations(start, 3)
    g = start
    for k in range(3):
        g = ctx.perform_iteration(g)
        np.testing.assert_allclose(chain[k], g, rtol=1e-12)
    ctx.close()


@pytest.mark.gpu
def test_learned_warm_start_saves_iterations(built):
    """A sequence of random-walk intervals (the learned-warm-start recipe at
    reduced size): trained on the plain solver's solutions of the first
    intervals, the two-stage network start needs fewer iterations plus
    feature passes than the previous-solution start on the later intervals.
    Accuracy: against a tight-tolerance (1e-8) solve of each interval, the
    warm-started solution is within 1e-4, or within 1.5x the plain solver's
    own distance when that exceeds 1e-4 (tolerance 1e-5 bounds the step,
    not the distance to the fixed point, which slow modes keep near 1e-4);
    warm and plain agree within 3e-4."""
    from dp3_b200 import ddsolve, synth
    cfg = synth.ObservationConfig("warm test: 24 st, 4 dir, 24 ch / 6 cb, 2 t", 24, 0,
                                  2000.0, 4, 10, 24, 120e6, 160e6, [4] * 6, 2, seed=77)
    n_int, n_train = 64, 44
    seq = synth.gain_sequence(cfg, n_int)
    n_sub = sum(cfg.nspd)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
    st = ddsolve.default_settings()
    st.max_iterations, st.accuracy, st.step_size = 100, 1e-5, 0.2
    tight = ddsolve.default_settings()
    tight.max_iterations, tight.accuracy, tight.step_size = 400, 1e-8, 0.2
    tight.detect_stalling = 0
    ctx.set_settings(st)
    ws = warmstart.LearnedWarmStart(cfg.n_channel_blocks, cfg.n_stations, n_sub, 2,
                                    passes=(3, 3), provisional_after=16)

    def load(i):
        obs = synth.observe(cfg, true_gains=seq[i], start_time_s=i * cfg.n_times * 10.0,
                            noise_seed=cfg.seed * 31 + i)
        for cb, nc in enumerate(cfg.cb_channels):
            ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                          obs.model[cb], obs.antenna1, obs.antenna2)

    sols = [np.ones((cfg.n_channel_blocks, cfg.n_stations, n_sub, 2), np.complex128)] * 4
    plain_it, warm_it, d_wp, d_w, d_p = [], [], [], [], []
    for i in range(n_int):
        load(i)
        s = sols[-1].copy()
        r = ctx.solve(s)
        if i >= n_train:
            plain_it.append(r.iterations)
            g = ws.start(ctx, [sols[-1], sols[-2], sols[-3], sols[-4]])
            rw = ctx.solve(g)
            warm_it.append(rw.iterations + ws.passes)
            ref = s.copy()
            ctx.set_settings(tight)
            ctx.solve(ref)
            ctx.set_settings(st)
            d_wp.append(H.max_rel_diff(g, s))
            d_w.append(H.max_rel_diff(g, ref))
            d_p.append(H.max_rel_diff(s, ref))
        elif i >= 4:
            ws.add_interval(ctx, [sols[-1], sols[-2], sols[-3], sols[-4]], s)
        if i == n_train - 1:
            ws.fit()
        sols.append(s)
    ws.close()
    ctx.close()
    assert np.mean(warm_it) < 0.8 * np.mean(plain_it), (np.mean(warm_it), np.mean(plain_it))
    for w, p in zip(d_w, d_p):
        assert w < max(PASS_RTOL, 1.5 * p), (w, p)
    assert max(d_wp) < 3 * PASS_RTOL, max(d_wp)


@pytest.mark.gpu
def test_device_start_matches_host_start(built):
    """The asynchronous device path of LearnedWarmStart.start (solver stream,
    no host waits) gives the start of the host path."""
    import torch
    from dp3_b200 import ddsolve
    obs = H.small_observation(n_stations=10, n_directions=2, n_channels=8, n_cb=2,
                              n_times=2, seed=9)
    cfg = obs.cfg
    n_sub = sum(cfg.nspd)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                      obs.model[cb], obs.antenna1, obs.antenna2)
    ws = warmstart.LearnedWarmStart(cfg.n_channel_blocks, cfg.n_stations, n_sub, 2,
                                    passes=(2, 2), hidden=64)
    rng = np.random.default_rng(4)
    shape = (cfg.n_channel_blocks, cfg.n_stations, n_sub, 2)
    hist = [np.exp(0.05 * (rng.normal(size=shape) + 1j * rng.normal(size=shape)))
            for _ in range(4)]
    host = ws.start(ctx, hist)
    dev = ws.start(ctx, [torch.from_numpy(h).cuda() for h in hist])
    got = dev.cpu().numpy()  # the current stream is ordered after the solver's
    np.testing.assert_allclose(got, host, rtol=1e-12)
    r = ctx.solve(dev)
    assert r.iterations > 0
    ws.close()
    ctx.close()
