"""Learned warm start for the direction-iterative solver.

`MLP` binds libddwarm_b200.so (the C ABI in include/ddwarm_b200.h): a
three-layer perceptron whose forward and training passes run on the B200
tensor cores (BF16 weights, FP32 accumulation). `LearnedWarmStart` turns
solver state into network samples and back:

* one sample per (antenna, sub-solution), across all channel blocks and
  polarizations;
* inputs: the last four converged solutions h1..h4 of that antenna and
  direction (h1 = the previous interval) and the current interval's one-pass
  residual statistic z = the undamped solver update from h1 (the
  `PerformIteration` output next = num / den, ddsolve_perform_iteration), all
  as complex logarithms relative to h1: log(h_k / h1), k = 2..4, and
  log(z / h1), real and imaginary parts, scaled by `scale`;
* target: log(g / h1) of the converged solution g of the interval, scaled
  alike; prediction g_hat = h1 * exp(y / scale).

The solver then runs from g_hat to the same tolerance as from the previous
solutions (DDECal's solution propagation), so only the iteration count
changes: the network is a source of initial values, never of the answer.
Entries that are not finite (flagged antennas) are zero in the inputs and
fall back to h1 in the prediction.

There is no CPU fallback: loading fails loudly when the library is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libddwarm_b200.so")

# Every symbol declared in include/ddwarm_b200.h.
EXPORTED_SYMBOLS = (
    "ddwarm_create", "ddwarm_destroy", "ddwarm_last_error", "ddwarm_param_count",
    "ddwarm_get_params", "ddwarm_set_params", "ddwarm_predict",
    "ddwarm_gradients", "ddwarm_train",
)

_lib = None


def lib():
    """Loads the warm-start library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python dp3_b200/build.py`"
                " (the warm start has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, i32, f32 = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                  ctypes.c_int, ctypes.c_float)
        L.ddwarm_create.argtypes = [u32, u32, u32, u64, i32, ctypes.POINTER(vp)]
        L.ddwarm_destroy.argtypes = [vp]
        L.ddwarm_destroy.restype = None
        L.ddwarm_last_error.argtypes = [vp]
        L.ddwarm_last_error.restype = ctypes.c_char_p
        L.ddwarm_param_count.argtypes = [vp]
        L.ddwarm_param_count.restype = u64
        L.ddwarm_get_params.argtypes = [vp, vp]
        L.ddwarm_set_params.argtypes = [vp, vp]
        L.ddwarm_predict.argtypes = [vp, u32, vp, vp]
        L.ddwarm_gradients.argtypes = [vp, u32, vp, vp, vp, vp]
        L.ddwarm_train.argtypes = [vp, u32, vp, vp, u32, u32, f32, u64, vp]
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class MLP:
    """n_in -> hidden -> hidden -> n_out perceptron with ReLU, on the GPU."""

    def __init__(self, n_in, n_out, hidden=256, seed=1, device=0):
        self.n_in, self.n_out, self.hidden = n_in, n_out, hidden
        h = ctypes.c_void_p()
        rc = lib().ddwarm_create(n_in, hidden, n_out, seed, device, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"ddwarm_create failed ({rc})")
        self._h = h

    def close(self):
        if self._h:
            lib().ddwarm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(lib().ddwarm_last_error(self._h).decode() or f"status {rc}")

    def shapes(self):
        """Logical parameter shapes in packed order."""
        i, h, o = self.n_in, self.hidden, self.n_out
        return [(h, i), (h,), (h, h), (h,), (o, h), (o,)]

    def params(self):
        out = np.zeros(lib().ddwarm_param_count(self._h), np.float32)
        self._check(lib().ddwarm_get_params(self._h, _ptr(out)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(lib().ddwarm_set_params(self._h, _ptr(p)))

    def unpack(self, flat):
        out, off = [], 0
        for s in self.shapes():
            n = int(np.prod(s))
            out.append(flat[off:off + n].reshape(s))
            off += n
        return out

    def predict(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], self.n_out), np.float32)
        if x.shape[0]:
            self._check(lib().ddwarm_predict(self._h, x.shape[0], _ptr(x), _ptr(y)))
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(lib().ddwarm_param_count(self._h), np.float32)
        loss = ctypes.c_float()
        self._check(lib().ddwarm_gradients(self._h, x.shape[0], _ptr(x), _ptr(t), _ptr(g),
                                           ctypes.byref(loss)))
        return g, float(loss.value)

    def train(self, x, t, epochs=100, batch=1024, lr=1e-3, seed=1):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(lib().ddwarm_train(self._h, x.shape[0], _ptr(x), _ptr(t), epochs, batch,
                                       ctypes.c_float(lr), seed, _ptr(losses)))
        return losses[:epochs]


def _clog(r):
    """Complex log with non-finite / zero entries mapped to 0."""
    with np.errstate(all="ignore"):
        out = np.log(r)
    bad = ~np.isfinite(out)
    out[bad] = 0.0
    return out


class LearnedWarmStart:
    """Features, targets and predictions for solutions shaped
    [n_cb][n_ant][n_sub][n_pol] (the solver's layout)."""

    HISTORY = 4

    def __init__(self, n_cb, n_ant, n_sub, n_pol, hidden=256, scale=20.0, seed=1, device=0):
        self.n_cb, self.n_ant, self.n_sub, self.n_pol = n_cb, n_ant, n_sub, n_pol
        self.scale = scale
        self.width = n_cb * n_pol  # complex values per sample and solution set
        self.n_in = 2 * self.width * self.HISTORY  # 3 history ratios + z
        self.n_out = 2 * self.width
        if self.n_in > 256 or self.n_out > 256:
            raise ValueError("too many channel blocks x polarizations for the network")
        self.mlp = MLP(self.n_in, self.n_out, hidden=hidden, seed=seed, device=device)

    def _samples(self, a):
        """[cb][ant][sub][pol] -> [ant * sub][cb * pol] (sample-major)."""
        return np.transpose(a, (1, 2, 0, 3)).reshape(self.n_ant * self.n_sub, self.width)

    def _unsamples(self, s):
        return np.transpose(s.reshape(self.n_ant, self.n_sub, self.n_cb, self.n_pol),
                            (2, 0, 1, 3))

    def features(self, history, z):
        """history: [h1, h2, h3, h4] (most recent first); z: the one-pass
        update from h1. Returns [n_ant * n_sub][n_in] float32."""
        h1 = self._samples(history[0])
        parts = []
        with np.errstate(all="ignore"):
            for h in history[1:self.HISTORY]:
                parts.append(_clog(self._samples(h) / h1))
            parts.append(_clog(self._samples(z) / h1))
        x = np.concatenate([np.concatenate([p.real, p.imag], axis=1) for p in parts], axis=1)
        return (x * self.scale).astype(np.float32)

    def targets(self, h1, g):
        with np.errstate(all="ignore"):
            r = _clog(self._samples(g) / self._samples(h1))
        return (np.concatenate([r.real, r.imag], axis=1) * self.scale).astype(np.float32)

    def predict(self, history, z):
        """Initial solutions of the new interval."""
        y = self.mlp.predict(self.features(history, z)).astype(np.float64) / self.scale
        w = self.width
        logr = y[:, :w] + 1j * y[:, w:]
        h1 = self._samples(history[0])
        g = h1 * np.exp(logr)
        bad = ~np.isfinite(g)
        g[bad] = h1[bad]
        return np.ascontiguousarray(self._unsamples(g))

    def train(self, x, t, **kw):
        return self.mlp.train(x, t, **kw)

    def close(self):
        self.mlp.close()
