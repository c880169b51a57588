"""Learned warm start for the direction-iterative solver.

`MLP` binds libddwarm_b200.so (the C ABI in include/ddwarm_b200.h): a
three-layer perceptron (two hidden layers of 256) whose forward and training
passes run on the B200 tensor cores (BF16 weights, FP32 accumulation).
`LearnedWarmStart` predicts the initial solutions of a new solution interval
in two stages, each a network over one sample per (antenna, sub-solution)
across all channel blocks and polarizations:

* inputs are complex logarithms of solution sets relative to a base set
  (features computed on the GPU, ddwarm_features): stage 1 uses the last four
  converged solutions h1..h4 (base h1) and K1 chained undamped passes of the
  solver over the current interval from h1 (the `PerformIteration` output
  next = num / den, ddsolve_perform_iterations: the per-antenna-direction
  residual statistics of the new data); stage 2 uses stage 1's prediction g1
  (base) and K2 passes from g1;
* targets are log(g / base) of the plain solver's converged solution g;
* prediction: base * exp(output) (ddwarm_predict_start).

The solver then runs from the prediction to the same tolerance as from the
previous solutions (DDECal's solution propagation), so only the iteration
count changes: the networks are a source of initial values, never of the
answer. Entries that are not finite (flagged antennas) are zero in the inputs
and keep the base value in the prediction.

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
    "ddwarm_gradients", "ddwarm_train", "ddwarm_features", "ddwarm_predict_start",
    "ddwarm_set_stream", "ddwarm_trace",
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
        L.ddwarm_features.argtypes = [vp, vp, u32, vp, vp]
        L.ddwarm_predict_start.argtypes = [vp, vp, u32, vp, vp]
        L.ddwarm_set_stream.argtypes = [vp, vp]
        L.ddwarm_trace.argtypes = [vp, u32, vp, vp, vp]
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

    def trace(self, x, t=None):
        """Intermediate values of one pass (ddwarm_trace): dict with xb, h1,
        h2, y and, with a target t, dy, dz2, dz1, grads and loss."""
        x = np.ascontiguousarray(x, np.float32)
        n = x.shape[0]
        h, o = self.hidden, self.n_out
        out = {"xb": np.zeros((n, self.n_in), np.float32), "h1": np.zeros((n, h), np.float32),
               "h2": np.zeros((n, h), np.float32), "y": np.zeros((n, o), np.float32)}
        if t is not None:
            t = np.ascontiguousarray(t, np.float32)
            out.update(dy=np.zeros((n, o), np.float32), dz2=np.zeros((n, h), np.float32),
                       dz1=np.zeros((n, h), np.float32),
                       grads=np.zeros(lib().ddwarm_param_count(self._h), np.float32),
                       loss=np.zeros(1, np.float32))
        st = TraceOut(*[ctypes.c_void_p(out[k].ctypes.data) if k in out else None
                        for k in TraceOut.KEYS])
        self._check(lib().ddwarm_trace(self._h, n, _ptr(x), _ptr(t) if t is not None else None,
                                       ctypes.byref(st)))
        if t is not None:
            out["loss"] = float(out["loss"][0])
        return out

    def train(self, x, t, epochs=100, batch=1024, lr=1e-3, seed=1):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        losses = np.zeros(max(epochs, 1), np.float32)
        self._check(lib().ddwarm_train(self._h, x.shape[0], _ptr(x), _ptr(t), epochs, batch,
                                       ctypes.c_float(lr), seed, _ptr(losses)))
        return losses[:epochs]


class TraceOut(ctypes.Structure):
    """ddwarm_trace_out (include/ddwarm_b200.h)."""
    KEYS = ("xb", "h1", "h2", "y", "dy", "dz2", "dz1", "grads", "loss")
    _fields_ = [(k, ctypes.c_void_p) for k in KEYS]


class Layout(ctypes.Structure):
    _fields_ = [("n_channel_blocks", ctypes.c_uint32), ("n_antennas", ctypes.c_uint32),
                ("n_sub", ctypes.c_uint32), ("n_pol", ctypes.c_uint32),
                ("scale", ctypes.c_double)]


def _sets_arg(sets):
    """Pointer array to solution sets: numpy arrays (host) or contiguous
    complex128 torch tensors (host or GPU)."""
    arrs, addrs = [], []
    for x in sets:
        if hasattr(x, "data_ptr"):
            x = x.contiguous()
            addrs.append(x.data_ptr())
        else:
            x = np.ascontiguousarray(x, np.complex128)
            addrs.append(x.ctypes.data)
        arrs.append(x)
    return arrs, (ctypes.c_void_p * len(arrs))(*addrs)


class Stage:
    """One network from solution sets [base, others...] to initial solutions
    (ddwarm_features / ddwarm_predict_start)."""

    def __init__(self, layout, n_sets, hidden=256, seed=1, device=0):
        self.layout = layout
        self.n_sets = n_sets
        self.width = layout.n_channel_blocks * layout.n_pol
        self.mlp = MLP(2 * self.width * (n_sets - 1), 2 * self.width, hidden=hidden, seed=seed,
                       device=device)
        self.x, self.t = [], []

    def features(self, sets):
        arrs, ptrs = _sets_arg(sets)
        rows = self.layout.n_antennas * self.layout.n_sub
        x = np.zeros((rows, 2 * self.width * (len(sets) - 1)), np.float32)
        self.mlp._check(lib().ddwarm_features(self.mlp._h, ctypes.byref(self.layout), len(arrs),
                                              ptrs, _ptr(x)))
        return x

    def add(self, sets, converged):
        """One training interval: features of `sets`, target log(converged / base)."""
        self.x.append(self.features(sets))
        self.t.append(self.features([sets[0], converged]))

    def fit(self, epochs=150, batch=1024, lr=1e-3, seed=1):
        return self.mlp.train(np.concatenate(self.x), np.concatenate(self.t), epochs=epochs,
                              batch=batch, lr=lr, seed=seed)

    def set_stream(self, stream_ptr):
        """Runs this network's work on a CUDA stream (e.g. the solver's)."""
        self.mlp._check(lib().ddwarm_set_stream(self.mlp._h, ctypes.c_void_p(stream_ptr)))

    def predict(self, sets, out=None):
        """Initial solutions, on the device of sets[0] (numpy in, numpy out;
        CUDA tensors in: a CUDA tensor out, `out` if given, and the call
        returns without waiting)."""
        arrs, ptrs = _sets_arg(sets)
        if hasattr(arrs[0], "data_ptr"):
            import torch
            start = torch.empty_like(arrs[0]) if out is None else out
            out = ctypes.c_void_p(start.data_ptr())
        else:
            start = np.empty_like(arrs[0])
            out = _ptr(start)
        self.mlp._check(lib().ddwarm_predict_start(self.mlp._h, ctypes.byref(self.layout),
                                                   len(arrs), ptrs, out))
        return start

    def close(self):
        self.mlp.close()


class LearnedWarmStart:
    """Two-stage learned warm start for solutions shaped
    [n_cb][n_ant][n_sub][n_pol] (the solver's layout).

    Stage 1 maps [h1, h2, h3, h4, z_1..z_K1] to g1, where h1..h4 are the last
    four converged solutions (h1 the previous interval's) and z_k are K1
    chained undamped passes over the current interval from h1
    (ddsolve_perform_iterations). Stage 2 maps [g1, y_1..y_K2], K2 passes from
    g1, to g2, the start of the solve. Training (`add_interval`, `fit`) uses
    intervals that the plain solver has solved; stage 2 learns from stage-1
    predictions of a provisional stage-1 network that has not seen the
    interval (fitted after `provisional_after` intervals), so that its inputs
    carry out-of-sample stage-1 errors.
    """

    HISTORY = 4

    def __init__(self, n_cb, n_ant, n_sub, n_pol, passes=(3, 3), hidden=256, scale=20.0,
                 seed=1, device=0, provisional_after=36):
        self.layout = Layout(n_cb, n_ant, n_sub, n_pol, scale)
        self.k1, self.k2 = passes
        self.provisional_after = provisional_after
        if 2 * n_cb * n_pol * (self.HISTORY - 1 + self.k1) > 1024 or 2 * n_cb * n_pol > 256:
            raise ValueError("too many channel blocks x polarizations for the network")
        self.stage1 = Stage(self.layout, self.HISTORY + self.k1, hidden, seed, device)
        self.stage2 = Stage(self.layout, 1 + self.k2, hidden, seed + 1, device)
        self._provisional = None
        self._args = (hidden, seed + 2, device)

    @property
    def passes(self):
        return self.k1 + self.k2

    def add_interval(self, solver, history, converged):
        """Adds one solved training interval whose data is loaded in
        `solver` (a ddsolve.Context); history = [h1, h2, h3, h4]."""
        z = solver.perform_iterations(history[0], self.k1)
        sets1 = list(history[:self.HISTORY]) + list(z)
        if self._provisional is not None:
            g1 = self._provisional.predict(sets1)
            y = solver.perform_iterations(g1, self.k2)
            self.stage2.add([g1] + list(y), converged)
        self.stage1.add(sets1, converged)
        if self._provisional is None and len(self.stage1.x) >= self.provisional_after:
            hidden, seed, device = self._args
            self._provisional = Stage(self.layout, self.stage1.n_sets, hidden, seed, device)
            self._provisional.x, self._provisional.t = list(self.stage1.x), list(self.stage1.t)
            self._provisional.fit()

    def fit(self, **kw):
        """Trains both stages on the collected intervals; returns the final
        epoch losses."""
        if not self.stage2.x:
            raise RuntimeError("not enough training intervals for the second stage")
        l1 = self.stage1.fit(**kw)
        l2 = self.stage2.fit(**kw)
        if self._provisional is not None:
            self._provisional.close()
            self._provisional = None
        return float(l1[-1]), float(l2[-1])

    def start(self, solver, history):
        """Initial solutions of the interval loaded in `solver`. With the
        history as CUDA tensors every step stays on the GPU, on the solver's
        stream, without host waits: the solver's stream first waits for the
        caller's current stream (which wrote the history), and the current
        stream then waits for the solver's stream, so the returned CUDA tensor
        is ready in the caller's stream order (and in the solver's)."""
        h1 = history[0]
        if not (hasattr(h1, "is_cuda") and h1.is_cuda):
            z = solver.perform_iterations(h1, self.k1)
            g1 = self.stage1.predict(list(history[:self.HISTORY]) + list(z))
            y = solver.perform_iterations(g1, self.k2)
            return self.stage2.predict([g1] + list(y))
        import torch
        ptr = solver.stream_ptr()
        if getattr(self, "_stream", None) != ptr:
            for st in (self.stage1, self.stage2):
                st.set_stream(ptr)
            self._stream = ptr
            # persistent work buffers: reused in stream order by later calls
            self._z = torch.empty((self.k1,) + tuple(h1.shape), dtype=h1.dtype, device=h1.device)
            self._y = torch.empty((self.k2,) + tuple(h1.shape), dtype=h1.dtype, device=h1.device)
            self._g1 = torch.empty_like(h1)
            self._torch_stream = torch.cuda.ExternalStream(ptr, device=h1.device)
        cur = torch.cuda.current_stream(h1.device)
        g2 = torch.empty_like(h1)
        # the history and g2's allocation are in the current stream's order
        self._torch_stream.wait_stream(cur)
        z = solver.perform_iterations(h1, self.k1, out=self._z)
        self.stage1.predict(list(history[:self.HISTORY]) + list(z), out=self._g1)
        y = solver.perform_iterations(self._g1, self.k2, out=self._y)
        self.stage2.predict([self._g1] + list(y), out=g2)
        # g2 (written on the solver's stream) is used and freed in the
        # current stream's order
        cur.wait_stream(self._torch_stream)
        return g2

    def close(self):
        for st in (self.stage1, self.stage2, self._provisional):
            if st is not None:
                st.close()
