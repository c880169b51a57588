"""CPU oracle of the warm-start network (test infrastructure only).

A numpy restatement of the forward pass and the loss gradient that
libddwarm_b200.so computes on the tensor cores (include/ddwarm_b200.h): the
same three layers (ReLU, ReLU, linear), the same BF16 rounding points (weights;
the input; the hidden activations after ReLU; dL/dY; dL/dZ2 and dL/dZ1 after
the ReLU mask), FP64 accumulation instead of the GPU's FP32. With
`rounding=False` every quantity stays FP64, which the finite-difference test
uses to pin the gradient formulas themselves.

The reference (DP3) has no learned component, so this oracle is pinned by
finite differences of its own FP64 loss, not by a reference test.
"""
import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    nan = np.isnan(x)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def unpack(flat, n_in, hidden, n_out):
    shapes = [(hidden, n_in), (hidden,), (hidden, hidden), (hidden,), (n_out, hidden), (n_out,)]
    out, off = [], 0
    for s in shapes:
        n = int(np.prod(s))
        out.append(np.asarray(flat[off:off + n], np.float64).reshape(s))
        off += n
    return out


def forward(params, x, rounding=True):
    w1, b1, w2, b2, w3, b3 = params
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    # the GPU rounds each FP32 weight to BF16 once
    w1r, w2r, w3r = (r(np.asarray(w, np.float32)) if rounding else w for w in (w1, w2, w3))
    xb = r(x)
    z1 = xb @ w1r.T + b1
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ w2r.T + b2
    h2 = r(np.maximum(z2, 0.0))
    y = h2 @ w3r.T + b3
    return {"x": xb, "h1": h1, "h2": h2, "y": y, "w": (w1r, w2r, w3r)}


def loss_and_gradients(params, x, t, rounding=True):
    """Loss = mean((y - t)^2) and its gradient, packed like the parameters."""
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    f = forward(params, x, rounding)
    w1r, w2r, w3r = f["w"]
    n, n_out = t.shape
    d = f["y"] - t
    loss = float(np.mean(d * d))
    dy = r(2.0 * d / (n * n_out))
    gw3 = dy.T @ f["h2"]
    gb3 = dy.sum(0)
    dz2 = r((dy @ w3r) * (f["h2"] > 0))
    gw2 = dz2.T @ f["h1"]
    gb2 = dz2.sum(0)
    dz1 = r((dz2 @ w2r) * (f["h1"] > 0))
    gw1 = dz1.T @ f["x"]
    gb1 = dz1.sum(0)
    grads = np.concatenate([g.ravel() for g in (gw1, gb1, gw2, gb2, gw3, gb3)])
    return loss, grads
