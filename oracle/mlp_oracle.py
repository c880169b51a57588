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

Layer-wise checks (`check_trace`): each tensor-core product is checked on its
own, fed the GPU's own BF16 input of that layer (ddwarm_trace). BF16 x BF16
products are exact in FP32, so only the FP32 accumulation separates the GPU's
pre-activation z_gpu from the exact FP64 value z of the same inputs:
|z_gpu - z| <= e = (K + 2) 2^-23 (sum_k |a_k w_k| + |b|) for K terms (one
FP32 unit in the last place per addition, which also covers adders that
truncate instead of rounding). Rounding to BF16 and the ReLU are monotone, so
a correct BF16 output must lie in [bf16(relu(z - e)), bf16(relu(z + e))]
element by element: a value outside that interval is a bug (wrong bias,
element, mask or epilogue), never a rounding effect, while a value inside it
that differs from bf16(relu(z)) is a neighbour rounding ("flip"), counted.
FP32 outputs (y, the weight gradients, the column sums) must lie within e of
the exact value. The end-to-end comparison with `forward` (the oracle's own
chain from x) is then explained exactly by linearity: y_gpu - y_oracle =
(h2_gpu - h2_oracle) W3^T plus the last product's accumulation error, so
|y_gpu - y_oracle| <= |h2_gpu - h2_oracle| |W3|^T + e3.
"""
import numpy as np

ULP32 = 2.0 ** -23  # FP32 unit in the last place at 1


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


def check_case(shapes, flat, n, seed):
    """Inputs shared by smoke() and the forward/gradient tests: the network's
    parameters `flat` (packed, logical `shapes`) with non-zero biases added
    (they exercise the bias epilogue), an input x [n][n_in] ~ N(0, 1) and a
    target t [n][n_out] ~ N(0, 1), all from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    flat = np.asarray(flat, np.float32).copy()
    off = 0
    for s in shapes:
        k = int(np.prod(s))
        if len(s) == 1:
            flat[off:off + k] += rng.normal(0, 0.05, k).astype(np.float32)
        off += k
    n_in, n_out = shapes[0][1], shapes[4][0]
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32)
    return flat, x, t


def _product(a, w, b=None):
    """Exact z = a w^T (+ b) in FP64 and its FP32-accumulation bound e."""
    a = np.asarray(a, np.float64)
    w = np.asarray(w, np.float64)
    z = a @ w.T
    mag = np.abs(a) @ np.abs(w).T
    if b is not None:
        z = z + b
        mag = mag + np.abs(b)
    return z, (a.shape[1] + 2) * ULP32 * mag


def _bf16_interval(name, got, lo_pre, hi_pre, exact_pre, report):
    """got must lie in [bf16(lo_pre), bf16(hi_pre)]; counts flips against
    bf16(exact_pre)."""
    lo, hi = bf16(lo_pre), bf16(hi_pre)
    got = np.asarray(got, np.float64)
    bad = ~((got >= lo) & (got <= hi))
    report[name + "_outside"] = int(bad.sum())
    report[name + "_flips"] = int((got != bf16(exact_pre)).sum())
    report[name + "_count"] = int(got.size)
    if bad.any():
        i = np.argwhere(bad)[0]
        report.setdefault("failures", []).append(
            f"{name}{tuple(int(v) for v in i)}: {got[tuple(i)]!r} not in "
            f"[{lo[tuple(i)]!r}, {hi[tuple(i)]!r}]")


def _within(name, got, exact, e, report):
    d = np.abs(np.asarray(got, np.float64) - exact)
    bad = ~(d <= e)
    report[name + "_outside"] = int(bad.sum())
    report[name + "_max_err_over_bound"] = float(np.max(d / np.maximum(e, 1e-300)))
    if bad.any():
        i = np.argwhere(bad)[0]
        report.setdefault("failures", []).append(
            f"{name}{tuple(int(v) for v in i)}: |{got[tuple(i)]!r} - {exact[tuple(i)]!r}| "
            f"> {e[tuple(i)]!r}")


def check_trace(params, x, trace, t=None):
    """Layer-wise check of one GPU pass (ddwarm_trace output `trace`) against
    this oracle fed the GPU's own inputs of each layer (bounds in the module
    docstring). Returns a report dict; report['failures'] lists the elements
    outside their bounds (empty when the pass is correct)."""
    w1, b1, w2, b2, w3, b3 = params
    w1r, w2r, w3r = (bf16(np.asarray(w, np.float32)) for w in (w1, w2, w3))
    rep = {"failures": []}
    xb = np.asarray(trace["xb"], np.float64)
    if not np.array_equal(xb, bf16(x)):
        rep["failures"].append("xb differs from bf16(x)")
    relu = lambda v: np.maximum(v, 0.0)  # noqa: E731
    z1, e1 = _product(xb, w1r, b1)
    _bf16_interval("h1", trace["h1"], relu(z1 - e1), relu(z1 + e1), relu(z1), rep)
    h1 = np.asarray(trace["h1"], np.float64)
    z2, e2 = _product(h1, w2r, b2)
    _bf16_interval("h2", trace["h2"], relu(z2 - e2), relu(z2 + e2), relu(z2), rep)
    h2 = np.asarray(trace["h2"], np.float64)
    z3, e3 = _product(h2, w3r, b3)
    _within("y", trace["y"], z3, e3, rep)
    # end to end: the oracle's own chain from x, differences explained by the
    # hidden-layer differences (linearity of the last product)
    f = forward(params, x)
    rep["h1_vs_chain_differ"] = int((h1 != f["h1"]).sum())
    rep["h2_vs_chain_differ"] = int((h2 != f["h2"]).sum())
    e_chain = np.abs(h2 - f["h2"]) @ np.abs(w3r).T + e3
    _within("y_vs_chain", trace["y"], f["y"], e_chain, rep)
    rep["y_vs_chain_max_rel"] = float(np.max(np.abs(trace["y"] - f["y"]))
                                      / np.max(np.abs(f["y"])))
    if t is None:
        return rep
    n, n_out = np.shape(t)
    y = np.asarray(trace["y"], np.float64)
    t64 = np.asarray(t, np.float64)
    g = 2.0 * (y - t64) / (n * n_out)
    eg = 4 * 2.0 ** -24 * np.abs(g)  # fl(y - t), fl(2 / (n n_out)), fl(product)
    _bf16_interval("dy", trace["dy"], g - eg, g + eg, g, rep)
    dy = np.asarray(trace["dy"], np.float64)
    p2, ep2 = _product(dy, w3r.T)
    m2 = h2 > 0
    _bf16_interval("dz2", trace["dz2"], np.where(m2, p2 - ep2, 0.0),
                   np.where(m2, p2 + ep2, 0.0), np.where(m2, p2, 0.0), rep)
    dz2 = np.asarray(trace["dz2"], np.float64)
    p1, ep1 = _product(dz2, w2r.T)
    m1 = h1 > 0
    _bf16_interval("dz1", trace["dz1"], np.where(m1, p1 - ep1, 0.0),
                   np.where(m1, p1 + ep1, 0.0), np.where(m1, p1, 0.0), rep)
    dz1 = np.asarray(trace["dz1"], np.float64)
    shapes = [w.shape for w in (w1, b1, w2, b2, w3, b3)]
    grads = unpack(trace["grads"], shapes[0][1], shapes[0][0], shapes[4][0])
    for name, dz, a, k in (("gw3", dy, h2, 4), ("gw2", dz2, h1, 2), ("gw1", dz1, xb, 0)):
        z, e = _product(dz.T, a.T)
        _within(name, grads[k], z, e, rep)
        zb = dz.sum(0)
        _within(name.replace("w", "b"), grads[k + 1], zb,
                (n + 2) * ULP32 * np.abs(dz).sum(0), rep)
    loss = float(np.mean((y - t64) ** 2))
    _within("loss", np.array([trace["loss"]]), np.array([loss]),
            np.array([1e-6 * loss]), rep)
    return rep


def check_network(mlp, n, seed, with_target):
    """Sets check_case's parameters (non-zero biases) on the GPU network
    `mlp` (dp3_b200.warmstart.MLP), runs one traced pass on check_case's
    input (and target) and checks it layer by layer. Shared by smoke() and
    the tests, so that both check the same inputs. Returns the report."""
    flat, x, t = check_case(mlp.shapes(), mlp.params(), n, seed)
    mlp.set_params(flat)
    params = mlp.unpack(mlp.params())
    trace = mlp.trace(x, t if with_target else None)
    return check_trace(params, x, trace, t if with_target else None)
