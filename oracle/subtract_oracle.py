"""DDECal's model correction and subtraction restated in numpy (test
infrastructure only).

Follows DDECal::CorrectAndSubtractModels (steps/DDECal.cc:1081-1125) and
ApplySolutionAndSubtract (:1031-1079): for every visibility of the interval
(autocorrelations included) and every direction, the direction's model
(complex<float>, widened to complex<double>) is corrected with the solutions
of the visibility's channel block and antennas, in FP64:
  * full-Jones  J_1.Multiply(M).MultiplyHerm(J_2)           (:1004-1011)
  * diagonal    (diag(g_1) M) diag(g_2)^H                    (:1013-1019)
  * scalar      M (g_1 conj(g_2))                            (:1021-1027)
with aocommon's 2x2 products (r_ij = a_i0 b_0j + a_i1 b_1j, the Hermitian
variant with conj(b_ji)). The corrected models are summed over directions
from zero in direction order, kept as complex<float> when keepmodel is set
(AssignTo), and subtracted from the data as float(double(data) - sum) when
subtract is set (complex<float> -= complex<double>). The solutions of channel
ch are those of the even-split channel block cb with
cb n_ch / n_cb <= ch < (cb + 1) n_ch / n_cb (DDECal.cc:308-313).

Every complex product is written out as real multiplies and adds, each a
separately rounded numpy float64 operation: the arithmetic of the reference
built without fused multiply-adds (a build for a host with FMA and GCC's
default contraction may fuse some of them, which moves FP64 values by an ulp).
"""
import numpy as np


def _mul(a, b):
    (ar, ai), (br, bi) = a, b
    return ar * br - ai * bi, ar * bi + ai * br


def _add(a, b):
    return a[0] + b[0], a[1] + b[1]


def _conj(a):
    return a[0], -a[1]


def _parts(z):
    return np.ascontiguousarray(z.real, np.float64), np.ascontiguousarray(z.imag, np.float64)


def channel_block_of_channel(n_ch, n_cb):
    cb = np.empty(n_ch, np.int64)
    for c in range(n_cb):
        cb[c * n_ch // n_cb:(c + 1) * n_ch // n_cb] = c
    return cb


def correct_and_subtract(data, model, solutions, antenna1, antenna2, subtract=True,
                         keep_model=False):
    """data complex64 [t][bl][ch][4]; model complex64 [dir][t][bl][ch][4];
    solutions complex128 [n_cb][n_ant][n_dir][n_pol] (n_pol 1, 2 or 4).
    Returns (data_out or None, corrected models or None), complex64."""
    n_dir, n_t, n_bl, n_ch, _ = model.shape
    n_cb, _, n_dir_s, n_pol = solutions.shape
    assert n_dir_s == n_dir
    cb = channel_block_of_channel(n_ch, n_cb)
    a1 = np.asarray(antenna1, np.int64)
    a2 = np.asarray(antenna2, np.int64)
    # gains per (baseline, channel): [bl][ch][dir][pol]
    s1 = solutions[cb[None, :], a1[:, None]]
    s2 = solutions[cb[None, :], a2[:, None]]
    zero = np.zeros((n_t, n_bl, n_ch), np.float64)
    total = [(zero.copy(), zero.copy()) for _ in range(4)]
    kept = np.empty(model.shape, np.complex64) if keep_model else None
    for d in range(n_dir):
        m = [_parts(model[d, ..., k].astype(np.complex128)) for k in range(4)]
        g1 = [_parts(s1[None, :, :, d, p]) for p in range(n_pol)]
        g2 = [_parts(s2[None, :, :, d, p]) for p in range(n_pol)]
        if n_pol == 4:
            t = [_add(_mul(g1[2 * i], m[j]), _mul(g1[2 * i + 1], m[2 + j]))
                 for i in range(2) for j in range(2)]
            h = [_conj(x) for x in g2]
            c = [_add(_mul(t[2 * i], h[2 * j]), _mul(t[2 * i + 1], h[2 * j + 1]))
                 for i in range(2) for j in range(2)]
        elif n_pol == 2:
            h = [_conj(x) for x in g2]
            c = [_mul(_mul(g1[k // 2], m[k]), h[k % 2]) for k in range(4)]
        else:
            f = _mul(g1[0], _conj(g2[0]))
            c = [_mul(m[k], f) for k in range(4)]
        for k in range(4):
            total[k] = _add(total[k], c[k])
            if keep_model:
                kept[d, ..., k].real = np.broadcast_to(c[k][0], zero.shape).astype(np.float32)
                kept[d, ..., k].imag = np.broadcast_to(c[k][1], zero.shape).astype(np.float32)
    out = None
    if subtract:
        out = np.empty(data.shape, np.complex64)
        for k in range(4):
            dr, di = _parts(data[..., k].astype(np.complex128))
            re = (dr - total[k][0]).astype(np.float32)
            im = (di - total[k][1]).astype(np.float32)
            out[..., k].real = re
            out[..., k].imag = im
    return out, kept
