"""CPU oracle of DDECal's weighting and packing of one interval (test
infrastructure only).

A numpy restatement of what ddsolve_set_interval_buffers does on the GPU
(include/ddsolve_b200.h), from DP3's raw per-interval buffers
([time][baseline][channel][XX XY YX YY]) to the per-channel-block arrays of
the regular SolveData constructor:

* AssignAndWeight (ddecal/gain_solvers/SolverTools.cc:81-167): one flag per
  visibility, the OR over correlations of the buffer's flag, a non-finite
  data value and a non-finite model value of any direction (:112-124);
  prepared weights sqrt(w) in FP32, or w in linear mode (:131-139); data and
  each direction's model multiplied by the prepared weight per correlation
  (Weigh, :48-79); flagged visibilities set to zero in the data and every
  model (:145-162);
* the regular SolveData constructor (SolveData.cc:77-188): channel block
  cb = channels [cb n_ch / n_cb, (cb + 1) n_ch / n_cb) (:112-113),
  autocorrelations dropped (:100, :137), visibility order time -> baseline ->
  channel, ToSpecificMatrix (:18-31): XX and YY for 2 correlations,
  0.5 (XX + YY) for 1, all four for 4.

FP32 arithmetic as the reference's (complex<float> times float); pinned by
those reference lines (the reference's own tests of AssignAndWeight,
tSolverTools.cc, need its DPBuffer with casacore).
"""
import numpy as np


def weigh_and_pack(data, weights, flags, models, antenna1, antenna2, n_cb, n_corr,
                   linear=False):
    """data complex64 [n_t][n_bl][n_ch][4]; weights float32 [..][4]; flags
    bool/uint8 [..][4] or None; models complex64 [n_dir][n_t][n_bl][n_ch][4].
    Returns (data_cb, model_cb, a1_cross, a2_cross): per channel block
    float32 [n_vis, n_corr, 2] and [n_dir, n_vis, n_corr, 2]."""
    data = np.asarray(data, np.complex64)
    models = np.asarray(models, np.complex64)
    w = np.asarray(weights, np.float32)
    fin = lambda z: np.isfinite(z.real) & np.isfinite(z.imag)  # noqa: E731
    flag = (~fin(data)).any(-1)
    if flags is not None:
        flag |= np.asarray(flags, bool).any(-1)
    for m in models:
        flag |= (~fin(m)).any(-1)
    pw = w if linear else np.sqrt(w, dtype=np.float32)
    wd = (data * pw).astype(np.complex64)
    wm = (models * pw).astype(np.complex64)
    wd[flag] = 0
    wm[:, flag] = 0
    a1 = np.asarray(antenna1)
    a2 = np.asarray(antenna2)
    cross = a1 != a2
    wd, wm = wd[:, cross], wm[:, :, cross]
    n_ch = data.shape[2]

    def conv(z):
        if n_corr == 4:
            return z
        if n_corr == 2:
            return z[..., [0, 3]]
        return (np.float32(0.5) * (z[..., :1] + z[..., 3:])).astype(np.complex64)

    out_d, out_m = [], []
    for cb in range(n_cb):
        c0, c1 = cb * n_ch // n_cb, (cb + 1) * n_ch // n_cb
        d = conv(wd[:, :, c0:c1]).reshape(-1, n_corr)
        m = conv(wm[:, :, :, c0:c1]).reshape(models.shape[0], -1, n_corr)
        out_d.append(np.ascontiguousarray(np.stack([d.real, d.imag], -1), np.float32))
        out_m.append(np.ascontiguousarray(np.stack([m.real, m.imag], -1), np.float32))
    return out_d, out_m, a1[cross].astype(np.uint32), a2[cross].astype(np.uint32)
