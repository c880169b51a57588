"""CPU oracle of the point-source predict (test infrastructure only).

A numpy restatement of DP3's predict of point sources, as
ddsolve_predict_regular computes it on the GPU (include/ddsolve_b200.h):

* station phases (base/Simulator.cc:477-520, phases()):
  stationPhases[p] = 2 pi / c (u_p l + v_p m + w_p (n - 1)), and per channel
  the shift exp(i stationPhases[p] nu) (separate sin and cos, :508-517);
* spectrum (:522-547, spectrum()) of a flat-spectrum source:
  XX = I + Q, XY = U + iV, YX = U - iV, YY = I - Q;
* visibility (:156-245, visit(PointSource)): per baseline (p, q) and
  channel, shift_q conj(shift_p) times the spectrum, summed over the
  direction's sources; autocorrelations are skipped (:160-161).

Everything in FP64 (as the reference's dcomplex buffer), rounded to
complex64 at the end, in the layout of the regular SolveData constructor:
model [n_dir][(t * n_baselines + b) * n_channels + c][n_corr][2]. The
single-correlation form is (XX + YY) / 2 = I, as SolveData's
ToSpecificMatrix for complex<float> (ddecal/gain_solvers/SolveData.cc:28-31)
reduces it. This oracle is pinned by the reference's formulas above (there
are no reference golden vectors for the predict here: DP3's predict tests
need casacore measurement sets).
"""
import numpy as np

C_LIGHT = 299792458.0


def predict(freqs, station_uvw, antenna1, antenna2, sky, n_corr):
    """freqs [n_ch] Hz; station_uvw [n_t][n_st][3] m; antenna1/2 [n_bl];
    sky: per direction (lmn [n_src][3], stokes [n_src][4]).
    Returns float32 [n_dir][n_t * n_bl * n_ch][n_corr][2]."""
    freqs = np.asarray(freqs, np.float64)
    uvw = np.asarray(station_uvw, np.float64)
    a1 = np.asarray(antenna1, np.int64)
    a2 = np.asarray(antenna2, np.int64)
    n_t, n_st, _ = uvw.shape
    n_bl, n_ch = len(a1), len(freqs)
    out = np.zeros((len(sky), n_t * n_bl * n_ch, n_corr, 2), np.float32)
    cinv = 2.0 * np.pi / C_LIGHT
    for d, (lmn, stokes) in enumerate(sky):
        lmn = np.asarray(lmn, np.float64).reshape(-1, 3)
        stokes = np.asarray(stokes, np.float64).reshape(-1, 4)
        vis = np.zeros((n_t, n_bl, n_ch, 4), np.complex128)
        for s in range(lmn.shape[0]):
            l, m, n = lmn[s]
            I, Q, U, V = stokes[s]
            spec = np.array([I + Q, U + 1j * V, U - 1j * V, I - Q])
            # [n_t][n_st] station phases, then [n_t][n_st][n_ch] shifts
            phase = cinv * (uvw[..., 0] * l + uvw[..., 1] * m + uvw[..., 2] * (n - 1.0))
            arg = phase[..., None] * freqs
            shift = np.cos(arg) + 1j * np.sin(arg)
            prod = shift[:, a2, :] * np.conj(shift[:, a1, :])  # [n_t][n_bl][n_ch]
            vis += prod[..., None] * spec
        vis[:, a1 == a2] = 0.0
        if n_corr == 4:
            v = vis
        elif n_corr == 2:
            v = vis[..., [0, 3]]
        else:
            v = 0.5 * (vis[..., :1] + vis[..., 3:])
        v = v.reshape(n_t * n_bl * n_ch, n_corr)
        out[d, :, :, 0] = v.real
        out[d, :, :, 1] = v.imag
    return out


def predict_raw(freqs, station_uvw, antenna1, antenna2, sky):
    """The same model in DP3's buffer layout: complex64
    [n_dir][n_t][n_bl][n_ch][4] (all four correlations, autocorrelations
    zero)."""
    n_t = np.shape(station_uvw)[0]
    m = predict(freqs, station_uvw, antenna1, antenna2, sky, 4)
    m = m[..., 0] + 1j * m[..., 1]
    return m.astype(np.complex64).reshape(len(sky), n_t, len(antenna1), len(freqs), 4)
