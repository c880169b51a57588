"""Seeded synthetic observations of the benchmark configurations.

Python front end of libdp3b200_synth.so (dp3_b200/csrc/synth.{h,cc}). The
configurations follow the benchmark definitions of this solver: station
layouts, point-source models per direction, gains, noise, channelisation and
solution intervals. No public dataset exists for this benchmark; seeded
synthetic inputs with the stated shapes and distributions stand in for one.
"""
import ctypes
import os
from dataclasses import dataclass, field, replace
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdp3b200_synth.so")


class _Cfg(ctypes.Structure):
    _fields_ = [("n_stations", ctypes.c_uint32), ("layout", ctypes.c_uint32),
                ("radius_m", ctypes.c_double),
                ("n_directions", ctypes.c_uint32),
                ("n_sources", ctypes.c_uint32),
                ("max_offset_deg", ctypes.c_double),
                ("flux_min_jy", ctypes.c_double),
                ("flux_max_jy", ctypes.c_double),
                ("n_channels", ctypes.c_uint32),
                ("freq_lo_hz", ctypes.c_double),
                ("freq_hi_hz", ctypes.c_double),
                ("n_times", ctypes.c_uint32),
                ("time_step_s", ctypes.c_double),
                ("start_time_s", ctypes.c_double),
                ("dec_deg", ctypes.c_double), ("lat_deg", ctypes.c_double),
                ("noise_sigma_jy", ctypes.c_double),
                ("sky_seed", ctypes.c_uint64), ("noise_seed", ctypes.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build_synth()
        L = ctypes.CDLL(LIB_PATH)
        L.synth_n_baselines.restype = ctypes.c_uint64
        _lib = L
    return _lib


@dataclass
class ObservationConfig:
    """One benchmark configuration (one solution interval)."""
    name: str
    n_stations: int
    layout: int  # 0 disk, 1 log spiral
    radius_m: float
    n_directions: int
    n_sources: int
    n_channels: int
    freq_lo_hz: float
    freq_hi_hz: float
    cb_channels: List[int]
    n_times: int
    time_step_s: float = 10.0
    dec_deg: float = 50.0
    lat_deg: float = 52.9
    max_offset_deg: float = 2.0
    flux_min_jy: float = 0.1
    flux_max_jy: float = 10.0
    noise_sigma_jy: float = 0.01
    gain_amp_sigma: float = 0.1
    gain_delay_sigma_ns: float = 2.0
    seed: int = 1000
    n_solutions_per_direction: Optional[List[int]] = None
    # solver settings of the configuration
    step_size: float = 0.2
    max_iterations: int = 50
    tolerance: float = 1e-5

    @property
    def n_channel_blocks(self):
        return len(self.cb_channels)

    @property
    def n_baselines(self):
        return self.n_stations * (self.n_stations - 1) // 2

    @property
    def n_vis(self):
        return self.n_times * self.n_baselines * self.n_channels

    @property
    def nspd(self):
        return self.n_solutions_per_direction or [1] * self.n_directions

    def c_config(self, start_time_s=0.0, noise_seed=None):
        return _Cfg(self.n_stations, self.layout, self.radius_m,
                    self.n_directions, self.n_sources, self.max_offset_deg,
                    self.flux_min_jy, self.flux_max_jy, self.n_channels,
                    self.freq_lo_hz, self.freq_hi_hz, self.n_times,
                    self.time_step_s, start_time_s, self.dec_deg, self.lat_deg,
                    self.noise_sigma_jy, self.seed,
                    self.seed * 7919 + 17 if noise_seed is None else noise_seed)


def _even_blocks(n_ch, n_cb):
    """Channel split of the regular SolveData constructor
    (ddecal/gain_solvers/SolveData.cc:112-113)."""
    edges = [(cb * n_ch) // n_cb for cb in range(n_cb + 1)]
    return [edges[i + 1] - edges[i] for i in range(n_cb)]


def _uneven_blocks(n_ch, seed, lo=3, hi=12):
    rng = np.random.default_rng(seed)
    sizes = []
    left = n_ch
    while left > 0:
        if left <= hi:
            if left >= lo or not sizes:
                sizes.append(left)
            else:
                sizes[-1] += left
            break
        s = int(rng.integers(lo, hi + 1))
        if left - s < lo:
            s = left - lo if left - lo >= lo else left
        sizes.append(s)
        left -= s
    return sizes


def benchmark_configs():
    """The five benchmark configurations, by index."""
    c0 = ObservationConfig("c0: 24 st, 2 dir, 16 ch / 4 cb, 2 t", 24, 0, 2000.0,
                           2, 5, 16, 120e6, 160e6, _even_blocks(16, 4), 2,
                           seed=1000)
    c1 = ObservationConfig("c1: 62 st, 10 dir, 240 ch / 24 cb, 8 t", 62, 0,
                           2000.0, 10, 20, 240, 120e6, 160e6,
                           _even_blocks(240, 24), 8, seed=1001)
    c2 = ObservationConfig("c2: 62 st, 40 dir DD {1,2,4,8}, 120 ch uneven, 8 t",
                           62, 0, 2000.0, 40, 20, 120, 120e6, 160e6,
                           _uneven_blocks(120, 1002), 8, seed=1002,
                           n_solutions_per_direction=[(8, 4, 2, 1)[d % 4]
                                                      for d in range(40)])
    c3 = ObservationConfig("c3: 512 st, 5 dir, 64 ch / 16 cb, 2 t", 512, 1,
                           40000.0, 5, 50, 64, 50e6, 350e6,
                           _even_blocks(64, 16), 2, seed=1003)
    c4 = ObservationConfig("c4: 62 st, 10 dir, 120 ch / 12 cb, 2 t", 62, 0,
                           2000.0, 10, 20, 120, 120e6, 160e6,
                           _even_blocks(120, 12), 2, seed=1004)
    return [c0, c1, c2, c3, c4]


def small_config(n_stations=8, n_directions=2, n_channels=8, n_cb=2, n_times=2,
                 seed=7, nspd=None, n_sources=3):
    """A small configuration of the same recipe, for parity tests."""
    return ObservationConfig(
        f"small {n_stations}st {n_directions}dir", n_stations, 0, 2000.0,
        n_directions, n_sources, n_channels, 120e6, 160e6,
        _even_blocks(n_channels, n_cb), n_times, seed=seed,
        n_solutions_per_direction=nspd)


def gains(cfg: ObservationConfig, seed=None):
    """True gains [n_channels, n_stations, n_directions, 2] complex128."""
    c = cfg.c_config()
    g = np.zeros((cfg.n_channels, cfg.n_stations, cfg.n_directions, 2),
                 np.complex128)
    rc = lib().synth_gains(ctypes.byref(c),
                           ctypes.c_uint64(cfg.seed + 1 if seed is None else seed),
                           ctypes.c_double(cfg.gain_amp_sigma),
                           ctypes.c_double(cfg.gain_delay_sigma_ns),
                           ctypes.c_void_p(g.ctypes.data))
    assert rc == 0
    return g


def frequencies(cfg: ObservationConfig):
    c = cfg.c_config()
    f = np.zeros(cfg.n_channels, np.float64)
    lib().synth_frequencies(ctypes.byref(c), ctypes.c_void_p(f.ctypes.data))
    return f


def station_uvw(cfg: ObservationConfig, start_time_s=0.0):
    """Station UVW (m) per time step [n_times][n_stations][3], as observe()
    uses them for an interval starting at start_time_s."""
    c = cfg.c_config(start_time_s)
    uvw = np.zeros((cfg.n_times, cfg.n_stations, 3), np.float64)
    if lib().synth_station_uvw(ctypes.byref(c), ctypes.c_void_p(uvw.ctypes.data)) != 0:
        raise RuntimeError("synth_station_uvw failed")
    return uvw


def sky(cfg: ObservationConfig):
    """The point-source sky of cfg: per direction (lmn [n_sources][3], Stokes
    [n_sources][4] with I = the flux, Q = U = V = 0)."""
    c = cfg.c_config()
    n = cfg.n_directions * cfg.n_sources
    lmn = np.zeros((n, 3), np.float64)
    flux = np.zeros(n, np.float64)
    if lib().synth_sky(ctypes.byref(c), ctypes.c_void_p(lmn.ctypes.data),
                       ctypes.c_void_p(flux.ctypes.data)) != 0:
        raise RuntimeError("synth_sky failed")
    out = []
    for d in range(cfg.n_directions):
        sl = slice(d * cfg.n_sources, (d + 1) * cfg.n_sources)
        st = np.zeros((cfg.n_sources, 4), np.float64)
        st[:, 0] = flux[sl]
        out.append((np.ascontiguousarray(lmn[sl]), st))
    return out


def gain_sequence(cfg: ObservationConfig, n_intervals, seed=None, phase_sigma=0.05,
                  amp_sigma=0.01, dispersive_sigma=0.05):
    """True gains of `n_intervals` consecutive solution intervals,
    [n_intervals, n_channels, n_stations, n_directions, 2] complex128.

    Interval 0 has the gains of `gains(cfg)`. From one interval to the next,
    per station, direction and polarization the phase takes a Gaussian
    random-walk step (phase_sigma rad) and the log-amplitude one of
    amp_sigma (lognormal drift); per station and direction a dispersive phase
    kappa * nu_mid / nu is added whose coefficient kappa random-walks with
    steps of dispersive_sigma rad (at the band centre nu_mid). Seeded
    numpy PCG64 streams."""
    g0 = gains(cfg)
    rng = np.random.Generator(np.random.PCG64(cfg.seed * 7 + 3 if seed is None else seed))
    freqs = frequencies(cfg)
    nu_mid = 0.5 * (cfg.freq_lo_hz + cfg.freq_hi_hz)
    ns, nd = cfg.n_stations, cfg.n_directions
    phase = np.zeros((ns, nd, 2))
    logamp = np.zeros((ns, nd, 2))
    kappa = np.zeros((ns, nd))
    out = np.zeros((n_intervals,) + g0.shape, np.complex128)
    disp_shape = (nu_mid / freqs)[:, None, None, None]
    for i in range(n_intervals):
        if i > 0:
            phase += rng.normal(0.0, phase_sigma, phase.shape)
            logamp += rng.normal(0.0, amp_sigma, logamp.shape)
            kappa += rng.normal(0.0, dispersive_sigma, kappa.shape)
        drift = np.exp(logamp + 1j * phase)[None, :, :, :]
        disp = np.exp(1j * kappa[None, :, :, None] * disp_shape)
        out[i] = g0 * drift * disp
    return out


def _alloc(shape, pinned):
    if pinned:
        import torch
        return torch.empty(int(np.prod(shape)), dtype=torch.float32,
                           pin_memory=True).view(*shape)
    return np.empty(shape, np.float32)


def _addr(a):
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


@dataclass
class Observation:
    """One solution interval in the regular SolveData layout (XX/YY)."""
    cfg: ObservationConfig
    data: list          # per channel block [n_vis_cb, 2, 2] float32
    model: list         # per channel block [n_dir, n_vis_cb, 2, 2] float32
    antenna1: np.ndarray
    antenna2: np.ndarray
    true_gains: np.ndarray  # [n_channels, n_stations, n_dir, 2]

    def solve_data(self):
        from .solvers import SolveData
        return SolveData.regular(self.data, self.model, self.cfg.n_times,
                                 self.cfg.n_baselines, self.cfg.cb_channels,
                                 self.antenna1, self.antenna2, 2)

    def generic_arrays(self):
        """Per-visibility antenna_pairs / solution_map arrays of the regular
        SolveData constructor (SolveData.cc:129-185)."""
        cfg = self.cfg
        nspd = np.minimum(np.asarray(cfg.nspd), cfg.n_times)
        start = np.concatenate([[0], np.cumsum(nspd)[:-1]])
        ap, sm = [], []
        for nc in cfg.cb_channels:
            a = np.stack([self.antenna1, self.antenna2], 1)
            a = np.repeat(a, nc, axis=0)
            ap.append(np.tile(a, (cfg.n_times, 1)).astype(np.uint32))
            t = np.repeat(np.arange(cfg.n_times), cfg.n_baselines * nc)
            sm.append(np.stack([(t * nspd[d]) // cfg.n_times + start[d]
                                for d in range(cfg.n_directions)]).astype(np.uint32))
        return ap, sm

    def bytes_per_iteration(self):
        return self.cfg.n_vis * 16 * (1 + self.cfg.n_directions)


def observe(cfg: ObservationConfig, true_gains=None, start_time_s=0.0,
            noise_seed=None, pinned=False, with_data=True):
    """Generates one solution interval (model + data) of `cfg`."""
    if true_gains is None:
        true_gains = gains(cfg)
    true_gains = np.ascontiguousarray(true_gains, np.complex128)
    c = cfg.c_config(start_time_s, noise_seed)
    nbl = cfg.n_baselines
    data, model = [], []
    for nc in cfg.cb_channels:
        nv = cfg.n_times * nbl * nc
        data.append(_alloc((nv, 2, 2), pinned) if with_data else None)
        model.append(_alloc((cfg.n_directions, nv, 2, 2), pinned))
    a1 = np.zeros(nbl, np.uint32)
    a2 = np.zeros(nbl, np.uint32)
    n_cb = len(cfg.cb_channels)
    cbs = (ctypes.c_uint32 * n_cb)(*cfg.cb_channels)
    dp = (ctypes.c_void_p * n_cb)(*[_addr(d) if d is not None else None
                                     for d in data])
    mp = (ctypes.c_void_p * n_cb)(*[_addr(m) for m in model])
    rc = lib().synth_observe(ctypes.byref(c), ctypes.c_uint32(n_cb), cbs,
                             ctypes.c_void_p(true_gains.ctypes.data),
                             dp if with_data else None, mp,
                             ctypes.c_void_p(a1.ctypes.data),
                             ctypes.c_void_p(a2.ctypes.data))
    if rc != 0:
        raise RuntimeError(f"synth_observe failed ({rc})")
    return Observation(cfg, data, model, a1, a2, true_gains)
