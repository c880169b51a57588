"""ctypes binding of libddsolve_b200.so (the C ABI in include/ddsolve_b200.h).

The shared library is built in-tree by dp3_b200/build.py. Loading fails loudly
when it is missing: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libddsolve_b200.so")

DDSOLVE_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "call out of order",
          4: "unsupported", 5: "device wait timed out"}

# Every symbol declared in include/ddsolve_b200.h.
EXPORTED_SYMBOLS = (
    "ddsolve_create", "ddsolve_destroy", "ddsolve_last_error",
    "ddsolve_default_settings", "ddsolve_set_settings",
    "ddsolve_set_channel_block", "ddsolve_set_channel_block_regular",
    "ddsolve_solve", "ddsolve_perform_iteration", "ddsolve_stream",
    "ddsolve_set_tuning", "ddsolve_time_stream_kernel",
    "ddsolve_last_launch_count", "ddsolve_perform_iteration_noalloc",
    "ddsolve_perform_iterations", "ddsolve_get_tuning", "ddsolve_set_plan_tuning",
    "ddsolve_autotune", "ddsolve_set_intervals", "ddsolve_solve_batch",
    "ddsolve_set_channel_block_regular_sky", "ddsolve_predict_regular",
    "ddsolve_set_interval_buffers", "ddsolve_add_smoothness_constraint",
    "ddsolve_add_antenna_constraint", "ddsolve_add_reference_antenna_constraint",
    "ddsolve_clear_constraints", "ddsolve_correct_and_subtract",
)


class Dims(ctypes.Structure):
    _fields_ = [("n_antennas", ctypes.c_uint32),
                ("n_directions", ctypes.c_uint32),
                ("n_channel_blocks", ctypes.c_uint32),
                ("n_correlations", ctypes.c_uint32),
                ("n_solution_polarizations", ctypes.c_uint32),
                ("n_solutions_per_direction", ctypes.POINTER(ctypes.c_uint32))]


class Settings(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_uint32),
                ("min_iterations", ctypes.c_uint32),
                ("accuracy", ctypes.c_double),
                ("constraint_accuracy", ctypes.c_double),
                ("step_size", ctypes.c_double),
                ("detect_stalling", ctypes.c_int32),
                ("step_diff_sigma", ctypes.c_double),
                ("phase_only", ctypes.c_int32)]


class Tuning(ctypes.Structure):
    _fields_ = [("use_pipe", ctypes.c_int32),
                ("direction_groups", ctypes.c_uint32),
                ("stages", ctypes.c_uint32),
                ("model_powers", ctypes.c_int32),
                ("gain_buffers", ctypes.c_uint32)]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class Result(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint32),
                ("constraint_iterations", ctypes.c_uint32),
                ("has_converged", ctypes.c_int32),
                ("has_stalled", ctypes.c_int32)]


_lib = None


def lib():
    """Loads the solver library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python dp3_b200/build.py`"
                " (the solver has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, i32 = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                             ctypes.c_int)
        L.ddsolve_create.argtypes = [ctypes.POINTER(Dims), i32,
                                     ctypes.POINTER(vp)]
        L.ddsolve_destroy.argtypes = [vp]
        L.ddsolve_last_error.argtypes = [vp]
        L.ddsolve_last_error.restype = ctypes.c_char_p
        L.ddsolve_default_settings.argtypes = [ctypes.POINTER(Settings)]
        L.ddsolve_default_settings.restype = None
        L.ddsolve_set_settings.argtypes = [vp, ctypes.POINTER(Settings)]
        L.ddsolve_set_channel_block.argtypes = [vp, u32, u64, vp, vp, vp, vp]
        L.ddsolve_set_channel_block_regular.argtypes = [vp, u32, u32, u32, u32,
                                                        vp, vp, vp, vp]
        L.ddsolve_set_channel_block_regular_sky.argtypes = [vp, u32, u32, u32, u32, vp, vp,
                                                            vp, vp, vp, vp]
        L.ddsolve_predict_regular.argtypes = [vp, u32, u32, u32, vp, vp, vp, vp, vp, vp]
        L.ddsolve_set_interval_buffers.argtypes = [vp, vp]
        L.ddsolve_correct_and_subtract.argtypes = [vp, vp, vp, vp, vp]
        L.ddsolve_solve.argtypes = [vp, vp, ctypes.POINTER(Result), vp]
        L.ddsolve_perform_iteration.argtypes = [vp, vp, vp]
        L.ddsolve_perform_iterations.argtypes = [vp, vp, u32, vp]
        L.ddsolve_set_intervals.argtypes = [vp, u32, vp]
        L.ddsolve_solve_batch.argtypes = [vp, vp, vp, vp]
        L.ddsolve_add_smoothness_constraint.argtypes = [vp, ctypes.POINTER(Smoothness)]
        L.ddsolve_add_antenna_constraint.argtypes = [vp, u32, vp, vp]
        L.ddsolve_add_reference_antenna_constraint.argtypes = [vp]
        L.ddsolve_clear_constraints.argtypes = [vp]
        L.ddsolve_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.ddsolve_set_plan_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.ddsolve_autotune.argtypes = [vp, u32, ctypes.POINTER(Tuning),
                                       ctypes.POINTER(ctypes.c_float)]
        L.ddsolve_stream.argtypes = [vp]
        L.ddsolve_stream.restype = vp
        L.ddsolve_set_tuning.argtypes = [vp, u32, u32]
        L.ddsolve_time_stream_kernel.argtypes = [vp, u32,
                                                 ctypes.POINTER(ctypes.c_float)]
        L.ddsolve_last_launch_count.argtypes = [vp]
        L.ddsolve_last_launch_count.restype = u64
        _lib = L
    return _lib


def default_settings():
    s = Settings()
    lib().ddsolve_default_settings(ctypes.byref(s))
    return s


def _addr(a):
    """Address of a numpy array or of a torch tensor (host or CUDA)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


def _is_torch(a):
    return hasattr(a, "data_ptr") and hasattr(a, "is_cuda")


class SkyDirection(ctypes.Structure):
    """ddsolve_sky_direction (include/ddsolve_b200.h)."""
    _fields_ = [("n_sources", ctypes.c_uint32), ("lmn", ctypes.c_void_p),
                ("stokes", ctypes.c_void_p)]


class Smoothness(ctypes.Structure):
    """ddsolve_smoothness (include/ddsolve_b200.h)."""
    _fields_ = [("frequencies", ctypes.c_void_p), ("bandwidth_hz", ctypes.c_double),
                ("bandwidth_ref_frequency_hz", ctypes.c_double),
                ("spectral_exponent", ctypes.c_double), ("kernel_truncation", ctypes.c_int32),
                ("weights", ctypes.c_void_p), ("sub_solution_weights", ctypes.c_void_p),
                ("antenna_factors", ctypes.c_void_p), ("dd_factors", ctypes.c_void_p)]


class SubtractBuffers(ctypes.Structure):
    """ddsolve_subtract_buffers (include/ddsolve_b200.h)."""
    _fields_ = [("n_times", ctypes.c_uint32), ("n_baselines", ctypes.c_uint32),
                ("n_channels", ctypes.c_uint32), ("antenna1", ctypes.c_void_p),
                ("antenna2", ctypes.c_void_p), ("data", ctypes.c_void_p),
                ("models", ctypes.c_void_p), ("frequencies", ctypes.c_void_p),
                ("station_uvw", ctypes.c_void_p), ("sky", ctypes.c_void_p)]


class IntervalBuffers(ctypes.Structure):
    """ddsolve_interval_buffers (include/ddsolve_b200.h)."""
    _fields_ = [("n_times", ctypes.c_uint32), ("n_baselines", ctypes.c_uint32),
                ("n_channels", ctypes.c_uint32), ("antenna1", ctypes.c_void_p),
                ("antenna2", ctypes.c_void_p), ("data", ctypes.c_void_p),
                ("weights", ctypes.c_void_p), ("flags", ctypes.c_void_p),
                ("model", ctypes.c_void_p), ("frequencies", ctypes.c_void_p),
                ("station_uvw", ctypes.c_void_p), ("sky", ctypes.c_void_p),
                ("linear_weighting", ctypes.c_int32)]


def _interval_struct(antenna1, antenna2, data, model, frequencies, station_uvw, sky,
                     subtract=False):
    """ddsolve_interval_buffers (or with subtract=True ddsolve_subtract_buffers,
    one model pointer per direction) of numpy arrays, weights and flags unset,
    and the arrays it points into."""
    a1 = np.ascontiguousarray(antenna1, dtype=np.uint32)
    a2 = np.ascontiguousarray(antenna2, dtype=np.uint32)
    keep = [a1, a2]
    ib = SubtractBuffers() if subtract else IntervalBuffers()
    if data is not None:
        n_times, n_baselines, n_channels, _ = data.shape
        keep.append(data)
        ib.data = data.ctypes.data
    else:
        _, n_times, n_baselines, n_channels, _ = np.shape(model)
    ib.n_times, ib.n_baselines, ib.n_channels = n_times, n_baselines, n_channels
    ib.antenna1, ib.antenna2 = a1.ctypes.data, a2.ctypes.data
    if model is not None:
        model = np.ascontiguousarray(model, np.complex64)
        keep.append(model)
        if subtract:
            ptrs = (ctypes.c_void_p * len(model))(*[m.ctypes.data for m in model])
            keep.append(ptrs)
            ib.models = ctypes.cast(ptrs, ctypes.c_void_p).value
        else:
            ib.model = model.ctypes.data
    elif sky is not None:
        freqs = np.ascontiguousarray(frequencies, np.float64)
        uvw = np.ascontiguousarray(station_uvw, np.float64)
        sky_arr, sk = _sky_struct(sky)
        keep += [freqs, uvw, sky_arr, sk]
        ib.frequencies, ib.station_uvw = freqs.ctypes.data, uvw.ctypes.data
        ib.sky = ctypes.cast(sky_arr, ctypes.c_void_p).value
    # (neither model nor sky: the library refuses the call)
    return ib, keep


def _sky_struct(sky):
    """ddsolve_sky_direction array of [(lmn [n][3], stokes [n][4]), ...]."""
    keep = []
    arr = (SkyDirection * len(sky))()
    for d, (lmn, stokes) in enumerate(sky):
        lmn = np.ascontiguousarray(lmn, np.float64).reshape(-1, 3)
        stokes = np.ascontiguousarray(stokes, np.float64).reshape(-1, 4)
        assert lmn.shape[0] == stokes.shape[0]
        keep += [lmn, stokes]
        arr[d] = SkyDirection(lmn.shape[0], lmn.ctypes.data, stokes.ctypes.data)
    return arr, keep


class Context:
    """Owns one ddsolve_ctx (one CUDA stream on one device)."""

    def __init__(self, n_antennas, n_solutions_per_direction, n_channel_blocks,
                 n_correlations, n_pol, device=0):
        self._nspd = np.ascontiguousarray(n_solutions_per_direction,
                                          dtype=np.uint32)
        self.n_antennas = int(n_antennas)
        self.n_directions = len(self._nspd)
        self.n_channel_blocks = int(n_channel_blocks)
        self.n_correlations = int(n_correlations)
        self.n_pol = int(n_pol)
        self.n_sub = int(self._nspd.sum())
        dims = Dims(self.n_antennas, self.n_directions, self.n_channel_blocks,
                    self.n_correlations, self.n_pol,
                    self._nspd.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        h = ctypes.c_void_p()
        rc = lib().ddsolve_create(ctypes.byref(dims), int(device),
                                  ctypes.byref(h))
        if rc != DDSOLVE_OK:
            raise RuntimeError("ddsolve_create: "
                               + lib().ddsolve_last_error(None).decode())
        self._h = h
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().ddsolve_destroy(self._h)
            self._h = None
            self._tstream = None  # wrapped the destroyed stream

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != DDSOLVE_OK:
            msg = lib().ddsolve_last_error(self._h).decode()
            raise RuntimeError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")

    @property
    def handle(self):
        return self._h

    def stream_ptr(self):
        return lib().ddsolve_stream(self._h)

    def _after_current_stream(self, t):
        """Orders this context's stream after torch's current stream on the
        device of CUDA tensor `t` (which may have pending writes there), and
        returns (this stream, the current stream) as torch streams."""
        import torch
        ts = getattr(self, "_tstream", None)
        if ts is None:
            ts = self._tstream = torch.cuda.ExternalStream(self.stream_ptr(), device=t.device)
        cur = torch.cuda.current_stream(t.device)
        ts.wait_stream(cur)
        return ts, cur

    def set_settings(self, settings):
        self._check(lib().ddsolve_set_settings(self._h, ctypes.byref(settings)),
                    "ddsolve_set_settings")

    def set_tuning(self, direction_groups=0, max_slab_times=0):
        self._check(lib().ddsolve_set_tuning(self._h, direction_groups,
                                             max_slab_times), "ddsolve_set_tuning")

    def set_channel_block(self, cb, data, model, antenna_pairs, solution_map):
        data = np.ascontiguousarray(data, dtype=np.float32)
        model = np.ascontiguousarray(model, dtype=np.float32)
        ap = np.ascontiguousarray(antenna_pairs, dtype=np.uint32)
        sm = np.ascontiguousarray(solution_map, dtype=np.uint32)
        n_vis = data.shape[0] if data.ndim else 0
        self._check(lib().ddsolve_set_channel_block(
            self._h, cb, n_vis, _addr(data), _addr(model), _addr(ap), _addr(sm)),
            "ddsolve_set_channel_block")

    def set_channel_block_regular(self, cb, n_times, n_baselines, n_channels,
                                  data, model, antenna1, antenna2):
        # Arrays must stay valid until the copy is done: the call synchronises
        # implicitly for pageable memory; pinned arrays are kept alive here.
        a1 = np.ascontiguousarray(antenna1, dtype=np.uint32)
        a2 = np.ascontiguousarray(antenna2, dtype=np.uint32)
        data = _host_buffer(data)
        model = _host_buffer(model)
        self._keep[cb] = (data, model)
        self._check(lib().ddsolve_set_channel_block_regular(
            self._h, cb, n_times, n_baselines, n_channels, _ptr_any(data),
            _ptr_any(model), _addr(a1), _addr(a2)),
            "ddsolve_set_channel_block_regular")

    def set_channel_block_regular_sky(self, cb, n_times, n_baselines, data, frequencies,
                                      station_uvw, antenna1, antenna2, sky):
        """ddsolve_set_channel_block_regular_sky: the model predicted on the
        GPU from `sky` (per direction (lmn [n][3], stokes [n][4])) at this
        block's `frequencies`; only `data` is uploaded."""
        freqs = np.ascontiguousarray(frequencies, np.float64)
        uvw = np.ascontiguousarray(station_uvw, np.float64)
        a1 = np.ascontiguousarray(antenna1, dtype=np.uint32)
        a2 = np.ascontiguousarray(antenna2, dtype=np.uint32)
        sky_arr, keep = _sky_struct(sky)
        data = _host_buffer(data)
        self._keep[cb] = (data,)
        self._check(lib().ddsolve_set_channel_block_regular_sky(
            self._h, cb, n_times, n_baselines, len(freqs), _ptr_any(data), _addr(freqs),
            _addr(uvw), _addr(a1), _addr(a2), ctypes.cast(sky_arr, ctypes.c_void_p)),
            "ddsolve_set_channel_block_regular_sky")

    def predict_regular(self, n_times, n_baselines, frequencies, station_uvw, antenna1,
                        antenna2, sky, out=None):
        """ddsolve_predict_regular: model [n_dir][n_times * n_baselines *
        n_channels][n_corr][2] float32 (numpy, or `out`: a contiguous
        float32 torch tensor on the context's GPU)."""
        freqs = np.ascontiguousarray(frequencies, np.float64)
        uvw = np.ascontiguousarray(station_uvw, np.float64)
        a1 = np.ascontiguousarray(antenna1, dtype=np.uint32)
        a2 = np.ascontiguousarray(antenna2, dtype=np.uint32)
        sky_arr, keep = _sky_struct(sky)
        n_vis = n_times * n_baselines * len(freqs)
        if out is None:
            out = np.zeros((len(sky), n_vis, self.n_correlations, 2), np.float32)
        self._check(lib().ddsolve_predict_regular(
            self._h, n_times, n_baselines, len(freqs), _addr(freqs), _addr(uvw), _addr(a1),
            _addr(a2), ctypes.cast(sky_arr, ctypes.c_void_p), _ptr_any(out)),
            "ddsolve_predict_regular")
        return out

    def set_interval_buffers(self, antenna1, antenna2, data, weights, flags=None, model=None,
                             frequencies=None, station_uvw=None, sky=None,
                             linear_weighting=False):
        """ddsolve_set_interval_buffers: one interval in DP3's buffer layout
        (data complex64 [n_t][n_bl][n_ch][4], weights float32 [..][4], flags
        uint8 [..][4] or None, model complex64 [n_dir][n_t][n_bl][n_ch][4] or
        None with frequencies / station_uvw / sky to predict it)."""
        data = np.ascontiguousarray(data, np.complex64)
        weights = np.ascontiguousarray(weights, np.float32)
        ib, keep = _interval_struct(antenna1, antenna2, data, model, frequencies,
                                    station_uvw, sky)
        ib.weights = weights.ctypes.data
        keep.append(weights)
        if flags is not None:
            flags = np.ascontiguousarray(flags, np.uint8)
            keep.append(flags)
            ib.flags = flags.ctypes.data
        ib.linear_weighting = int(linear_weighting)
        self._check(lib().ddsolve_set_interval_buffers(self._h, ctypes.byref(ib)),
                    "ddsolve_set_interval_buffers")

    def correct_and_subtract(self, antenna1, antenna2, solutions, data=None, model=None,
                             frequencies=None, station_uvw=None, sky=None,
                             subtract=True, keep_model=False):
        """ddsolve_correct_and_subtract (DDECal::CorrectAndSubtractModels):
        data complex64 [n_t][n_bl][n_ch][4], model complex64
        [n_dir][n_t][n_bl][n_ch][4] or None with frequencies / station_uvw /
        sky to predict it, solutions complex128 [n_cb][n_ant][n_dir][n_pol].
        Returns (data - sum of corrected models or None, corrected models or
        None) as new arrays."""
        assert data is not None, "the data give the interval's shape"
        data = np.ascontiguousarray(data, np.complex64)
        ib, keep = _interval_struct(antenna1, antenna2, data, model, frequencies,
                                    station_uvw, sky, subtract=True)
        sol = np.ascontiguousarray(solutions, np.complex128)
        assert sol.size == self.n_channel_blocks * self.n_antennas * self.n_directions * \
            self.n_pol
        d_out = np.empty(data.shape, np.complex64) if subtract else None
        m_out = np.empty((self.n_directions,) + data.shape, np.complex64) if keep_model else None
        m_ptrs = None
        if m_out is not None:
            m_ptrs = (ctypes.c_void_p * self.n_directions)(*[m.ctypes.data for m in m_out])
        self._check(lib().ddsolve_correct_and_subtract(
            self._h, ctypes.byref(ib), _addr(sol), _addr(d_out),
            ctypes.cast(m_ptrs, ctypes.c_void_p) if m_ptrs is not None else None),
            "ddsolve_correct_and_subtract")
        del keep
        return d_out, m_out

    def solve(self, solutions, step_magnitudes=None):
        """solutions: complex128 [n_cb, n_ant, n_sub, n_pol], updated in place
        (a numpy array, or a contiguous torch tensor on the host or on the
        context's GPU)."""
        if _is_torch(solutions):
            import torch
            assert solutions.dtype == torch.complex128 and solutions.is_contiguous()
            if solutions.is_cuda:  # the solve returns after its own stream
                self._after_current_stream(solutions)
        else:
            assert solutions.dtype == np.complex128 and solutions.flags.c_contiguous
        res = Result()
        self._check(lib().ddsolve_solve(self._h, _addr(solutions),
                                        ctypes.byref(res),
                                        _addr(step_magnitudes)), "ddsolve_solve")
        return res

    def perform_iteration(self, solutions):
        solutions = np.ascontiguousarray(solutions, dtype=np.complex128)
        nxt = np.empty_like(solutions)
        self._check(lib().ddsolve_perform_iteration(self._h, _addr(solutions),
                                                    _addr(nxt)),
                    "ddsolve_perform_iteration")
        return nxt

    def set_intervals(self, first_channel_block):
        """Independent intervals: channel blocks [first[g], first[g+1])."""
        f = np.ascontiguousarray(first_channel_block, np.uint32)
        self._check(lib().ddsolve_set_intervals(self._h, len(f) - 1, _addr(f)),
                    "ddsolve_set_intervals")
        self.n_intervals = len(f) - 1

    def add_smoothness_constraint(self, frequencies, bandwidth_hz, weights=None,
                                  bandwidth_ref_frequency_hz=0.0, spectral_exponent=-1.0,
                                  kernel_truncation=True, sub_solution_weights=None,
                                  antenna_factors=None, dd_factors=None):
        """Device SmoothnessConstraint (ddsolve_add_smoothness_constraint):
        frequencies [n_cb] Hz; weights [n_ant * n_cb] or sub_solution_weights
        [n_sub][n_ant * n_cb]; antenna_factors [n_ant]; dd_factors [n_sub]."""
        arrays = [None if a is None else np.ascontiguousarray(a, np.float64)
                  for a in (frequencies, weights, sub_solution_weights, antenna_factors,
                            dd_factors)]
        f, w, sw, af, dd = arrays
        s = Smoothness(f.ctypes.data, float(bandwidth_hz), float(bandwidth_ref_frequency_hz),
                       float(spectral_exponent), int(bool(kernel_truncation)),
                       None if w is None else w.ctypes.data,
                       None if sw is None else sw.ctypes.data,
                       None if af is None else af.ctypes.data,
                       None if dd is None else dd.ctypes.data)
        self._check(lib().ddsolve_add_smoothness_constraint(self._h, ctypes.byref(s)),
                    "ddsolve_add_smoothness_constraint")

    def add_antenna_constraint(self, antenna_sets):
        """Device AntennaConstraint over a list of antenna sets."""
        sizes = [len(a) for a in antenna_sets]
        off = np.ascontiguousarray(np.concatenate([[0], np.cumsum(sizes)]), np.uint32)
        members = np.ascontiguousarray(
            np.concatenate([np.asarray(a, np.uint32) for a in antenna_sets])
            if antenna_sets else np.zeros(0, np.uint32), np.uint32)
        self._check(lib().ddsolve_add_antenna_constraint(
            self._h, len(antenna_sets), _addr(off), _addr(members)),
            "ddsolve_add_antenna_constraint")

    def add_reference_antenna_constraint(self):
        """Device phase referencing (Constraint::ApplyReferenceAntenna)."""
        self._check(lib().ddsolve_add_reference_antenna_constraint(self._h),
                    "ddsolve_add_reference_antenna_constraint")

    def clear_constraints(self):
        self._check(lib().ddsolve_clear_constraints(self._h), "ddsolve_clear_constraints")

    def solve_batch(self, solutions, step_magnitudes=None):
        """Solves every interval; solutions [n_cb, ...] updated in place.
        Returns the list of per-interval Results."""
        n = getattr(self, "n_intervals", 1)
        res = (Result * n)()
        self._check(lib().ddsolve_solve_batch(self._h, _addr(solutions), res,
                                              _addr(step_magnitudes)), "ddsolve_solve_batch")
        return list(res)

    def perform_iterations(self, start, n_passes, out=None):
        """n_passes chained PerformIteration passes from `start`; returns
        [n_passes] + start.shape (pass k starts from pass k - 1's output).
        A CUDA torch tensor in gives a CUDA tensor out (no host copies, and
        the call returns without waiting: the passes run on this context's
        stream, ordered after torch's current stream, and the current stream
        is ordered after them); `out` may supply that tensor."""
        streams = None
        if _is_torch(start):
            import torch
            start = start.contiguous()
            if out is None:
                out = torch.empty((n_passes,) + tuple(start.shape), dtype=torch.complex128,
                                  device=start.device)
            if start.is_cuda:
                streams = self._after_current_stream(start)
        else:
            start = np.ascontiguousarray(start, dtype=np.complex128)
            out = np.empty((n_passes,) + start.shape, np.complex128)
        self._check(lib().ddsolve_perform_iterations(self._h, _addr(start), n_passes,
                                                     _addr(out)),
                    "ddsolve_perform_iterations")
        if streams is not None:
            streams[1].wait_stream(streams[0])
        return out

    def autotune(self, launches=5):
        """Times the plan variants on the uploaded data and keeps the fastest
        (cached per process by problem shape). Returns (tuning dict, ms per
        iteration)."""
        t = Tuning()
        ms = ctypes.c_float()
        self._check(lib().ddsolve_autotune(self._h, launches, ctypes.byref(t),
                                           ctypes.byref(ms)), "ddsolve_autotune")
        return t.as_dict(), ms.value

    def tuning(self):
        t = Tuning()
        self._check(lib().ddsolve_get_tuning(self._h, ctypes.byref(t)), "ddsolve_get_tuning")
        return t.as_dict()

    def set_plan_tuning(self, **kw):
        t = Tuning(**{**{"use_pipe": -1, "direction_groups": 0, "stages": 0,
                         "model_powers": -1, "gain_buffers": 0}, **kw})
        self._check(lib().ddsolve_set_plan_tuning(self._h, ctypes.byref(t)),
                    "ddsolve_set_plan_tuning")

    def time_stream_kernel(self, n_launches=10):
        ms = ctypes.c_float()
        self._check(lib().ddsolve_time_stream_kernel(self._h, n_launches,
                                                     ctypes.byref(ms)),
                    "ddsolve_time_stream_kernel")
        return ms.value

    def last_launch_count(self):
        return int(lib().ddsolve_last_launch_count(self._h))


def _host_buffer(a):
    """A contiguous float32 host buffer: numpy array or CPU torch tensor
    (pinned tensors make the upload asynchronous)."""
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous() and not a.is_cuda
        return a
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr_any(a):
    """Address of a contiguous numpy array or CPU torch tensor."""
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)
