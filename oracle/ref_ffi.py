"""ctypes binding of the reference-code oracle (oracle/_ref/libddecal_ref.so).

TEST INFRASTRUCTURE ONLY: the reference's own IterativeDiagonalSolver /
IterativeScalarSolver / SolverBase / SolveData (and SmoothnessConstraint,
AntennaConstraint) compiled here from the reference sources, unmodified, by
oracle/Makefile (target _ref/libddecal_ref.so) against the project's
stand-ins for DP3's external headers. Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline legs load it.

The library is built where the reference tree is present (build() compiles
it); elsewhere the prebuilt oracle/_ref/libddecal_ref.so is used as it is.

Input: one regular solution interval (the layout of the reference's regular
SolveData constructor, ddecal/gain_solvers/SolveData.cc:77-188), per channel
block data float32 [n_times * n_baselines * n_ch_cb, ncorr, 2] and model
float32 [n_dir, n_times * n_baselines * n_ch_cb, ncorr, 2], visibility order
time -> baseline -> channel; the channel blocks must be the reference's even
split (block cb = channels [cb n_ch / n_cb, (cb + 1) n_ch / n_cb)).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libddecal_ref.so")
REFERENCE = os.environ.get("DP3_REFERENCE", "/root/reference")

DIAGONAL_DUO, DIAGONAL_FULL, SCALAR_UNI, SCALAR_DUO, SCALAR_FULL, FULL_JONES = range(6)


def available():
    return os.path.exists(LIB_PATH) or os.path.isdir(REFERENCE)


def build(force=False):
    """Compiles _ref/libddecal_ref.so from the reference tree when present."""
    if os.path.isdir(REFERENCE):
        cmd = ["make", "-C", HERE, f"REF={REFERENCE}", "_ref/libddecal_ref.so"]
        if force:
            cmd.insert(1, "-B")
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL)
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing and the reference tree is absent")
    return LIB_PATH


class Problem(ctypes.Structure):
    _fields_ = [("n_antennas", ctypes.c_uint32), ("n_times", ctypes.c_uint32),
                ("n_baselines", ctypes.c_uint32), ("n_channels", ctypes.c_uint32),
                ("n_channel_blocks", ctypes.c_uint32), ("n_directions", ctypes.c_uint32),
                ("n_correlations_in", ctypes.c_uint32),
                ("n_solutions_per_direction", ctypes.POINTER(ctypes.c_uint32)),
                ("antenna1", ctypes.POINTER(ctypes.c_int32)),
                ("antenna2", ctypes.POINTER(ctypes.c_int32)),
                ("data", ctypes.POINTER(ctypes.c_void_p)),
                ("model", ctypes.POINTER(ctypes.c_void_p))]


class Settings(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_uint32), ("min_iterations", ctypes.c_uint32),
                ("accuracy", ctypes.c_double), ("constraint_accuracy", ctypes.c_double),
                ("step_size", ctypes.c_double), ("detect_stalling", ctypes.c_int32),
                ("step_diff_sigma", ctypes.c_double), ("phase_only", ctypes.c_int32)]


class Constraints(ctypes.Structure):
    _fields_ = [("n_antenna_sets", ctypes.c_uint32),
                ("antenna_set_sizes", ctypes.c_void_p),
                ("antenna_set_members", ctypes.c_void_p),
                ("smoothness", ctypes.c_int32), ("bandwidth_hz", ctypes.c_double),
                ("bandwidth_ref_frequency_hz", ctypes.c_double),
                ("spectral_exponent", ctypes.c_double), ("kernel_truncation", ctypes.c_int32),
                ("smoothness_weights", ctypes.c_void_p),
                ("channel_block_frequencies", ctypes.c_void_p),
                ("antenna_factors", ctypes.c_void_p), ("dd_factors", ctypes.c_void_p),
                ("sub_solution_weights", ctypes.c_void_p),
                ("reference_antenna", ctypes.c_int32)]


class Result(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint32), ("constraint_iterations", ctypes.c_uint32),
                ("seconds_packing", ctypes.c_double), ("seconds_solve", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.ref_solve.restype = ctypes.c_int
        L.ref_solve.argtypes = [ctypes.POINTER(Problem), ctypes.POINTER(Settings), ctypes.c_int,
                                ctypes.c_uint32, ctypes.POINTER(Constraints), ctypes.c_void_p,
                                ctypes.POINTER(Result)]
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_prepare.restype = ctypes.c_int
        L.ref_prepare.argtypes = [ctypes.POINTER(Problem), ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_double)]
        L.ref_solve_prepared.restype = ctypes.c_int
        L.ref_solve_prepared.argtypes = [ctypes.c_void_p, ctypes.POINTER(Problem),
                                         ctypes.POINTER(Settings), ctypes.c_uint32,
                                         ctypes.POINTER(Constraints), ctypes.c_void_p,
                                         ctypes.POINTER(Result)]
        L.ref_release.restype = None
        L.ref_release.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def settings(max_iterations=50, min_iterations=0, accuracy=1e-5, constraint_accuracy=1e-4,
             step_size=0.2, detect_stalling=True, step_diff_sigma=0.1, phase_only=False):
    return Settings(max_iterations, min_iterations, accuracy, constraint_accuracy, step_size,
                    int(detect_stalling), step_diff_sigma, int(phase_only))


def kind_of(ncorr, npol):
    if npol == 4:
        assert ncorr == 4, "the full-Jones solver needs 4 correlations"
        return FULL_JONES
    if npol == 2:
        return {2: DIAGONAL_DUO, 4: DIAGONAL_FULL}[ncorr]
    return {1: SCALAR_UNI, 2: SCALAR_DUO, 4: SCALAR_FULL}[ncorr]


def _problem(cfg, antenna1, antenna2, data, model, ncorr):
    """Problem struct of one regular interval and the arrays it points to."""
    n_cb = len(cfg.cb_channels)
    n_ch = sum(cfg.cb_channels)
    for cb, nc in enumerate(cfg.cb_channels):
        if nc != (cb + 1) * n_ch // n_cb - cb * n_ch // n_cb:
            raise ValueError("channel blocks are not the reference's even split")
    nspd = np.ascontiguousarray(cfg.nspd, np.uint32)
    a1 = np.ascontiguousarray(antenna1, np.int32)
    a2 = np.ascontiguousarray(antenna2, np.int32)
    data = [np.ascontiguousarray(d, np.float32) for d in data]
    model = [np.ascontiguousarray(m, np.float32) for m in model]
    dp = (ctypes.c_void_p * n_cb)(*[d.ctypes.data for d in data])
    mp = (ctypes.c_void_p * n_cb)(*[m.ctypes.data for m in model])
    p = Problem(cfg.n_stations, cfg.n_times, cfg.n_baselines, n_ch, n_cb, len(nspd), ncorr,
                nspd.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                a1.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                a2.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                ctypes.cast(dp, ctypes.POINTER(ctypes.c_void_p)),
                ctypes.cast(mp, ctypes.POINTER(ctypes.c_void_p)))
    return p, (nspd, a1, a2, data, model, dp, mp)


def _constraints(antenna_sets, smoothness, cb_frequencies, reference_antenna=False):
    if not (antenna_sets or smoothness or reference_antenna):
        return None, ()
    freqs = np.ascontiguousarray(cb_frequencies, np.float64)
    keep = [freqs]
    cons = Constraints()
    cons.channel_block_frequencies = freqs.ctypes.data
    if antenna_sets:
        sizes = np.array([len(s) for s in antenna_sets], np.uint32)
        members = np.concatenate([np.asarray(s, np.uint32) for s in antenna_sets])
        keep += [sizes, members]
        cons.n_antenna_sets = len(antenna_sets)
        cons.antenna_set_sizes = sizes.ctypes.data
        cons.antenna_set_members = members.ctypes.data
    if smoothness:
        cons.smoothness = 1
        cons.bandwidth_hz = smoothness["bandwidth_hz"]
        cons.bandwidth_ref_frequency_hz = smoothness.get("bandwidth_ref_frequency_hz", 0.0)
        cons.spectral_exponent = smoothness.get("spectral_exponent", -1.0)
        cons.kernel_truncation = int(smoothness.get("kernel_truncation", True))
        for key, field in (("weights", "smoothness_weights"),
                           ("antenna_factors", "antenna_factors"),
                           ("dd_factors", "dd_factors"),
                           ("sub_solution_weights", "sub_solution_weights")):
            if smoothness.get(key) is not None:
                a = np.ascontiguousarray(smoothness[key], np.float64)
                keep.append(a)
                setattr(cons, field, a.ctypes.data)
    cons.reference_antenna = int(bool(reference_antenna))
    return cons, keep


def solve(cfg, antenna1, antenna2, data, model, ncorr, npol, solutions, st, n_threads=1,
          antenna_sets=None, smoothness=None, cb_frequencies=None, reference_antenna=False):
    """Runs the reference's Solve on one regular interval.

    cfg: an ObservationConfig-like object (n_stations, n_times, n_baselines,
    cb_channels, nspd). solutions: complex128 [n_cb, n_ant, n_sub, npol],
    updated in place. antenna_sets: list of antenna-index lists
    (AntennaConstraint); smoothness: dict(bandwidth_hz=...,
    bandwidth_ref_frequency_hz=0, spectral_exponent=-1, kernel_truncation=True)
    (SmoothnessConstraint; optional weights [n_ant * n_cb], antenna_factors
    [n_ant], dd_factors [n_sub], sub_solution_weights [n_sub][n_ant * n_cb]);
    reference_antenna: a last constraint that applies
    Constraint::ApplyReferenceAntenna; cb_frequencies: mean frequency per
    channel block (needed with any constraint). Returns the Result (iterations,
    constraint_iterations, seconds_packing, seconds_solve)."""
    assert solutions.dtype == np.complex128 and solutions.flags.c_contiguous
    p, keep = _problem(cfg, antenna1, antenna2, data, model, ncorr)
    cons, keep_c = _constraints(antenna_sets, smoothness, cb_frequencies, reference_antenna)
    res = Result()
    rc = lib().ref_solve(ctypes.byref(p), ctypes.byref(st), kind_of(ncorr, npol), n_threads,
                         ctypes.byref(cons) if cons is not None else None,
                         solutions.ctypes.data, ctypes.byref(res))
    if rc != 0:
        raise RuntimeError("ref_solve: " + lib().ref_last_error().decode())
    return res


class Prepared:
    """One interval packed once through the reference's SolveData
    constructor (seconds_packing), then solved with any settings."""

    def __init__(self, cfg, antenna1, antenna2, data, model, ncorr, npol):
        self._p, self._keep = _problem(cfg, antenna1, antenna2, data, model, ncorr)
        self._h = ctypes.c_void_p()
        t = ctypes.c_double()
        rc = lib().ref_prepare(ctypes.byref(self._p), kind_of(ncorr, npol), ctypes.byref(self._h),
                               ctypes.byref(t))
        if rc != 0:
            raise RuntimeError("ref_prepare: " + lib().ref_last_error().decode())
        self.seconds_packing = t.value

    def solve(self, solutions, st, n_threads=1):
        assert solutions.dtype == np.complex128 and solutions.flags.c_contiguous
        res = Result()
        rc = lib().ref_solve_prepared(self._h, ctypes.byref(self._p), ctypes.byref(st),
                                      n_threads, None, solutions.ctypes.data, ctypes.byref(res))
        if rc != 0:
            raise RuntimeError("ref_solve_prepared: " + lib().ref_last_error().decode())
        return res

    def close(self):
        if self._h:
            lib().ref_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def perform_iteration(cfg, antenna1, antenna2, data, model, ncorr, npol, solutions,
                      n_threads=1):
    """One reference PerformIteration: Solve with max_iterations = 1 and step
    size 1, so that Step leaves next_solutions unchanged (SolverBase.cc:107-110:
    sol * 0 + next * 1) and AssignSolutions copies them out."""
    out = np.ascontiguousarray(solutions, np.complex128).copy()
    solve(cfg, antenna1, antenna2, data, model, ncorr, npol, out,
          settings(max_iterations=1, step_size=1.0, detect_stalling=False), n_threads)
    return out
