"""ctypes binding of the CPU oracle (oracle/ddecal_oracle.{h,cc}).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA solver. Only tests/,
__graft_entry__.smoke() and the CPU-baseline legs of bench.py import it.

Problem layout (identical to the reference SolveData, see
ddecal/gain_solvers/SolveData.h:28-194):
  per channel block: data float32 [n_vis, ncorr, 2], model float32
  [n_dir, n_vis, ncorr, 2], antenna_pairs uint32 [n_vis, 2], solution_map
  uint32 [n_dir, n_vis]; solutions complex128 [n_cb, n_ant, n_sub, n_pol].
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build(force=False):
    """Compile liboracle.so with g++ (portable x86-64-v3 code)."""
    src = os.path.join(HERE, "ddecal_oracle.cc")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    subprocess.check_call(["make", "-C", HERE, "liboracle.so"])
    return LIB_PATH


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


class ChannelBlock(ctypes.Structure):
    _fields_ = [("n_vis", ctypes.c_uint64),
                ("data", ctypes.c_void_p),
                ("model", ctypes.c_void_p),
                ("antenna_pairs", ctypes.c_void_p),
                ("solution_map", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint32),
                ("constraint_iterations", ctypes.c_uint32),
                ("has_converged", ctypes.c_int32),
                ("has_stalled", ctypes.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_solve.restype = ctypes.c_int
        _lib.oracle_perform_iteration.restype = ctypes.c_int
        _lib.oracle_solver_tester_fill.restype = ctypes.c_int
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _marshal(problem):
    """Returns (dims, cb_array, keepalive) for a problem dict."""
    nspd = np.ascontiguousarray(problem["n_solutions_per_direction"],
                                dtype=np.uint32)
    dims = Dims(problem["n_antennas"], len(nspd), len(problem["data"]),
                problem["n_correlations"], problem["n_pol"],
                nspd.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    cbs = (ChannelBlock * len(problem["data"]))()
    for i in range(len(problem["data"])):
        d = problem["data"][i]
        cbs[i] = ChannelBlock(d.shape[0], d.ctypes.data,
                              problem["model"][i].ctypes.data,
                              problem["antenna_pairs"][i].ctypes.data,
                              problem["solution_map"][i].ctypes.data)
    return dims, cbs, nspd


def settings(max_iterations=50, min_iterations=0, accuracy=1e-5,
             constraint_accuracy=1e-4, step_size=0.2, detect_stalling=True,
             step_diff_sigma=0.1, phase_only=False):
    return Settings(max_iterations, min_iterations, accuracy,
                    constraint_accuracy, step_size, int(detect_stalling),
                    step_diff_sigma, int(phase_only))


def solve(problem, solutions, st, precision=32, n_threads=None):
    """Runs the restated IterativeDiagonal/ScalarSolver::Solve.

    solutions: complex128 array [n_cb, n_ant, n_sub, n_pol], updated in place.
    Returns (Result, step_magnitudes ndarray)."""
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    dims, cbs, keep = _marshal(problem)
    assert solutions.dtype == np.complex128 and solutions.flags.c_contiguous
    mags = np.zeros(max(1, st.max_iterations), dtype=np.float64)
    res = Result()
    rc = lib().oracle_solve(ctypes.byref(dims), ctypes.byref(st), cbs,
                            precision, n_threads, _ptr(solutions), _ptr(mags),
                            ctypes.byref(res))
    if rc != 0:
        raise RuntimeError("oracle_solve failed: unsupported combination")
    n_it = min(res.iterations, st.max_iterations)
    return res, mags[:max(n_it, 0)].copy()


def perform_iteration(problem, solutions, precision=32, n_threads=None):
    """One PerformIteration on all channel blocks; returns next solutions."""
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    dims, cbs, keep = _marshal(problem)
    solutions = np.ascontiguousarray(solutions, dtype=np.complex128)
    nxt = np.empty_like(solutions)
    rc = lib().oracle_perform_iteration(ctypes.byref(dims), cbs, precision,
                                        n_threads, _ptr(solutions), _ptr(nxt))
    if rc != 0:
        raise RuntimeError("oracle_perform_iteration failed")
    return nxt


# SolverTester sizes (ddecal/test/unit/SolverTester.h:103-125)
TESTER_N_ANTENNAS = 50
TESTER_N_DIRECTIONS = 3
TESTER_N_CHANNEL_BLOCKS = 4
TESTER_N_TIMES = 50
TESTER_N_BASELINES = 50 * 49 // 2
TESTER_DD_SOLUTIONS = (1, 2, 5)


def solver_tester_problem(diagonal, dd_intervals, n_correlations):
    """SolverTester::FillDdIntervalData + regular SolveData, restated.

    Returns (problem dict, true gains complex128 [n_ant, n_sub, 2],
    unit initial solutions)."""
    nspd = TESTER_DD_SOLUTIONS if dd_intervals else (1, 1, 1)
    n_sub = sum(nspd)
    n_vis = TESTER_N_TIMES * TESTER_N_BASELINES * 4
    ncb = TESTER_N_CHANNEL_BLOCKS
    data = [np.zeros((n_vis, n_correlations, 2), np.float32) for _ in range(ncb)]
    model = [np.zeros((3, n_vis, n_correlations, 2), np.float32)
             for _ in range(ncb)]
    ant = [np.zeros((n_vis, 2), np.uint32) for _ in range(ncb)]
    smap = [np.zeros((3, n_vis), np.uint32) for _ in range(ncb)]
    inp = np.zeros((TESTER_N_ANTENNAS, n_sub, 2), np.complex128)

    def arr(lst, ctype):
        a = (ctypes.POINTER(ctype) * ncb)()
        for i, x in enumerate(lst):
            a[i] = x.ctypes.data_as(ctypes.POINTER(ctype))
        return a

    rc = lib().oracle_solver_tester_fill(
        int(diagonal), int(dd_intervals), n_correlations,
        arr(data, ctypes.c_float), arr(model, ctypes.c_float),
        arr(ant, ctypes.c_uint32), arr(smap, ctypes.c_uint32), _ptr(inp))
    if rc != 0:
        raise RuntimeError("oracle_solver_tester_fill failed")
    n_pol = 2 if diagonal else 1
    problem = dict(n_antennas=TESTER_N_ANTENNAS, n_correlations=n_correlations,
                   n_pol=n_pol, n_solutions_per_direction=list(nspd),
                   data=data, model=model, antenna_pairs=ant, solution_map=smap)
    init = np.ones((ncb, TESTER_N_ANTENNAS, n_sub, n_pol), np.complex128)
    return problem, inp, init
