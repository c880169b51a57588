"""CPU tests of the C ABI library: it loads, exports every symbol that
include/*.h declares, and fails loudly (no CPU fallback) without a GPU."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(ddsolve_\w+)\s*\(", text,
                             flags=re.M):
            syms.add(m.group(1))
    return syms


def test_header_declares_expected_entry_points():
    from dp3_b200 import ddsolve
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    assert set(ddsolve.EXPORTED_SYMBOLS) <= declared


def test_library_exports_every_declared_symbol(built):
    from dp3_b200 import ddsolve
    lib = ctypes.CDLL(ddsolve.LIB_PATH)
    missing = [s for s in sorted(_declared_symbols()) if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", ddsolve.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert _declared_symbols() <= exported


def test_default_settings_match_solverbase(built):
    # SolverBase::SolverBase (ddecal/gain_solvers/SolverBase.cc:27-39)
    from dp3_b200 import ddsolve
    s = ddsolve.default_settings()
    assert s.max_iterations == 100 and s.min_iterations == 0
    assert s.accuracy == 1e-5 and s.constraint_accuracy == 1e-4
    assert s.step_size == 0.2 and s.detect_stalling == 1
    assert s.step_diff_sigma == 0.1 and s.phase_only == 0


def test_create_rejects_bad_dims(built):
    from dp3_b200 import ddsolve
    nspd = (ctypes.c_uint32 * 2)(1, 1)
    h = ctypes.c_void_p()
    # unsupported combination (1 correlation with a diagonal solver)
    dims = ddsolve.Dims(10, 2, 1, 1, 2, ctypes.cast(nspd, ctypes.POINTER(ctypes.c_uint32)))
    rc = ddsolve.lib().ddsolve_create(ctypes.byref(dims), 0, ctypes.byref(h))
    assert rc == 4 and not h.value
    dims = ddsolve.Dims(1, 2, 1, 2, 2, ctypes.cast(nspd, ctypes.POINTER(ctypes.c_uint32)))
    rc = ddsolve.lib().ddsolve_create(ctypes.byref(dims), 0, ctypes.byref(h))
    assert rc == 1
    assert ddsolve.lib().ddsolve_last_error(None)


def test_no_cpu_fallback_without_gpu(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dp3_b200 import ddsolve
    with pytest.raises(RuntimeError, match="ddsolve_create"):
        ddsolve.Context(10, [1, 1], 2, 2, 2)
