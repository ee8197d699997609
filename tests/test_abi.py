"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares (no compute calls here)."""

from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(jst_\w+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_cb")))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "jst_create" in names and "jst_run" in names and len(names) >= 18


def test_library_exports_all_declared_symbols():
    from purinecfd_b200 import solver
    if not solver.LIB_PATH.exists():
        pytest.fail(f"{solver.LIB_PATH} not built")
    lib = ctypes.CDLL(str(solver.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_every_export():
    """Every entry point the header declares is bound by the Python layer
    (the solver module or the batch module), and nothing else is listed."""
    from purinecfd_b200 import batch, solver
    declared = set(declared_functions())
    bound = set(solver.EXPORTS) | set(solver.DEBUG_EXPORTS) | set(batch.BATCH_EXPORTS)
    assert declared == bound, (sorted(declared - bound), sorted(bound - declared))


def test_library_exports_nothing_undeclared():
    """Every jst_* symbol the library exports is declared in include/*.h (the
    public ABI in jst_gpu.h, the test hooks in jst_gpu_debug.h)."""
    import shutil
    import subprocess
    from purinecfd_b200 import solver
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-D", "--defined-only", str(solver.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[-1].startswith("jst_")}
    undeclared = sorted(exported - set(declared_functions()))
    assert not undeclared, undeclared


def test_version_string():
    from purinecfd_b200 import solver
    assert b"sm_100a" in solver.lib().jst_version()
