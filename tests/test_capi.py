"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(cth_[A-Za-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols(pkg):
    L = pkg.capi.load()
    names = declared_symbols()
    assert len(names) >= 14
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(pkg.capi.EXPORTS) <= names


def test_version_and_errors(pkg):
    L = pkg.capi.load()
    assert b"sm_100a" in L.cth_version()
    # argument errors are reported without touching a GPU
    h = ctypes.c_void_p()
    ib = (ctypes.c_int * 2)(1, 4)
    rc = L.cth_grid_create(0, 4, ib, ib, 1, 0, ctypes.byref(h))
    assert rc == pkg.capi.CTH_ERR_ARG
    assert "invalid" in pkg.capi.last_error()
