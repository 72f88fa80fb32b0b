"""The header-only C++ drop-in (include/cathode_solver.hpp) compiles against the
reference-style vector<vector<double>> interface and, on a GPU, solves through
libcathode_b200.so."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "02_cathode-08_modulerev_b200")
SRC = os.path.join(ROOT, "tests", "cxx", "smg_dropin.cpp")


def _build(tmp_path):
    exe = str(tmp_path / "smg_dropin")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           SRC, "-o", exe, "-L", PKG, "-lcathode_b200", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cxx_shim_compiles_and_links(pkg, tmp_path):
    pkg.capi.load()  # the library exists
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cxx_shim_solves(pkg, tmp_path, cuda_device):
    exe = _build(tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    vals = dict(line.split() for line in out.strip().splitlines())
    assert float(vals["smg_relres"]) < 1e-11
    assert float(vals["sor_relres"]) < 1e-9
