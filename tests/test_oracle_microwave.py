"""The microwave oracle reproduces the reference's own coax calibration run.

Golden vectors: tests/golden/coax_er_deg{0,5}.csv, extracted from the
reference's test/校正/result_deg*.csv by tests/golden/make_coax_golden.py.
The CSV holds 6 significant digits, so agreement is expected at ~1e-6.
"""
import csv
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def golden(n):
    g = np.zeros((194, 7), complex)
    ga = np.zeros((194, 7), complex)
    for r in csv.DictReader(open(os.path.join(HERE, "golden", f"coax_er_deg{n}.csv"))):
        i, j = int(r["i"]) - 1, int(r["j"]) - 1
        g[i, j] = float(r["Er(R)"]) + 1j * float(r["Er(I)"])
        ga[i, j] = float(r["Er_anly(R)"]) + 1j * float(r["Er_anly(I)"])
    return g, ga


@pytest.fixture(scope="module")
def coax():
    from oracle import microwave as mw
    p = mw.coax_params()
    s = mw.coax_er_system(p)
    E = mw.solve_c5_direct(s)
    Es, J, port = mw.coax_postprocess(E, p)
    return mw, p, s, Es, J, port


@pytest.mark.parametrize("n", [0, 5])
def test_coax_oracle_matches_reference_fixture(coax, n):
    mw, p, s, Es, J, port = coax
    Er, An = mw.coax_output(Es, J, p, n)
    g, ga = golden(n)
    assert np.linalg.norm(Er - g) / np.linalg.norm(g) < 5e-6
    assert np.max(np.abs(Er - g)) / np.max(np.abs(g)) < 1e-5
    assert np.linalg.norm(An - ga) / np.linalg.norm(ga) < 5e-6
    # the reference's own error against the analytic TEM field (1.04e-4)
    assert abs(np.linalg.norm(g - ga) / np.linalg.norm(ga) - 1.04e-4) < 0.02e-4


def test_coax_port_power(coax):
    mw, p, s, Es, J, port = coax
    assert port["P_fwd"] * port["ratio"] == pytest.approx(p["Pmw"], rel=1e-12)
    assert port["P_ref"] / port["P_fwd"] < 1e-6  # matched line: almost no reflection
