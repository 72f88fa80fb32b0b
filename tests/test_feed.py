"""Two-port feed helpers (host code of the library, no GPU) against the oracle
restatement of cmpMat2.hpp / initialModule.hpp and against textbook identities."""
import numpy as np
import pytest


def _rand_s(rng):
    return [complex(*rng.uniform(-0.6, 0.6, 2)) for _ in range(4)]


def test_lossless_line_abcd_identity(pkg):
    """A matched line of electrical length theta: S11 = S22 = 0, S21 = S12 = e^{-j theta}
    has ABCD [[cos, j Z0 sin], [j sin / Z0, cos]]."""
    Z0, th = 50.0, 0.7
    T = pkg.feed.sparam_to_abcd(0, np.exp(-1j * th), np.exp(-1j * th), 0, Z0)
    ref = np.array([[np.cos(th), 1j * Z0 * np.sin(th)], [1j * np.sin(th) / Z0, np.cos(th)]])
    assert np.abs(T - ref).max() < 1e-14


def test_conversions_match_oracle_and_round_trip(pkg):
    from oracle import microwave as mw
    rng = np.random.default_rng(0)
    for _ in range(50):
        S = _rand_s(rng)
        Z0 = rng.uniform(10, 100)
        T = pkg.feed.sparam_to_abcd(*S, Z0)
        assert np.abs(T - mw.s_to_abcd(*S, Z0)).max() <= 1e-13 * np.abs(T).max()
        back = pkg.feed.abcd_to_sparam(T, Z0)
        assert max(abs(a - b) for a, b in zip(back, S)) < 1e-12
        ref = mw.abcd_to_s(T, Z0)
        assert max(abs(a - b) for a, b in zip(back, ref)) < 1e-13


def test_matrix_product_and_inverse(pkg):
    rng = np.random.default_rng(1)
    X = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
    Y = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
    assert np.abs(pkg.feed.cmat2_mul(X, Y) - X @ Y).max() < 1e-13
    assert np.abs(pkg.feed.cmat2_mul(X, pkg.feed.cmat2_inv(X)) - np.eye(2)).max() < 1e-12


def test_setup_matches_oracle(pkg):
    from oracle import microwave as mw
    rng = np.random.default_rng(2)
    for _ in range(20):
        p = dict(S11_mag=rng.uniform(0, 0.9), S11_arg_deg=rng.uniform(-180, 180), S21_mag=rng.uniform(0.2, 1),
                 S21_arg_deg=rng.uniform(-180, 180), S12_mag=rng.uniform(0.2, 1), S12_arg_deg=rng.uniform(-180, 180),
                 S22_mag=rng.uniform(0, 0.9), S22_arg_deg=rng.uniform(-180, 180), Z0=50.0,
                 phase_pre_deg=rng.uniform(0, 90), omegam=2.67e10, epsr_diele=rng.uniform(1, 4),
                 h0_stab=rng.uniform(0.1, 0.3), dh_stab=rng.uniform(-0.02, 0.02), dl_cable=rng.uniform(0, 0.1))
        S, ph = pkg.feed.sparam_setup(p)
        Sr, phr = mw.sparam_setup(p)
        assert max(abs(a - b) for a, b in zip(S, Sr)) < 1e-11
        assert ph == pytest.approx(phr, rel=1e-14)


def test_errors_where_the_reference_throws(pkg):
    with pytest.raises(pkg.capi.CathodeError):
        pkg.feed.sparam_to_abcd(0.1, 0.0, 0.2, 0.1, 50.0)
    with pytest.raises(pkg.capi.CathodeError):
        pkg.feed.abcd_to_sparam(np.array([[1.0, 0.0], [0.0, -1.0]]), 50.0)
