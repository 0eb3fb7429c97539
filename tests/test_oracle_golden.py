"""Pins the CPU oracle's building blocks against numpy/scipy golden vectors and analytic known answers.

The reference ships no golden vectors (it has no tests); these fixtures are
generated by tests/golden/make_golden.py from independent implementations.
"""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def orc(oracle_lib):
    return oracle_lib


def test_fft_matches_numpy(orc):
    z = np.load(GOLD / "fft.npz")
    for key in z.files:
        if not key.startswith("x_"):
            continue
        x = z[key]
        y = z["y_" + key[2:]]
        got = orc.fft3(x, sign=-1)
        assert np.max(np.abs(got - y)) <= 1e-12 * np.max(np.abs(y)), key
        back = orc.fft3(got, sign=+1) / np.prod(x.shape[1:])
        assert np.max(np.abs(back - x)) <= 1e-13 * np.max(np.abs(x)), key


def test_expm_both_branches(orc):
    z = np.load(GOLD / "expm.npz")
    for a, e in zip(z["a_small"], z["e_small"]):
        np.testing.assert_allclose(orc.expm(a), e, rtol=0, atol=1e-15)
    for a, e in zip(z["a_big"], z["e_big"]):
        got = orc.expm(a)
        assert np.max(np.abs(got - e)) <= 1e-12 * np.max(np.abs(e))


def test_polar_matches_scipy(orc):
    z = np.load(GOLD / "polar.npz")
    for f, r, u in zip(z["f"], z["r"], z["u"]):
        R, U = orc.polar(f)
        np.testing.assert_allclose(R, r, atol=1e-12)
        np.testing.assert_allclose(U, u, atol=1e-12 * np.max(np.abs(u)))
        np.testing.assert_allclose(R @ U, f, atol=1e-12 * np.max(np.abs(f)))


def test_cond_estimate_bounds(orc):
    z = np.load(GOLD / "cond.npz")
    for a, c in zip(z["a"], z["cond"]):
        est = orc.cond1(a)
        assert est <= c * (1 + 1e-12)
        assert est >= c / 3.0
    # the estimator is exact on diagonal matrices
    d = np.diag([1.0, 2.0, 4.0, 8.0, 16.0, 32.0])
    assert abs(orc.cond1(d) - 32.0) <= 1e-12


def test_chg_basis_round_trips(orc):
    rng = np.random.default_rng(1)
    for _ in range(10):
        a = rng.standard_normal((3, 3))
        s = 0.5 * (a + a.T)
        b6 = orc.chg_t2_to_b6(s)
        np.testing.assert_allclose(orc.chg_b6_to_t2(b6), s, atol=1e-14)
        # orthonormal basis: the b6 norm equals the Frobenius norm
        assert abs(np.linalg.norm(b6) - np.linalg.norm(s)) <= 1e-14 * np.linalg.norm(s)
        m = rng.standard_normal((6, 6))
        np.testing.assert_allclose(orc.chg_t4_to_b66(orc.chg_b66_to_t4(m)), m, atol=1e-13)
    # the symmetric 4th-order identity maps to the 6x6 identity
    I4 = np.zeros((3, 3, 3, 3))
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for l in range(3):
                    I4[i, j, k, l] = 0.5 * ((i == k) * (j == l) + (i == l) * (j == k))
    np.testing.assert_allclose(orc.chg_t4_to_b66(I4), np.eye(6), atol=1e-15)


def test_power_law_single_slip(orc):
    """gamdot = gamd0 |tau/tauc|^n sign(tau) with tau = S:sigma (plastic_strain_rate)."""
    import math

    s = np.zeros((1, 5))
    s[0, 4] = 1.0  # unit Schmid vector along b-basis component 5 (sigma_12 shear)
    tt = np.array([[100.0, 80.0]])
    for sig5, n in ((50.0, 10.0), (-30.0, 20.0), (120.0, 7.5)):
        sg6 = np.zeros(6)
        sg6[4] = sig5
        e6 = np.zeros(6); d = np.zeros(36); gd = np.zeros(1)
        import ctypes
        p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        orc.lib().oracle_plastic_rate(p(np.ascontiguousarray(s.ravel())), p(np.ascontiguousarray(tt.ravel())),
                                      p(np.array([n])), p(np.array([1e-3])), 1, p(sg6), p(e6), p(d), p(gd))
        tauc = 100.0 if sig5 >= 0 else 80.0
        expect = 1e-3 * abs(sig5 / tauc) ** n * math.copysign(1.0, sig5)
        assert abs(gd[0] - expect) <= 1e-14 * abs(expect)
        assert abs(e6[4] - expect) <= 1e-14 * abs(expect)
        assert abs(d.reshape(6, 6)[4, 4] - n * 1e-3 * abs(sig5 / tauc) ** (n - 1) / tauc) <= 1e-13 * abs(d[28])


def test_single_crystal_elastic_known_answer(orc, tmp_path):
    """The oracle's whole solve on a homogeneous elastic single crystal reproduces the cubic
    compliance (tests/single_crystal.py)."""
    from tests import single_crystal as sc

    fft = sc.write_deck(tmp_path / "deck")
    o = orc.OracleSolve(str(fft), out_dir=str(tmp_path / "out"), mix=1, modal=0, write_files=True)
    o.run()
    o.close()
    sc.check_first_increment(tmp_path / "out" / "results.csv")


def test_harden_is_the_exact_voce_increment(orc):
    """With a latent-hardening matrix of ones, harden's resistance increment is the Voce law's own
    increment tau(G1) - tau(G0), tau(G) = (tau1 + thet1 G)(1 - exp(-thet0 G / tau1)), G the
    accumulated shear (the reference integrates the law exactly over the step)."""
    rng = np.random.default_rng(5)
    tau1, thet0, thet1 = 40.0, 500.0, 20.0
    n = 12
    voce = lambda g: (tau1 + thet1 * g) * (1.0 - np.exp(-thet0 * g / tau1))
    for gamma0, tdot in ((0.0, 10.0), (0.013, 0.5), (0.2, 2.0)):
        gamdot = rng.uniform(-1e-4, 1e-4, n)
        crss = rng.uniform(90.0, 110.0, (n, 2))
        tau, g1 = orc.harden(tau1, thet0, thet1, np.ones((n, n)), gamdot, gamma0, crss, tdot)
        dg = np.sum(np.abs(gamdot)) * tdot
        assert abs(g1 - (gamma0 + dg)) <= 1e-15 * (gamma0 + dg)
        inc = voce(gamma0 + dg) - voce(gamma0)
        assert np.allclose(tau - crss, inc, rtol=1e-10, atol=1e-12 * tau1), (tau - crss, inc)
