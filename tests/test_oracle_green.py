"""Known answer for the oracle's Green operator (form_G igamma=0 + convolution_with_Goper).

For a compatible periodic strain field grad(u) free of DC and Nyquist content,
Gamma(xi) : c0 : (i xi (x) u(xi)) = -(i xi (x) u(xi)) exactly, because
Gamma_ijkl = -A^{-1}_ik xi_j xi_l with A = c0 : (xi (x) xi).
"""
import numpy as np

from tests import green_cases


def test_green_operator_inverts_compatible_field(oracle_lib):
    orc = oracle_lib
    for shape in ((8, 8, 8), (12, 10, 6)):
        c0, s0 = green_cases.medium(orc)
        tau, grad = green_cases.compatible_field(shape, c0)
        out = orc.green_apply(tau, shape, c0, s0)
        assert np.max(np.abs(out + grad)) <= 1e-12 * np.max(np.abs(grad)), shape


def test_green_operator_zeroes_uniform_field(oracle_lib):
    orc = oracle_lib
    c0, s0 = green_cases.medium(orc)
    tau = np.ones((9, 6 * 6 * 6))
    out = orc.green_apply(tau, (6, 6, 6), c0, s0)
    assert np.max(np.abs(out)) <= 1e-12
