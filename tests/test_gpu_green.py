"""evp_green_apply (the C-ABI Green-operator entry point) against the oracle."""
import ctypes

import numpy as np
import pytest

from tests import green_cases

pytestmark = pytest.mark.gpu


def _apply(tau, shape, c0, s0):
    import torch

    from creep_modeling_b200 import _lib

    L = _lib.load()
    t = torch.from_numpy(tau).cuda()
    out = torch.empty_like(t)
    p = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    c, s = np.ascontiguousarray(c0.reshape(-1)), np.ascontiguousarray(s0.reshape(-1))
    rc = L.evp_green_apply(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(out.data_ptr()), *shape, p(c), p(s), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 16, 16), (24, 20, 12), (8, 8, 1)])
def test_green_apply_matches_oracle(oracle_lib, shape):
    c0, s0 = green_cases.medium(oracle_lib)
    rng = np.random.default_rng(3)
    tau = rng.standard_normal((9, int(np.prod(shape))))
    got = _apply(tau, shape, c0, s0)
    ref = oracle_lib.green_apply(tau, shape, c0, s0)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_green_apply_compatible_field(oracle_lib):
    c0, s0 = green_cases.medium(oracle_lib)
    tau, grad = green_cases.compatible_field((16, 12, 8), c0)
    got = _apply(tau, (16, 12, 8), c0, s0)
    assert np.max(np.abs(got + grad)) <= 1e-12 * np.max(np.abs(grad))
