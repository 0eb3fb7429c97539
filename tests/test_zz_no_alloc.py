"""evp_green_apply_noalloc: the Green-operator entry point for callers that cannot allocate device memory.

Such callers (an application whose device memory belongs to another allocator,
or a latency-critical loop that cannot take the device-wide synchronization of
cudaMalloc/cudaFree) pass their own input and output buffers; the library's
scratch is a fixed array inside the library.  This test calls the new entry
point through the C ABI twice in a row, each time on new input, and checks it
against evp_green_apply on the same input within the Green-operator tests'
tolerance (1e-12 relative).  It also checks that a grid beyond the fixed
scratch is refused with a message.  This file is collected last so that a run
stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _medium():
    import oracle
    from tests import green_cases

    return green_cases.medium(oracle)


def _call(fn, tau_dev, out_dev, shape, c0, s0):
    p = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return fn(ctypes.c_void_p(tau_dev.data_ptr()), ctypes.c_void_p(out_dev.data_ptr()), *shape, p(c0), p(s0), None)


# 32^3 (power-of-two passes), 24 x 20 x 12 (radix-3/5 stages, a non-cubic box), 8 x 8 x 1 (a 2-D grid)
# and 33 x 32 x 32, a grid with an odd x edge exactly at the scratch limit:
# (33 / 2 + 1) * 32 * 32 = 17 * 1024 = 17408 half-spectrum points.
SHAPES = [(32, 32, 32), (24, 20, 12), (8, 8, 1), (33, 32, 32)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_noalloc_matches_allocating_entry_twice(shape):
    import torch

    from creep_modeling_b200 import _lib

    L = _lib.load()
    c0, s0 = _medium()
    n = int(np.prod(shape))
    rng = np.random.default_rng(11 + n)
    for call in range(2):
        tau = torch.from_numpy(rng.standard_normal((9, n))).cuda()
        out_ref = torch.empty_like(tau)
        out_new = torch.full_like(tau, float("nan"))
        _lib.check(_call(L.evp_green_apply, tau, out_ref, shape, c0, s0))
        _lib.check(_call(L.evp_green_apply_noalloc, tau, out_new, shape, c0, s0))
        torch.cuda.synchronize()
        a, b = out_new.cpu().numpy(), out_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call
        assert np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b)), call


def test_noalloc_rejects_grid_beyond_scratch():
    import torch

    from creep_modeling_b200 import _lib

    L = _lib.load()
    c0, s0 = _medium()
    shape = (64, 64, 64)
    tau = torch.zeros((9, 8), dtype=torch.float64, device="cuda")  # never read: the size check comes first
    rc = _call(L.evp_green_apply_noalloc, tau, tau, shape, c0, s0)
    assert rc == -7
    assert b"exceeds the fixed scratch" in L.evp_last_error()
