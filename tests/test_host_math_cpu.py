"""Identities the kernels' arithmetic relies on, checked on the host build of evp_math.cuh.

* k_prologue forms C~^-1 a column at a time from C~'s LU factors (lu_unrolled +
  lu_inverse_column) instead of eliminating [C~ | I] at once (inv_unrolled): the result must be
  the same to the bit, with and without row interchanges.
* k_upd2 rotates the crystal stiffness as Q c66 Q^T with the b-basis rotation Q = rot_b66(a)
  instead of index by index over 3x3x3x3 followed by chg_basis: the same tensor up to rounding,
  also for the non-orthogonal map a = Fe ag.
"""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

SRC = Path(__file__).resolve().parent / "host_math_check.cpp"


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("host_math") / "libhostmath.so"
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out), str(SRC)], check=True)
    L = ctypes.CDLL(str(out))
    L.check_inverse_columns.argtypes = [ctypes.c_int, ctypes.c_uint]
    L.check_inverse_columns.restype = ctypes.c_int
    L.check_rot_b66.argtypes = [ctypes.c_int, ctypes.c_uint]
    L.check_rot_b66.restype = ctypes.c_double
    return L


def test_column_inverse_has_the_bits_of_the_full_elimination(lib):
    assert lib.check_inverse_columns(4000, 7) == 0


def test_b_basis_rotation_equals_the_index_rotation(lib):
    assert lib.check_rot_b66(1000, 11) < 1e-14
