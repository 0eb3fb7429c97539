"""ctypes front end of the CPU FP64 oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference Fortran LS-EVPFFT solver in C++ (see
``evp_oracle.cpp``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` use it, as the checker; the product library never
imports it.  Parity against the Fortran executable itself is UNPINNED (no
Fortran toolchain here); the oracle is pinned by analytic known answers and
numpy/scipy golden vectors in ``tests/golden``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libevp_oracle.so"

RESULTS_COLS = (
    "iter,macrostep,ipr,sim_time,wall_time,tdot,tdot_ref,eav11,eav22,eav33,eav23,eav13,eav12,sav11,sav22,sav33,"
    "sav23,sav13,sav12,epav11,epav22,epav33,epav23,epav13,epav12,eelav11,eelav22,eelav33,eelav23,eelav13,"
    "eelav12,vgrad11,vgrad22,vgrad33,vgrad23,vgrad13,vgrad12,edotp11,edotp22,edotp33,edotp23,edotp13,edotp12,"
    "evm,evmp,dvm,dvmp,svm,gamma,g,geff").split(",")

_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (system g++, OpenMP, strict IEEE)."""
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, env=env)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        c_dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_open.restype = ctypes.c_void_p
        L.oracle_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.oracle_advance.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_advance.restype = ctypes.c_int
        L.oracle_get_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, c_dp, ctypes.c_long]
        L.oracle_get_field.restype = ctypes.c_long
        L.oracle_last_rows.argtypes = [ctypes.c_void_p, c_dp, c_dp]
        L.oracle_total_iters.argtypes = [ctypes.c_void_p]
        L.oracle_total_iters.restype = ctypes.c_long
        L.oracle_grid.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 3
        L.oracle_close.argtypes = [ctypes.c_void_p]
        L.oracle_run.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_char_p, ctypes.c_int]
        for name in ("oracle_chg_basis_t2_to_b6", "oracle_chg_basis_b6_to_t2", "oracle_chg_basis_t4_to_b66",
                     "oracle_chg_basis_b66_to_t4", "oracle_expm_adaptive"):
            getattr(L, name).argtypes = [c_dp, c_dp]
        L.oracle_polar.argtypes = [c_dp, c_dp, c_dp]
        L.oracle_cond1_6x6.argtypes = [c_dp]
        L.oracle_cond1_6x6.restype = ctypes.c_double
        L.oracle_fft3.argtypes = [c_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_plastic_rate.argtypes = [c_dp, c_dp, c_dp, c_dp, ctypes.c_int, c_dp, c_dp, c_dp, c_dp]
        L.oracle_green_apply.argtypes = [c_dp, c_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp, c_dp]
        L.oracle_green_apply.restype = ctypes.c_int
        L.oracle_harden.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, c_dp, c_dp,
                                    ctypes.c_double, c_dp, ctypes.c_double, c_dp]
        L.oracle_harden.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleSolve:
    """One oracle solve; mirrors the executable's start-up and macrostep loop."""

    def __init__(self, fft_in, out_dir="", mix=1, modal=0, nthreads=0, write_files=False):
        err = ctypes.create_string_buffer(512)
        self._h = lib().oracle_open(str(fft_in).encode(), str(out_dir).encode(), int(mix), int(modal), int(nthreads),
                                    int(write_files), err, 512)
        if not self._h:
            raise RuntimeError(f"oracle_open failed: {err.value.decode()}")
        n = [ctypes.c_int() for _ in range(3)]
        lib().oracle_grid(self._h, *[ctypes.byref(x) for x in n])
        self.shape = tuple(x.value for x in n)
        self.nvox = self.shape[0] * self.shape[1] * self.shape[2]

    def advance(self, nmacro=1) -> int:
        r = lib().oracle_advance(self._h, int(nmacro))
        if r < 0:
            raise RuntimeError(f"oracle solve failed with status {r}")
        return r

    def run(self) -> list:
        rows = []
        while self.advance(1) == 1:
            rows.append(self.rows()[0])
        return rows

    def field(self, name: str) -> np.ndarray:
        buf = np.zeros(self.nvox * 128 + 3 * (self.shape[0] + 1) * (self.shape[1] + 1) * (self.shape[2] + 1))
        n = lib().oracle_get_field(self._h, name.encode(), _p(buf), buf.size)
        if n < 0:
            raise KeyError(name)
        return buf[:n].copy()

    def rows(self):
        r = np.zeros(51)
        d = np.zeros(44)
        lib().oracle_last_rows(self._h, _p(r), _p(d))
        return r, d

    def total_iters(self) -> int:
        return int(lib().oracle_total_iters(self._h))

    def close(self):
        if self._h:
            lib().oracle_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_file(fft_in, out_dir, mix=1, modal=0, nthreads=0) -> int:
    err = ctypes.create_string_buffer(512)
    rc = lib().oracle_run(str(fft_in).encode(), str(out_dir).encode(), int(mix), int(modal), int(nthreads), err, 512)
    if rc != 0:
        raise RuntimeError(f"oracle_run failed: {err.value.decode()}")
    return rc


def chg_t2_to_b6(c33):
    c = np.ascontiguousarray(c33, dtype=np.float64).reshape(9)
    out = np.zeros(6)
    lib().oracle_chg_basis_t2_to_b6(_p(c), _p(out))
    return out


def chg_b6_to_t2(b6):
    b = np.ascontiguousarray(b6, dtype=np.float64).reshape(6)
    out = np.zeros(9)
    lib().oracle_chg_basis_b6_to_t2(_p(b), _p(out))
    return out.reshape(3, 3)


def chg_t4_to_b66(c4):
    c = np.ascontiguousarray(c4, dtype=np.float64).reshape(81)
    out = np.zeros(36)
    lib().oracle_chg_basis_t4_to_b66(_p(c), _p(out))
    return out.reshape(6, 6)


def chg_b66_to_t4(b66):
    b = np.ascontiguousarray(b66, dtype=np.float64).reshape(36)
    out = np.zeros(81)
    lib().oracle_chg_basis_b66_to_t4(_p(b), _p(out))
    return out.reshape(3, 3, 3, 3)


def expm(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    out = np.zeros(9)
    lib().oracle_expm_adaptive(_p(a), _p(out))
    return out.reshape(3, 3)


def polar(f):
    f = np.ascontiguousarray(f, dtype=np.float64).reshape(9)
    r = np.zeros(9)
    u = np.zeros(9)
    lib().oracle_polar(_p(f), _p(r), _p(u))
    return r.reshape(3, 3), u.reshape(3, 3)


def cond1(a66):
    a = np.ascontiguousarray(a66, dtype=np.float64).reshape(36)
    return float(lib().oracle_cond1_6x6(_p(a)))


def harden(tau1, thet0, thet1, hard, gamdot, gamma0, crss, tdot):
    """The oracle's harden (various_functions.f90:1439-1491) for one voxel of a one-mode phase:
    new resistances [nsyst, 2] and the new accumulated shear."""
    hard = np.ascontiguousarray(hard, dtype=np.float64)
    gamdot = np.ascontiguousarray(gamdot, dtype=np.float64)
    crss = np.ascontiguousarray(crss, dtype=np.float64)
    n = gamdot.size
    out = np.zeros((n, 2))
    g1 = lib().oracle_harden(n, float(tau1), float(thet0), float(thet1), _p(hard), _p(gamdot), float(gamma0), _p(crss),
                             float(tdot), _p(out))
    return out, g1


def green_apply(tau: np.ndarray, shape, c0: np.ndarray, s0: np.ndarray) -> np.ndarray:
    """Green operator of the reference medium applied to tau[9, N] (x fastest); returns out[9, N]."""
    n1, n2, n3 = shape
    t = np.ascontiguousarray(tau, dtype=np.float64).reshape(9, -1)
    out = np.zeros_like(t)
    c = np.ascontiguousarray(c0, dtype=np.float64).reshape(81)
    s = np.ascontiguousarray(s0, dtype=np.float64).reshape(81)
    rc = lib().oracle_green_apply(_p(t), _p(out), int(n1), int(n2), int(n3), _p(c), _p(s))
    if rc != 0:
        raise RuntimeError("oracle_green_apply failed")
    return out


def fft3(x: np.ndarray, sign=-1) -> np.ndarray:
    """3-D DFT over the last three axes of x[ncomp, n3, n2, n1] (x fastest)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    nc = x.shape[0]
    n3, n2, n1 = x.shape[1:]
    buf = x.view(np.float64).copy()
    lib().oracle_fft3(_p(buf), nc, n1, n2, n3, int(sign))
    return buf.view(np.complex128).reshape(x.shape)
