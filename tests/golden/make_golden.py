"""Generates the golden fixtures under tests/golden/ with numpy and scipy.

The reference ships no tests, outputs or golden vectors, and its Fortran build
(FFTW + LAPACK) cannot be compiled here, so the oracle's building blocks are
pinned against independent implementations of the same published algorithms:
  fft.npz    numpy.fft.fftn / ifftn (pocketfft) vs the oracle's mixed-radix DFT
             (stands in for FFTW's C2C plans, fourier_functions.f90:141-170)
  expm.npz   scipy.linalg.expm for the Pade-13 branch and the closed cubic
             Taylor polynomial for the ||A||_1 <= 0.1 branch
             (matrix_exp_adaptive, various_functions.f90:1955-1967)
  polar.npz  scipy.linalg.polar (polar_dcmp / dgesvd, tensor_functions.f90:367-393)
  cond.npz   numpy.linalg.cond(A, 1) bounds for the dgecon estimate (types.f90:710-731)
Run: python tests/golden/make_golden.py
"""
from pathlib import Path

import numpy as np
import scipy.linalg as sla

HERE = Path(__file__).resolve().parent


def main():
    rng = np.random.default_rng(20261203)
    shapes = [(5, 6, 8), (6, 10, 12), (8, 8, 8), (1, 8, 8), (7, 9, 11)]  # (n3, n2, n1)
    fft = {}
    for s in shapes:
        x = rng.standard_normal((2,) + s) + 1j * rng.standard_normal((2,) + s)
        fft[f"x_{s[0]}_{s[1]}_{s[2]}"] = x
        fft[f"y_{s[0]}_{s[1]}_{s[2]}"] = np.fft.fftn(x, axes=(1, 2, 3))
    np.savez_compressed(HERE / "fft.npz", **fft)

    a_small, e_small, a_big, e_big = [], [], [], []
    for _ in range(20):
        a = rng.standard_normal((3, 3))
        a *= rng.uniform(0.01, 0.099) / np.max(np.sum(np.abs(a), axis=0))
        a_small.append(a)
        e_small.append(np.eye(3) + a + a @ a / 2.0 + a @ a @ a / 6.0)
        b = rng.standard_normal((3, 3))
        b *= rng.uniform(0.2, 30.0) / np.max(np.sum(np.abs(b), axis=0))
        a_big.append(b)
        e_big.append(sla.expm(b))
    np.savez_compressed(HERE / "expm.npz", a_small=np.array(a_small), e_small=np.array(e_small), a_big=np.array(a_big),
                        e_big=np.array(e_big))

    fs, rs, us = [], [], []
    for k in range(30):
        if k < 15:
            f = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
        else:
            f = rng.standard_normal((3, 3))
            if np.linalg.det(f) < 0:
                f[:, 0] *= -1
        r, u = sla.polar(f, side="right")
        fs.append(f); rs.append(r); us.append(u)
    np.savez_compressed(HERE / "polar.npz", f=np.array(fs), r=np.array(rs), u=np.array(us))

    mats, conds = [], []
    for k in range(30):
        m = rng.standard_normal((6, 6)) + (6.0 if k % 2 == 0 else 0.5) * np.eye(6)
        mats.append(m)
        conds.append(np.linalg.cond(m, 1))
    np.savez_compressed(HERE / "cond.npz", a=np.array(mats), cond=np.array(conds))
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
