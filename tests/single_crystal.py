"""A homogeneous elastic single crystal under uniaxial stress: a known answer of the whole solve.

One grain with Bunge angles (0, 0, 0), the cubic stiffness of configuration 1 (C11 = 250, C12 = 150,
C44 = 120 GPa) and resistances of 1e8 MPa (no slip), held at sigma33 = 150 MPa with the other
stress components free.  The field is homogeneous, so the spectral solve reduces to one material
point and the first increment's average strains are the cubic compliance times the stress:
eps33 = s11 sigma, eps11 = eps22 = s12 sigma with s11 = (C11 + C12) / ((C11 - C12)(C11 + 2 C12)) and
s12 = -C12 / ((C11 - C12)(C11 + 2 C12)), up to the iteration's tolerance (1e-5)."""
from pathlib import Path

import numpy as np

from creep_modeling_b200 import decks

C11, C12, SIGMA = 250000.0, 150000.0, 150.0
S11 = (C11 + C12) / ((C11 - C12) * (C11 + 2.0 * C12))
S12 = -C12 / ((C11 - C12) * (C11 + 2.0 * C12))
TOL = 2e-5  # relative, on the first increment's strains (iteration tolerance 1e-5)


def write_deck(root: Path, n: int = 4) -> Path:
    c = decks.case_c1(nsteps=2)
    c.n, c.ngrains = n, 1
    c.material = decks.Material(c11=C11, c12=C12, tau0f=1e8, tau0b=1e8)
    c.processes[0].stress33 = SIGMA
    fft = decks.write_case(c, root)
    m = np.loadtxt(root / "micro.dat")
    m[:, 0:3] = 0.0  # crystal axes along the sample axes
    np.savetxt(root / "micro.dat", m, fmt=["%.6f"] * 3 + ["%d"] * 5)
    return fft


def check_first_increment(results_csv: Path) -> None:
    import pandas as pd

    r = pd.read_csv(results_csv)
    e11, e22, e33 = (float(r.loc[0, k]) for k in ("eav11", "eav22", "eav33"))
    assert abs(e33 / (S11 * SIGMA) - 1.0) <= TOL, e33
    assert abs(e11 / (S12 * SIGMA) - 1.0) <= TOL, e11
    assert abs(e22 / (S12 * SIGMA) - 1.0) <= TOL, e22
    assert abs(float(r.loc[0, "epav33"])) <= 1e-30  # no slip
