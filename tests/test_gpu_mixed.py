"""Mixed precision against the plain FP64 path on the same deck.

The mixed path keeps the equilibrium iteration's spectrum, FFTs and
Green-operator application in FP32 and everything else (local Newton,
reductions, F and rotation updates) in FP64.  Bar: every macroscopic tensor
curve of results.csv (average strain, stress, plastic strain, elastic strain,
velocity gradient and plastic strain rate; six components each) within 1e-4 of
the FP64 path, relative to the largest magnitude of its tensor over the run
(components held near zero by the boundary conditions are compared on the
tensor's scale, as the parity tests do); the
per-voxel von Mises stress within 1e-3 relative to its largest value (the
stated field tolerance).  Case: a two-phase creep polycrystal (5 vol % stiff
elastic spheres), the mixed-precision configuration at a size the test runs
in seconds.
"""
import numpy as np
import pytest

from creep_modeling_b200 import decks
from creep_modeling_b200.solver import Solve
from tests.parity import RESULT_GROUPS

pytestmark = pytest.mark.gpu

CURVE_TOL = 1e-4
FIELD_TOL = 1e-3


def _run(fft, precision, nsteps):
    s = Solve(fft, mix=1, modal=0, precision=precision)
    rows = []
    for _ in range(nsteps):
        assert s.advance(1) == 1
        rows.append(s.rows()[0])
    sg = s.field("sg").reshape(-1, 9)
    s.close()
    return np.array(rows), sg


def _vm(sg):
    s = sg.reshape(-1, 3, 3)
    dev = s - np.trace(s, axis1=1, axis2=2)[:, None, None] * np.eye(3) / 3.0
    return np.sqrt(1.5 * np.einsum("nij,nij->n", dev, dev))


def test_mixed_precision_curves_and_fields(tmp_path):
    case = decks.case_c3(stress33=150.0, nsteps=6, n=24, ngrains=40)
    fft = decks.write_case(case, tmp_path)
    r64, sg64 = _run(fft, 0, 6)
    r32, sg32 = _run(fft, 1, 6)
    errs = {}
    for grp in RESULT_GROUPS:
        scale = np.max(np.abs(r64[:, grp]))
        if scale < 1e-30:
            continue
        errs[grp[0]] = float(np.max(np.abs(r32[:, grp] - r64[:, grp])) / scale)
    print("curve errors by tensor (first column index):", errs)
    assert max(errs.values()) <= CURVE_TOL, errs
    vm64, vm32 = _vm(sg64), _vm(sg32)
    ferr = float(np.max(np.abs(vm32 - vm64)) / np.max(vm64))
    print("von Mises field error:", ferr)
    assert ferr <= FIELD_TOL


@pytest.mark.parametrize("igamma", [1, 2])
def test_mixed_precision_discrete_green(tmp_path, igamma):
    """The tabulated IGAMMA 1 / 2 operator read into the FP32 Green step: same bars."""
    case = decks.case_c3(stress33=150.0, nsteps=4, n=16, ngrains=20)
    case.processes[0].igamma = igamma
    fft = decks.write_case(case, tmp_path)
    r64, sg64 = _run(fft, 0, 4)
    r32, sg32 = _run(fft, 1, 4)
    for grp in RESULT_GROUPS:
        scale = np.max(np.abs(r64[:, grp]))
        if scale >= 1e-30:
            assert np.max(np.abs(r32[:, grp] - r64[:, grp])) / scale <= CURVE_TOL, grp
    vm64, vm32 = _vm(sg64), _vm(sg32)
    assert np.max(np.abs(vm32 - vm64)) / np.max(vm64) <= FIELD_TOL
