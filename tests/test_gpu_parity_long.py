"""Parity at the configurations the solver is used and measured on, against the CPU FP64 oracle.

Same bar as tests/test_gpu_parity.py: identical equilibrium iteration counts per
macrostep, 1e-8 relative on every results.csv column (tensor columns on their
tensor's scale), 1e-6 on diagnostics.csv, 1e-8 on every per-voxel field.

* configuration 1 over its full length: 16^3 creep, 64 grains, 100 increments;
* the benchmarked 64^3 tension deck (500 grains, n = 20, lattice rotation and
  grid update) for its first three increments;
* decks written by the reference's own simulation-case templates
  (utils/sim_cases/creep_calibration.py: 17 processes, a stress ramp then creep
  holds whose time step is cut and ramped back by the ictrl = -1 control;
  utils/sim_cases/tension.py: 6 processes) on a 16^3 sample of the shipped
  micro1.dat, run to their end: the process switch (LS-EVPFFT.f90:188-207), the
  sub-stepping with rollback (378-427) and the dt ramp (557-581) on the GPU;
* mixed precision against the oracle (not only against the FP64 GPU path) on a
  two-phase creep deck with the isotropic stiff phase: curves within 1e-4,
  per-voxel von Mises stress within 1e-3.
"""
import numpy as np
import pytest

from creep_modeling_b200 import decks
from tests import parity, ref_decks
from tests.test_gpu_parity import FIELDS

pytestmark = pytest.mark.gpu


def _check_fields(g, o, names=FIELDS):
    bad = {f: e for f in names if (e := parity.field_rel_err(g, o, f)) > parity.RTOL}
    assert not bad, bad


def test_creep16_full_length(tmp_path):
    """Configuration 1: 16^3 creep, 64 grains, 100 increments of 10 s, tolerance 1e-5."""
    fft = decks.write_case(decks.case_c1(nsteps=100), tmp_path)
    g, o, rg, ro, dg, do = parity.run_both(fft, 100)
    assert rg.shape[0] == 100
    parity.assert_rows_match(rg, ro, dg, do)
    _check_fields(g, o)


def test_tension64_benchmark_deck(tmp_path):
    """The benchmark workload (64^3, 500 grains, n = 20, udot33 = 1e-3/s, dt = 0.5 s,
    iupdate = 1) for its first three increments."""
    fft = decks.write_case(decks.case_c2(nsteps=3), tmp_path)
    g, o, rg, ro, dg, do = parity.run_both(fft, 3)
    assert rg.shape[0] == 3
    parity.assert_rows_match(rg, ro, dg, do)
    _check_fields(g, o)


@pytest.mark.parametrize("deck", ["creep_calibration_475", "tension"])
def test_reference_template_deck(tmp_path, deck):
    """A deck from the reference's own templates, every process to its end."""
    fft = ref_decks.materialize(deck, tmp_path)
    g, o, rg, ro, dg, do = parity.run_both(fft, 1000)
    assert g.advance(1) == 0 and o.advance(1) == 0  # both finished the deck
    assert len(set(rg[:, 2].astype(int))) > 1  # more than one process ran
    parity.assert_rows_match(rg, ro, dg, do)
    _check_fields(g, o)


def _vm(sg):
    s = sg.reshape(-1, 3, 3)
    dev = s - np.trace(s, axis1=1, axis2=2)[:, None, None] * np.eye(3) / 3.0
    return np.sqrt(1.5 * np.einsum("nij,nij->n", dev, dev))


def test_mixed_precision_against_oracle(tmp_path, oracle_lib):
    """Mixed precision (FP32 spectrum and Green operator) against the FP64 oracle on the
    two-phase creep grammar of the mixed-precision configuration (5 vol % isotropic stiff
    spheres, E = 400 GPa), 16^3, 4 increments."""
    from creep_modeling_b200.solver import Solve

    case = decks.case_c3(stress33=150.0, nsteps=4, n=16, ngrains=20)
    fft = decks.write_case(case, tmp_path)
    g = Solve(fft, mix=1, modal=0, precision=1)
    o = oracle_lib.OracleSolve(fft, mix=1, modal=0)
    rg, ro = [], []
    for _ in range(4):
        assert g.advance(1) == 1 and o.advance(1) == 1
        rg.append(g.rows()[0])
        ro.append(o.rows()[0])
    rg, ro = np.array(rg), np.array(ro)
    for grp in parity.RESULT_GROUPS:
        scale = np.max(np.abs(ro[:, grp]))
        if scale >= 1e-30:
            assert np.max(np.abs(rg[:, grp] - ro[:, grp])) / scale <= 1e-4, grp
    vg, vo = _vm(g.field("sg")), _vm(o.field("sg"))
    assert np.max(np.abs(vg - vo)) / np.max(vo) <= 1e-3
    g.close()
    o.close()
