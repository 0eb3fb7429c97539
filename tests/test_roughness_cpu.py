"""The surface-roughness restatement against the reference's own vtk_sweep.

tests/golden/roughness_golden.npz holds what the reference's
utils/data_utils.py:vtk_sweep returned on the oracle's VTK files of the free-surface
creep case (tests/roughness_case.py); the oracle writes the same files again here and
creep_modeling_b200.roughness must return the same Sa, Sz and slip statistics.
"""
from pathlib import Path

import numpy as np

from creep_modeling_b200 import roughness
from tests import roughness_case

GOLD = Path(__file__).resolve().parent / "golden" / "roughness_golden.npz"


def test_restatement_matches_reference_vtk_sweep(tmp_path, oracle_lib):
    fft, micro = roughness_case.write_case(tmp_path / "deck")
    o = oracle_lib.OracleSolve(fft, out_dir=str(tmp_path / "out"), mix=1, modal=0, write_files=True)
    o.run()
    o.close()
    got = roughness.vtk_sweep(tmp_path / "out", micro)
    ref = np.load(GOLD)
    np.testing.assert_array_equal(got["macrostep"], ref["macrostep"])
    for k in ("sa", "sz", "max_slip", "mean_slip"):
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-12, atol=1e-15, err_msg=k)
    assert np.max(ref["sa"][:, -1]) > 0.0  # the faces did roughen


def test_face_indices_count_gas_layers():
    phase = np.ones((6, 8, 10), dtype=int)
    phase[:, :, :2] = 2
    phase[:, :, -3:] = 2
    phase[:, :1, :] = 2
    assert roughness.face_indices(phase) == (2, 6, 1, 7)
