"""Surface roughness of the GPU solver's VTK files against the oracle's.

The free-surface creep case (tests/roughness_case.py: gas layers on the x and y sides,
VTK at every increment) is solved by the CUDA path and by the oracle; the
post-processing of the reference's vtk_sweep (restated in creep_modeling_b200.roughness
and pinned to the reference by tests/test_roughness_cpu.py) must give the same Sa, Sz
and slip statistics from both sets of files.  Bar: the VTK files print 9 significant
digits, so each metric must agree within 2e-8 of the largest magnitude it is computed
from (the node coordinates for Sa and Sz, the accumulated slip for the slip statistics).
"""
import numpy as np
import pytest

from creep_modeling_b200 import roughness
from creep_modeling_b200.solver import Solve
from tests import roughness_case

pytestmark = pytest.mark.gpu


def test_roughness_from_gpu_files_matches_oracle(tmp_path, oracle_lib):
    fft, micro = roughness_case.write_case(tmp_path / "deck")
    g = Solve(fft, out_dir=str(tmp_path / "gpu"), mix=1, modal=0, write_files=True)
    g.run()
    g.close()
    o = oracle_lib.OracleSolve(fft, out_dir=str(tmp_path / "oracle"), mix=1, modal=0, write_files=True)
    o.run()
    o.close()
    a = roughness.vtk_sweep(tmp_path / "gpu", micro)
    b = roughness.vtk_sweep(tmp_path / "oracle", micro)
    np.testing.assert_array_equal(a["macrostep"], b["macrostep"])
    coord_scale = float(roughness_case.N + 1)
    slip_scale = float(np.max(np.abs(b["max_slip"])))
    for k, scale in (("sa", coord_scale), ("sz", coord_scale), ("max_slip", slip_scale), ("mean_slip", slip_scale)):
        assert np.max(np.abs(a[k] - b[k])) <= 2e-8 * scale, (k, a[k], b[k])
    assert np.max(b["sa"][:, -1]) > 0.0
