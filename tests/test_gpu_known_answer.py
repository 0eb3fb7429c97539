"""The CUDA path's whole solve on a homogeneous elastic single crystal reproduces the cubic
compliance closed form (tests/single_crystal.py), in plain FP64 and in mixed precision."""
import pytest

from creep_modeling_b200.solver import Solve
from tests import single_crystal as sc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_single_crystal_elastic_known_answer(tmp_path, precision):
    fft = sc.write_deck(tmp_path / "deck")
    s = Solve(fft, out_dir=str(tmp_path / "out"), mix=1, modal=0, csv_only=True, precision=precision)
    s.run()
    s.close()
    sc.check_first_increment(tmp_path / "out" / "results.csv")
