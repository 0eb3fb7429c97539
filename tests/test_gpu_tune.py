"""The FFT tile autotuner and its cache file (the counterpart of the reference's FFTW wisdom).

Opening a solve whose grid the process has not seen times the candidate tiles of the
x-forward, y and z-with-Green-operator passes and keeps the fastest; with a cache file
set they are appended to it, and a later solve of the same grid reads them instead of
timing again.  The tile changes no result: rows with tuned tiles equal the rows with
the occupancy model's tiles (EVP_TUNE=0) exactly.
"""
import numpy as np
import pytest

from creep_modeling_b200 import decks
from creep_modeling_b200.solver import Solve, tune_cache

pytestmark = pytest.mark.gpu


def _rows(fft, n):
    s = Solve(fft, mix=1, modal=0)
    rows = []
    for _ in range(n):
        assert s.advance(1) == 1
        rows.append(s.rows()[0])
    s.close()
    return np.array(rows)


def test_tuned_tiles_are_cached_and_change_nothing(tmp_path, monkeypatch):
    case = decks.case_c1(nsteps=3)
    case.n, case.ngrains = (20, 18, 10), 16  # a grid no other test uses, so this process has not tuned it
    fft = decks.write_case(case, tmp_path / "deck")
    monkeypatch.setenv("EVP_TUNE", "0")
    before = _rows(fft, 3)  # the occupancy model's tiles
    monkeypatch.delenv("EVP_TUNE")
    cache = tmp_path / "tiles" / "fftw_wisdom.save"
    tune_cache(cache)
    try:
        tuned = _rows(fft, 3)
        lines = cache.read_text().splitlines()
        assert len(lines) >= 3 and all(l.startswith("evp-tile ") for l in lines)
        assert {int(l.split()[1]) for l in lines} == {0, 1, 2}  # x forward, y, z with the Green operator
        again = _rows(fft, 3)
        assert cache.read_text().splitlines() == lines  # known: not timed again
    finally:
        tune_cache(None)
    keep = [c for c in range(before.shape[1]) if c != 4]
    np.testing.assert_array_equal(tuned[:, keep], before[:, keep])
    np.testing.assert_array_equal(again[:, keep], before[:, keep])
