"""The written files against the oracle's: results.csv, diagnostics.csv and every VTK file.

A 12^3 tension solve with the lattice-rotation and grid updates and VTK output
at every increment (IWFIELDS = 1, IWSTEP = 1) is written by the CUDA path and
by the oracle.  The two output directories must hold the same file names; in
every VTK file the non-numeric tokens must be identical and each numeric token
must agree within 2e-8 of the largest magnitude in its block (a block is a run
of numbers between keywords: node coordinates, connectivity, one field), which
is the 1e-8 parity bar plus one unit in the ninth printed digit; the CSV files
must match as the parity tests require (wall-clock column excepted).
"""
import re
from pathlib import Path

import numpy as np
import pytest

from creep_modeling_b200 import decks
from creep_modeling_b200.solver import Solve
from tests import parity

pytestmark = pytest.mark.gpu

VTK_TOL = 2e-8
_num = re.compile(r"^[-+]?(\d+\.?\d*|\.\d+)([eEdD][-+]?\d+)?$")


def _blocks(path: Path):
    """(keyword tokens, numeric blocks) of a VTK file."""
    words, blocks, cur = [], [], []
    for tok in path.read_text().split():
        if _num.match(tok):
            cur.append(float(tok.replace("D", "E").replace("d", "e")))
        else:
            if cur:
                blocks.append(np.array(cur))
                cur = []
            words.append(tok)
    if cur:
        blocks.append(np.array(cur))
    return words, blocks


def test_written_files_match_the_oracle(tmp_path, oracle_lib):
    case = decks.case_c2(nsteps=2, n=12, ngrains=10)
    case.processes[0].iwfields = 1
    case.processes[0].iwstep = 1
    fft = decks.write_case(case, tmp_path / "deck")
    out_g, out_o = tmp_path / "gpu", tmp_path / "oracle"
    g = Solve(fft, out_dir=str(out_g), mix=1, modal=0, write_files=True)
    g.run()
    g.close()
    o = oracle_lib.OracleSolve(fft, out_dir=str(out_o), mix=1, modal=0, write_files=True)
    o.run()
    o.close()
    names_g = sorted(p.name for p in out_g.iterdir())
    names_o = sorted(p.name for p in out_o.iterdir())
    assert names_g == names_o
    vtks = [n for n in names_g if n.endswith(".vtk")]
    assert len(vtks) == 3, vtks  # step 0 and both increments
    for name in vtks:
        wg, bg = _blocks(out_g / name)
        wo, bo = _blocks(out_o / name)
        assert wg == wo, name
        assert [len(b) for b in bg] == [len(b) for b in bo], name
        for k, (a, b) in enumerate(zip(bg, bo)):
            scale = max(float(np.max(np.abs(b))), 1e-300)
            assert float(np.max(np.abs(a - b))) <= VTK_TOL * scale, (name, k, wo)
    rg = np.loadtxt(out_g / "results.csv", delimiter=",", skiprows=1, ndmin=2)
    ro = np.loadtxt(out_o / "results.csv", delimiter=",", skiprows=1, ndmin=2)
    dg = np.loadtxt(out_g / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
    do = np.loadtxt(out_o / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
    parity.assert_rows_match(rg, ro, dg, do)
    assert (out_g / "results.csv").read_text().splitlines()[0] == (out_o / "results.csv").read_text().splitlines()[0]
    assert (out_g / "diagnostics.csv").read_text().splitlines()[0] == (out_o / "diagnostics.csv").read_text().splitlines()[0]
    for name in ("results.csv", "diagnostics.csv"):  # every row has the header's field count (pandas reads by name)
        lines = (out_g / name).read_text().splitlines()
        assert {len(r.split(",")) for r in lines} == {len(lines[0].split(","))}, name
