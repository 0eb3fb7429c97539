"""The batching form: many solves of different grid sizes and material parameters advanced together.

Every equilibrium iteration of a batch is one launch per pass over all running members
plus the device-side controller, replayed as a CUDA graph.  Bars:

* each member's results.csv and diagnostics.csv equal its solve alone to 1e-12 relative
  (wall-clock column excepted; in practice the files are identical), for members of
  different grids (power-of-two and radix-3/5 FFTs, a 2-D grid), slip exponents,
  resistances, loadings (creep and tension) and increment counts, and for a
  mixed-precision member;
* two small members against the CPU FP64 oracle: identical iteration counts, every
  results.csv column within 1e-8;
* a member whose phase stiffness is singular stops with -3 while the others finish as
  they do alone.
"""
from pathlib import Path

import numpy as np
import pytest

from creep_modeling_b200 import decks
from creep_modeling_b200.solver import Batch, Solve, load_results
from tests import parity

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _members(root: Path):
    cases = []
    a = decks.case_c1(nsteps=4)
    a.n, a.ngrains = 8, 8
    cases.append(("c8", a, 0))
    b = decks.case_c2(nsteps=3, n=12, ngrains=10)
    cases.append(("t12", b, 0))
    c = decks.case_c1(nsteps=5)
    c.n, c.ngrains = (24, 20, 12), 20
    c.material = decks.Material(nrs=15.0, tau0f=80.0, tau0b=80.0, thet0=300.0)
    cases.append(("c24", c, 0))
    e = decks.case_c1(nsteps=3)
    e.n, e.ngrains = (16, 16, 1), 12
    cases.append(("c2d", e, 0))
    f = decks.case_c3(stress33=150.0, nsteps=3, n=16, ngrains=20)
    cases.append(("mix16", f, 1))
    return [(name, decks.write_case(case, root / name), prec) for name, case, prec in cases]


def _alone(fft, out, prec):
    s = Solve(fft, out_dir=str(out), mix=1, modal=0, csv_only=True, precision=prec)
    s.run()
    s.close()


def _same(a_dir: Path, b_dir: Path):
    for name in ("results.csv", "diagnostics.csv"):
        a = np.loadtxt(a_dir / name, delimiter=",", skiprows=1, ndmin=2)
        b = np.loadtxt(b_dir / name, delimiter=",", skiprows=1, ndmin=2)
        assert a.shape == b.shape, name
        keep = [c for c in range(a.shape[1]) if c != 4]
        a, b = a[:, keep], b[:, keep]
        scale = np.maximum(np.abs(a).max(axis=0), 1e-300)
        assert np.max(np.abs(a - b) / scale) <= TOL, name


def test_batch_members_equal_their_solves_alone(tmp_path):
    members = _members(tmp_path)
    for name, fft, prec in members:
        _alone(fft, tmp_path / f"alone_{name}", prec)
    with Batch() as b:
        slots = [b.add(fft, tmp_path / f"batch_{name}", mix=1, modal=0, precision=prec) for name, fft, prec in members]
        b.run()
        sts = [b.status(s) for s in slots]
    for (name, _, _), st in zip(members, sts):
        assert st["state"] == "done" and st["status"] == 0, (name, st)
        assert st["voxel_iters"] > 0
        _same(tmp_path / f"alone_{name}", tmp_path / f"batch_{name}")


def test_batch_members_against_oracle(tmp_path, oracle_lib):
    members = [m for m in _members(tmp_path) if m[0] in ("c8", "t12")]
    with Batch() as b:
        slots = [b.add(fft, tmp_path / f"batch_{name}") for name, fft, _ in members]
        b.run()
        assert all(b.status(s)["status"] == 0 for s in slots)
    for name, fft, _ in members:
        o = oracle_lib.OracleSolve(fft, out_dir=str(tmp_path / f"oracle_{name}"), mix=1, modal=0, write_files=True)
        o.run()
        o.close()
        rg = load_results(tmp_path / f"batch_{name}" / "results.csv")
        ro = load_results(tmp_path / f"oracle_{name}" / "results.csv")
        dg = np.loadtxt(tmp_path / f"batch_{name}" / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
        do = np.loadtxt(tmp_path / f"oracle_{name}" / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
        parity.assert_rows_match(rg, ro, dg, do)


def test_failing_member_leaves_the_others(tmp_path):
    members = [m for m in _members(tmp_path) if m[0] in ("c8", "c24")]
    for name, fft, prec in members:
        _alone(fft, tmp_path / f"alone_{name}", prec)
    bad = decks.write_case(decks.case_c1(nsteps=2), tmp_path / "singular")
    (bad.parent / "cuel.sx").write_text("0 \t\t\t\t\tISO\n" + "0.0 0.0 0.0 0.0 0.0 0.0\n" * 6)
    from creep_modeling_b200 import EvpError

    with Batch() as b:
        slots = [b.add(fft, tmp_path / f"batch_{name}") for name, fft, _ in members]
        with pytest.raises(EvpError) as ei:
            b.add(bad, tmp_path / "o_bad")
        assert ei.value.code == -3
        b.run()
        assert all(b.status(s)["status"] == 0 for s in slots)
    for name, _, _ in members:
        _same(tmp_path / f"alone_{name}", tmp_path / f"batch_{name}")


def test_members_sharing_one_newton_wave(tmp_path):
    """Two 40^3 members, each with a full wave of local-solve blocks (296): the batched launch
    runs two waves, and the members' files are identical to the solves alone."""
    members = []
    for i, stress in enumerate((120.0, 180.0)):
        c = decks.case_c1(nsteps=3)
        c.n, c.ngrains, c.seed = 40, 40, 11 + i
        c.processes[0].stress33 = stress
        members.append((f"c40_{i}", decks.write_case(c, tmp_path / f"c40_{i}"), 0))
    for name, fft, prec in members:
        _alone(fft, tmp_path / f"alone_{name}", prec)
    with Batch() as b:
        slots = [b.add(fft, tmp_path / f"batch_{name}") for name, fft, _ in members]
        b.run()
        assert all(b.status(s)["status"] == 0 for s in slots)
    for name, _, _ in members:
        _same(tmp_path / f"alone_{name}", tmp_path / f"batch_{name}")
