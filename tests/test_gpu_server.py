"""The resident server on the GPU: each solve gives the same results alone and in the mix.

Three solves of different grid sizes and loadings are run one by one through
the plain entry point and then submitted together to one server, where they
run concurrently on separate CUDA streams.  results.csv and diagnostics.csv of
every solve must agree (wall-clock columns excepted) to 1e-12 relative; the
kernels' reductions have a fixed order, so in practice they are identical.
A second case gives the server a memory budget that fits one solve at a time
and checks that admission then serialises them without changing the results.
"""
from pathlib import Path

import numpy as np
import pytest

from creep_modeling_b200 import decks
from creep_modeling_b200.serve import Server
from creep_modeling_b200.solver import Solve

pytestmark = pytest.mark.gpu

TOL = 1e-12
WALL = {"results.csv": [4], "diagnostics.csv": [4]}  # wall_time columns


def _cases(root: Path):
    out = []
    c = decks.case_c1(nsteps=3)
    c.n = (8, 8, 8)
    c.ngrains = 8
    out.append(decks.write_case(c, root / "c8"))
    out.append(decks.write_case(decks.case_c2(nsteps=3, n=12, ngrains=10), root / "t12"))
    out.append(decks.write_case(decks.case_c1(nsteps=2), root / "c16"))
    return out


def _alone(fft: Path, out: Path):
    s = Solve(fft, out_dir=str(out), mix=1, modal=0, csv_only=True)
    s.run()
    s.close()


def _load(path: Path) -> np.ndarray:
    return np.loadtxt(path, delimiter=",", skiprows=1, ndmin=2)


def _same(a_dir: Path, b_dir: Path):
    for name, skip in WALL.items():
        a, b = _load(a_dir / name), _load(b_dir / name)
        assert a.shape == b.shape, name
        keep = [c for c in range(a.shape[1]) if c not in skip]
        a, b = a[:, keep], b[:, keep]
        scale = np.maximum(np.abs(a).max(axis=0), 1e-300)
        assert np.max(np.abs(a - b) / scale) <= TOL, name


def test_results_same_alone_and_in_the_mix(tmp_path):
    ffts = _cases(tmp_path)
    for i, f in enumerate(ffts):
        _alone(f, tmp_path / f"alone{i}")
    with Server(0, 8) as srv:
        tickets = [srv.submit(f, tmp_path / f"mix{i}", mix=1, modal=0, csv_only=True) for i, f in enumerate(ffts)]
        sts = [srv.wait(t, timeout=600) for t in tickets]
    for st in sts:
        assert st["state"] == "done" and st["status"] == 0, st
        assert st["voxel_iters"] > 0 and st["footprint_bytes"] > 0
    for i in range(len(ffts)):
        _same(tmp_path / f"alone{i}", tmp_path / f"mix{i}")


def test_budget_admits_one_at_a_time(tmp_path):
    ffts = _cases(tmp_path)[:2]
    for i, f in enumerate(ffts):
        _alone(f, tmp_path / f"alone{i}")
    with Server(1, 8) as srv:  # 1 byte: every solve exceeds it, so each runs alone
        tickets = [srv.submit(f, tmp_path / f"one{i}", mix=1, modal=0, csv_only=True) for i, f in enumerate(ffts)]
        sts = [srv.wait(t, timeout=600) for t in tickets]
    assert all(st["status"] == 0 for st in sts)
    # the second waited for the first: its queueing time covers the first one's run
    assert sts[1]["queued_s"] >= 0.9 * sts[0]["run_s"]
    for i in range(len(ffts)):
        _same(tmp_path / f"alone{i}", tmp_path / f"one{i}")


def test_failing_solves_are_isolated(tmp_path):
    """Beside two good solves, one deck whose phase stiffness is singular (-3), one whose
    microstructure file is missing (-1) and one that overruns its wall-clock budget (-8):
    each failing request reports its own status and the good solves' files are the same
    as when they run alone."""
    good = _cases(tmp_path)[:2]
    for i, f in enumerate(good):
        _alone(f, tmp_path / f"alone{i}")
    sing = decks.write_case(decks.case_c1(nsteps=2), tmp_path / "singular")
    (sing.parent / "cuel.sx").write_text("0 \t\t\t\t\tISO\n" + "0.0 0.0 0.0 0.0 0.0 0.0\n" * 6)
    missing = decks.write_case(decks.case_c1(nsteps=2), tmp_path / "missing")
    (missing.parent / "micro.dat").unlink()
    big = decks.case_c1(nsteps=100)
    big.n = 32  # 100 increments at 32^3: seconds of work, far beyond its budget
    slow = decks.write_case(big, tmp_path / "slow")
    with Server(0, 8) as srv:
        tg = [srv.submit(f, tmp_path / f"mix{i}", mix=1, modal=0, csv_only=True) for i, f in enumerate(good)]
        ts = srv.submit(sing, tmp_path / "o_sing", mix=1, modal=0, csv_only=True)
        tm = srv.submit(missing, tmp_path / "o_miss", mix=1, modal=0, csv_only=True)
        td = srv.submit(slow, tmp_path / "o_slow", mix=1, modal=0, csv_only=True, deadline_s=0.3)
        sts = [srv.wait(t, timeout=600) for t in tg]
        s_sing, s_miss, s_slow = srv.wait(ts, timeout=600), srv.wait(tm, timeout=600), srv.wait(td, timeout=600)
    assert all(st["status"] == 0 for st in sts), sts
    assert s_sing["status"] == -3 and "ingular" in s_sing["error"], s_sing
    assert s_miss["status"] == -1, s_miss
    assert s_slow["status"] == -8 and "deadline" in s_slow["error"], s_slow
    assert 0 < s_slow["macrosteps"] < 100
    assert s_slow["run_s"] < 30.0
    for i in range(len(good)):
        _same(tmp_path / f"alone{i}", tmp_path / f"mix{i}")


def test_large_lane_runs_the_shortest_first(tmp_path):
    """Three 72^3 requests (373,248 voxels each; the large lane holds at most 2 x 64^3 =
    524,288 voxels, so one at a time there) submitted back to back: their runs do not overlap,
    and the two that queue behind the first (a longer one, so that both are queued when it ends)
    are admitted least work first (voxels x increments)."""
    import time

    nsteps = (20, 4, 2)
    ffts = []
    for i, k in enumerate(nsteps):
        c = decks.case_c1(nsteps=k)
        c.n, c.ngrains = 72, 40
        ffts.append(decks.write_case(c, tmp_path / f"d{i}"))
    with Server(0, 8) as srv:
        t0 = time.perf_counter()
        calls, tickets = [], []
        for i, f in enumerate(ffts):  # each submit reads its deck (~0.1 s at 72^3) on this thread
            calls.append(time.perf_counter() - t0)
            tickets.append(srv.submit(f, tmp_path / f"o{i}", mix=1, modal=0, csv_only=True))
        sts = [srv.wait(t, timeout=600) for t in tickets]
    assert all(st["status"] == 0 for st in sts), sts
    start = [calls[i] + sts[i]["queued_s"] for i in range(3)]
    end = [start[i] + sts[i]["run_s"] for i in range(3)]
    order = sorted(range(3), key=lambda i: start[i])
    for p, q in zip(order, order[1:]):
        assert start[q] >= end[p] - 0.01, (start, end, sts)
    assert order == [0, 2, 1], (order, start, end)
