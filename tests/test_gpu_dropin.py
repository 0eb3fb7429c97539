"""The drop-in executable and the whole-solve entry point, run the way the reference's callers run them.

utils/run.py:169-196 (run_solver) launches the solver with
    set -o pipefail; EXE --nthreads n --in F --out D --fftw_save P --mix m --modal a | tee LOG;
and then reads results.csv, diagnostics.csv and the VTK files it wrote.  Here
that command line, recorded from the reference's own run_solver
(tests/golden/make_run_solver_cmd.py), runs creep_modeling_b200/LS-EVPFFT as a process, and
evp_solve_file runs the same deck in-process; both output directories must hold
the oracle's files: same names, the CSV columns within the parity bar and every
VTK number within 2e-8 of its block's largest magnitude (tests/test_gpu_files.py).
The deck is the reference's own tension template (6 processes) on a 16^3 sample
of micro1.dat, its processes cut to two steps, with VTK output every second step
of its first process.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from creep_modeling_b200 import solver
from tests import parity, ref_decks
from tests.test_gpu_files import VTK_TOL, _blocks

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "creep_modeling_b200" / "LS-EVPFFT"
GOLD = ROOT / "tests" / "golden"


def _oracle_files(oracle_lib, fft, out, modal):
    o = oracle_lib.OracleSolve(fft, out_dir=str(out), mix=1, modal=modal, write_files=True)
    o.run()
    o.close()


def _compare_dirs(a: Path, b: Path):
    names_a = sorted(p.name for p in a.iterdir() if p.suffix in (".csv", ".vtk"))
    names_b = sorted(p.name for p in b.iterdir() if p.suffix in (".csv", ".vtk"))
    assert names_a == names_b
    assert any(n.endswith(".vtk") for n in names_a)
    ra, rb = solver.load_results(a / "results.csv"), solver.load_results(b / "results.csv")
    da = np.loadtxt(a / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
    db = np.loadtxt(b / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
    parity.assert_rows_match(ra, rb, da, db)
    for n in names_a:
        if not n.endswith(".vtk"):
            continue
        wa, ba = _blocks(a / n)
        wb, bb = _blocks(b / n)
        assert wa == wb, n
        assert len(ba) == len(bb), n
        for x, y in zip(ba, bb):
            assert x.shape == y.shape, n
            scale = max(float(np.max(np.abs(y))), 1e-300)
            assert float(np.max(np.abs(x - y))) <= VTK_TOL * scale, n


@pytest.fixture
def deck(tmp_path):
    return ref_decks.materialize("tension", tmp_path / "deck", max_steps=2)


def test_executable_as_run_solver_launches_it(tmp_path, deck, oracle_lib):
    """The command is the one the reference's run_solver builds (recorded from its own code in
    tests/golden/run_solver_cmd.txt), with this repository's executable as SOLVER_EXE."""
    out, log = tmp_path / "evpfft_outputs", tmp_path / "output.txt"
    wisdom = tmp_path / "fftw" / "fftw_wisdom.save"
    cmd = (GOLD / "run_solver_cmd.txt").read_text().strip()
    for k, v in (("@EXE@", EXE), ("@FFT@", deck), ("@OUT@", out), ("@WISDOM@", wisdom), ("@LOG@", log)):
        cmd = cmd.replace(k, str(v))
    env = {k: v for k, v in os.environ.items() if k != "EVP_SERVER_SOCKET"}
    r = subprocess.run(["bash", "-c", cmd], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MACROSTEPS=" in log.read_text()
    assert wisdom.read_text().startswith("evp-tile ")  # --fftw_save named the FFT tile cache
    _oracle_files(oracle_lib, deck, tmp_path / "oracle", 0)
    _compare_dirs(out, tmp_path / "oracle")


def test_evp_solve_file(tmp_path, deck, oracle_lib):
    out = tmp_path / "gpu"
    rep = solver.run_solver(deck, out, nthreads=0, fftw_save="", mix=1, modal=0)
    assert rep.status == 0 and rep.macrosteps == 12 and rep.voxel_iters == rep.equilibrium_iters * 16 ** 3
    _oracle_files(oracle_lib, deck, tmp_path / "oracle", 0)
    _compare_dirs(out, tmp_path / "oracle")


def test_executable_reports_a_deck_error(tmp_path):
    bad = tmp_path / "fft.in"
    bad.write_text("1\n16 16 16\n")
    r = subprocess.run([str(EXE), "--in", str(bad), "--out", str(tmp_path / "o")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 1 and "[-1:" in r.stderr


def test_run_solver_command_through_the_socket_server(tmp_path, deck, oracle_lib):
    """The same recorded run.py command with EVP_SERVER_SOCKET set: the shim submits the deck to
    a resident server (a real GPU Server behind the JSON socket) and returns when its files are
    written; they must equal the oracle's as in the direct run."""
    import threading
    import time

    from creep_modeling_b200.serve import Server, serve_socket, submit_via_socket

    sock = str(tmp_path / "evp.sock")
    stop = threading.Event()
    with Server(0, 4) as srv:
        th = threading.Thread(target=serve_socket, args=(sock, srv, stop), daemon=True)
        th.start()
        for _ in range(500):
            if os.path.exists(sock):
                break
            time.sleep(0.01)
        out, log = tmp_path / "served_outputs", tmp_path / "served.txt"
        cmd = (GOLD / "run_solver_cmd.txt").read_text().strip()
        for k, v in (("@EXE@", EXE), ("@FFT@", deck), ("@OUT@", out), ("@WISDOM@", tmp_path / "w.save"), ("@LOG@", log)):
            cmd = cmd.replace(k, str(v))
        env = dict(os.environ, EVP_SERVER_SOCKET=sock)
        r = subprocess.run(["bash", "-c", cmd], env=env, capture_output=True, text=True, timeout=600)
        stop.set()
        try:  # wake the accept loop so that it sees the stop flag
            submit_via_socket(sock, "x.in", "o")
        except Exception:
            pass
        th.join(timeout=10)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "(served)" in log.read_text()
    _oracle_files(oracle_lib, deck, tmp_path / "oracle", 0)
    _compare_dirs(out, tmp_path / "oracle")
