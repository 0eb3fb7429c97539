"""CPU-side checks of the drop-in boundary: exported C ABI, deck parsing, CLI flags.

No compute call is made here (there is no GPU on the CPU runner): a valid deck
makes evp_open stop at the device check (-6), an invalid deck is refused by the
parser first (-1 / -2), exactly as the reference's load_input stops.
"""
import ctypes
import re
from pathlib import Path

import pytest

from creep_modeling_b200 import _lib, cli, decks

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "evp.h").read_text()
    declared = set(re.findall(r"^\w[\w\s\*]*?\b(evp_\w+)\s*\(", header, flags=re.M))
    assert declared, "no declarations found"
    L = _lib.load()
    for name in sorted(declared):
        assert hasattr(L, name), name
    assert set(_lib.EXPORTED) == declared
    assert L.evp_version() >= 1


def _open(fft):
    L = _lib.load()
    h = ctypes.c_void_p()
    rc = L.evp_open(str(fft).encode(), b"", 1, 0, 0, ctypes.byref(h))
    return rc, L.evp_last_error().decode()


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_valid_deck_reaches_device_check(tmp_path):
    fft = decks.write_case(decks.case_c1(nsteps=2), tmp_path)
    rc, msg = _open(fft)
    assert rc == -6 and "CUDA" in msg


@pytest.mark.parametrize("mutate,code,needle", [
    (lambda s: s.replace("\t1       1       0                     |            \n",
                         "\t1       1       1                     |            \n", 1), -1, "boundary"),
    (lambda s: s.replace("2.0 0            XC0", "2.0 3            XC0", 1), -1, "igamma"),
    (lambda s: s.replace("0                      IDISPINI (if idispini=1, next line is filedispl)\n",
                         "3                      IDISPINI (if idispini=1, next line is filedispl)\nd.txt\n", 1), -1, "idispini"),
    (lambda s: s.replace("0                      IDISPINI (if idispini=1, next line is filedispl)\n",
                         "1                      IDISPINI (if idispini=1, next line is filedispl)\n/nonexistent/d.txt\n", 1),
     -1, "cannot open"),
])
def test_invalid_decks_are_refused(tmp_path, mutate, code, needle):
    fft = decks.write_case(decks.case_c1(nsteps=2), tmp_path)
    fft.write_text(mutate(fft.read_text()))
    rc, msg = _open(fft)
    assert rc == code, msg
    assert needle.lower() in msg.lower()


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
@pytest.mark.parametrize("igamma", [1, 2])
def test_discrete_green_decks_are_accepted(tmp_path, igamma):
    """IGAMMA 1 (central differences) and 2 (rotated scheme) pass the deck checks."""
    fft = decks.write_case(decks.case_c1(nsteps=2), tmp_path)
    fft.write_text(fft.read_text().replace("2.0 0            XC0", f"2.0 {igamma}            XC0", 1))
    rc, msg = _open(fft)
    assert rc == -6 and "CUDA" in msg


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
@pytest.mark.parametrize("kind", [1, 2])
def test_initial_displacement_decks_are_accepted(tmp_path, kind):
    """IDISPINI 1 (cell centres) and 2 (nodes): the displacement file is read with the deck."""
    c = decks.case_c1(nsteps=2)
    c.n = 8
    c.ngrains = 6
    c.dispini = kind
    rc, msg = _open(decks.write_case(c, tmp_path))
    assert rc == -6 and "CUDA" in msg


def test_missing_deck_is_refused(tmp_path):
    rc, msg = _open(tmp_path / "nope.in")
    assert rc == -1 and "cannot open" in msg


def test_oracle_parses_the_same_decks(oracle_lib, tmp_path):
    fft = decks.write_case(decks.case_c2(nsteps=1, n=8, ngrains=6), tmp_path)
    s = oracle_lib.OracleSolve(fft)
    assert s.shape == (8, 8, 8)
    s.close()


def test_cli_flags_match_the_reference():
    o = cli.parse(["--in", "a.in", "--out", "d/", "--nthreads", "4", "--fftw_save", "w", "--mix", "0", "--modal", "3"])
    assert o == {"in": "a.in", "out": "d/", "nthreads": 4, "fftw_save": "w", "mix": 0, "modal": 1}
    assert cli.parse(["--bogus"]) is None
    assert cli.parse(["-h"]) is None


def test_micro_file_grammar(tmp_path):
    g, p, e = decks.voronoi_micro(6, 5, seed=1)
    decks.write_micro(tmp_path / "m.dat", g, p, e)
    lines = (tmp_path / "m.dat").read_text().split("\n")
    assert len([x for x in lines if x]) == 216
    f = lines[0].split()
    assert len(f) == 8 and f[3:6] == ["1", "1", "1"]
    assert 1 <= int(f[6]) <= 5 and f[7] == "1"


def test_results_csv_rows_match_header(oracle_lib, tmp_path):
    """results.csv and diagnostics.csv rows have exactly the header's fields (51 and 44,
    IO_functions.f90:1264-1296, types.f90:787-834), so loaders that select columns by
    name (the reference's SimResults.load) read the right values."""
    import pandas as pd

    c = decks.case_c1(nsteps=1)
    c.n = 8
    c.ngrains = 6
    fft = decks.write_case(c, tmp_path / "d")
    assert oracle_lib.run_file(fft, tmp_path / "out") == 0
    for name, nf in (("results.csv", 51), ("diagnostics.csv", 44)):
        lines = (tmp_path / "out" / name).read_text().splitlines()
        assert [len(r.split(",")) for r in lines] == [nf] * len(lines), name
    df = pd.read_csv(tmp_path / "out" / "results.csv")
    assert list(df["macrostep"]) == [1] and df["iter"][0] > 1
    assert abs(df["sav33"][0] - 150.0) < 1.0
