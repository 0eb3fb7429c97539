"""Solver inputs from the reference-writer fixtures in tests/golden/ref_decks/.

The decks are the text that the reference's own simulation-case templates
(``utils/sim_cases/creep_calibration.py``, ``utils/sim_cases/tension.py``)
produce; ``tests/golden/make_reference_decks.py`` generated them.  Here the path
placeholders are filled in, the material files are copied, the sampled
``micro1.dat`` is written back in the ``.dat`` grammar, and optionally every
process's step count is capped so that a test stays short.
"""
from __future__ import annotations

import re
import shutil
from pathlib import Path

import numpy as np

FIX = Path(__file__).resolve().parent / "golden" / "ref_decks"


def write_micro(path: Path) -> int:
    """The 16^3 sample of micro1.dat as ``phi1 Phi phi2 i j k grain phase`` lines (x fastest)."""
    z = np.load(FIX / "micro1_16.npz")
    grain, gids, euler = z["grain"], z["grain_ids"], z["euler"]
    row = {int(g): i for i, g in enumerate(gids)}
    n1, n2, n3 = grain.shape
    lines = []
    for k in range(n3):
        for j in range(n2):
            for i in range(n1):
                g = int(grain[i, j, k])
                e = euler[row[g]]
                lines.append(f"{e[0]:.6f} {e[1]:.6f} {e[2]:.6f} {i + 1} {j + 1} {k + 1} {g} 1")
    Path(path).write_text("\n".join(lines) + "\n")
    return n1 * n2 * n3


def materialize(name: str, root: Path, max_steps: int | None = None, max_procs: int | None = None) -> Path:
    """Write deck ``name`` (e.g. "creep_calibration_475", "tension") and its inputs under root.

    max_steps caps every process's nsteps; max_procs keeps only the first processes."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    micro = root / "micro1_16.dat"
    write_micro(micro)
    for f in ("cuel.sx", "cupl2.sx"):
        shutil.copy(FIX / f, root / f)
    txt = (FIX / f"{name}.in").read_text()
    txt = (txt.replace("@MICRO@", str(micro)).replace("@CUPL2@", str(root / "cupl2.sx"))
           .replace("@CUEL@", str(root / "cuel.sx")).replace("@CUPL2_GAS@", str(root / "cupl2.sx"))
           .replace("@CUEL_GAS@", str(root / "cuel.sx")))
    lines = txt.splitlines()
    if max_steps is not None:
        for i, ln in enumerate(lines):
            m = re.match(r"^(\s*)(\d+)(\s+nsteps \(total number of time steps\).*)$", ln)
            if m and int(m.group(2)) > max_steps:
                lines[i] = f"{m.group(1)}{max_steps}{m.group(3)}"
    if max_procs is not None:
        head = [i for i, ln in enumerate(lines) if ln.strip().startswith("*INFORMATION ABOUT TEST CONDITIONS")]
        nproc_line = next(i for i, ln in enumerate(lines) if "number of processes (nproc)" in ln)
        n = int(lines[nproc_line].split()[0])
        if max_procs < n:
            lines = lines[: head[max_procs]]
            lines[nproc_line] = re.sub(r"^\s*\d+", str(max_procs), lines[nproc_line])
    fft = root / "fft.in"
    fft.write_text("\n".join(lines) + "\n")
    return fft
