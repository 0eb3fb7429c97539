"""Generate the reference-writer deck fixtures from the reference's own Python.

The solver's real callers write their decks with the reference's simulation-case
templates: ``utils/sim_cases/creep_calibration.py`` (17 processes: a stress ramp
to the creep load, then creep holds with sub-stepping enabled) and
``utils/sim_cases/tension.py`` (6 processes).  This script calls their
``build_fft`` functions, and ``utils/io_utils.py``'s ``write_cuel`` /
``write_cupl2`` with the reference's default material (``utils/config.py``), and
stores what they return under ``ref_decks/``:

  creep_calibration_<load>.in, tension.in   deck text (tension with a second, solid phase that no
                                            voxel uses: the template always writes a phase-2
                                            block); file paths are the placeholders
                                            @MICRO@, @CUPL2@, @CUEL@, @CUPL2_GAS@, @CUEL_GAS@
  cuel.sx, cupl2.sx                         material files
  micro1_16.npz                             the shipped microstructures/micro1.dat (32 x 32 x 64,
                                            850 grains) sampled every (2, 2, 4) voxels -> 16^3;
                                            grain ids per voxel and Bunge angles per grain

``tests/ref_decks.py`` turns them back into solver inputs.  The reference's
``config.py`` imports ``skopt`` only for a search-space type; a stub module
satisfies that import, and ``write_fft.FftConfig`` (a pydantic dataclass that
the templates only read attributes from) is replaced by a plain namespace.
The reference checkout is named by the first argument or by EVP_REFERENCE:

    python tests/golden/make_reference_decks.py PATH/TO/creep_modeling
"""
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "ref_decks"
LOADS = (475,)
PLACEHOLDERS = dict(microstructure="@MICRO@", cupl2="@CUPL2@", cuel="@CUEL@", cupl2_gas="@CUPL2_GAS@",
                    cuel_gas="@CUEL_GAS@")


def _import_reference(ref: Path):
    sk, sp = types.ModuleType("skopt"), types.ModuleType("skopt.space")

    class Real:  # only constructed by config.py's search-space tables
        def __init__(self, *a, **k):
            pass

    sp.Real = Real
    sk.space = sp
    sys.modules.setdefault("skopt", sk)
    sys.modules.setdefault("skopt.space", sp)
    wf = types.ModuleType("write_fft")
    wf.FftConfig = types.SimpleNamespace
    sys.modules["write_fft"] = wf
    sys.modules["utils.write_fft"] = wf
    sys.path.insert(0, str(ref / "utils"))
    import config
    import io_utils
    from sim_cases import creep_calibration, tension

    return config, io_utils, creep_calibration, tension


def _cfg(**kw):
    base = dict(sim_case="creep_calibration", igas=0, load=None, complgas=0, nphase=1, nx=16, ny=16, nz=16)
    base.update(PLACEHOLDERS)
    base.update(kw)
    return types.SimpleNamespace(**base)


def main(ref: str) -> None:
    ref = Path(ref)
    config, io_utils, creep_calibration, tension = _import_reference(ref)
    OUT.mkdir(parents=True, exist_ok=True)
    for load in LOADS:
        txt = creep_calibration.build_fft(_cfg(load=float(load)))
        (OUT / f"creep_calibration_{load}.in").write_text(txt if txt.endswith("\n") else txt + "\n")
    # the tension template always writes a phase-2 block, so it is only well formed with
    # nphase = 2; run.py passes the solid's files for a non-gas second phase (igas 0)
    txt = tension.build_fft(_cfg(sim_case="tension", nphase=2, igas=0))
    (OUT / "tension.in").write_text(txt if txt.endswith("\n") else txt + "\n")
    io_utils.write_cuel(OUT / "cuel.sx", elastic=config.SolidElastic(), iso=0)
    io_utils.write_cupl2(OUT / "cupl2.sx", plastic=config.SolidPlastic())
    a = np.loadtxt(ref / "microstructures" / "micro1.dat")
    ijk = a[:, 3:6].astype(int) - 1
    keep = (ijk[:, 0] % 2 == 0) & (ijk[:, 1] % 2 == 0) & (ijk[:, 2] % 4 == 0)
    sub = a[keep]
    grain = np.zeros((16, 16, 16), dtype=np.int16)
    s = sub[:, 3:6].astype(int) - 1
    grain[s[:, 0] // 2, s[:, 1] // 2, s[:, 2] // 4] = sub[:, 6].astype(np.int16)
    gids = np.unique(sub[:, 6].astype(int))
    euler = np.array([sub[sub[:, 6].astype(int) == g][0, :3] for g in gids])
    phase = np.unique(sub[:, 7].astype(int))
    assert phase.tolist() == [1]
    np.savez_compressed(OUT / "micro1_16.npz", grain=grain, grain_ids=gids.astype(np.int16), euler=euler)
    print("wrote", sorted(p.name for p in OUT.iterdir()))


if __name__ == "__main__":
    r = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EVP_REFERENCE")
    if not r:
        sys.exit("usage: make_reference_decks.py PATH/TO/reference (or set EVP_REFERENCE)")
    main(r)
