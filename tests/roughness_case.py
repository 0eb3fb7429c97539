"""A specimen with free side faces, for the surface-roughness post-processing.

A 12^3 periodic Voronoi polycrystal whose two outermost voxel layers on the x and y
sides are gas (phase 2, igas = 1), as the reference's damper-layer microstructures
have them, crept at 150 MPa along z for three increments with the lattice-rotation
and grid updates and VTK output at every increment.  Used by
tests/golden/make_roughness_golden.py and the roughness tests.
"""
from __future__ import annotations

from pathlib import Path

from creep_modeling_b200 import decks

N = 12
LAYERS = 2
NSTEPS = 3


def write_case(root: Path) -> tuple[Path, Path]:
    """Write the deck and its inputs under root; returns (fft.in, micro .dat)."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    grain, phase, euler = decks.voronoi_micro(N, 12, 4)
    phase[:LAYERS, :, :] = 2
    phase[-LAYERS:, :, :] = 2
    phase[:, :LAYERS, :] = 2
    phase[:, -LAYERS:, :] = 2
    micro = root / "micro.dat"
    decks.write_micro(micro, grain, phase, euler, euler2=(0.0, 0.0, 0.0))
    mat = decks.Material()
    decks.write_cuel(root / "cuel.sx", mat)
    decks.write_cupl2(root / "cupl2.sx", mat)
    decks.write_cuel(root / "cuel_gas.sx", iso=1, young=400000.0, nu=0.3)
    decks.write_cupl2(root / "cupl2_gas.sx", mat)
    proc = decks.Loading(kind="creep", stress33=150.0, udot33=1e-4, tdot=10.0, nsteps=NSTEPS, error=1e-5,
                         erroral=1e-9, itmax=200, iwfields=1, iwstep=1)
    fft = root / "fft.in"
    decks.write_fft_in(fft, N, micro, root / "cupl2.sx", root / "cuel.sx", [proc],
                       phase2=(1, root / "cupl2_gas.sx", root / "cuel_gas.sx"), complgas=1.0)
    return fft, micro
