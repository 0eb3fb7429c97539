"""Surface-roughness post-processing of the written VTK files (the reference's ``vtk_sweep``).

The reference's post-processing (``utils/data_utils.py:934-1004`` with the helpers of
``utils/calc_utils.py:158-315``) reads, from every ``microstr_cell_fields_stp_*.vtk`` an
output directory holds, the node coordinates (POINTS) and the accumulated slip
(``gamdot_acum``), finds the four free side faces of the specimen (the first solid
layer inside the gas layers on the x and y sides, ``get_face_idx``), and reports per
file and per face (x min, x max, y min, y max):

* Sa: the mean absolute surface height, the height of a face node being its outward
  coordinate minus the face's mean (corner columns averaged over their two faces);
* Sz: the height range (max - min) over the face;
* the largest and the mean accumulated slip of the face's cells.

This module restates those metrics so that they can be computed on the GPU solver's
files and on the oracle's; ``tests/golden/make_roughness_golden.py`` pins it to the
reference's own functions.  The reference's side effects (appending node fields to
the VTK files, writing a ``.vtk.series`` index) are not repeated: they decorate the
files for viewing and change no metric.
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np

GAS_PHASE = 2  # phase id of the gas (damper) phase in the microstructure file (utils/config.py PHASE_GAS)


def read_micro_phase(path) -> tuple[int, int, int, np.ndarray]:
    """(nx, ny, nz, phase[nz, ny, nx]) of a microstructure .dat file (columns 4-6 are 1-based
    x, y, z; column 8 the phase id), as ``MicrostructureInfo.load`` reads it."""
    arr = np.loadtxt(path)
    x, y, z = (arr[:, c].astype(int) for c in (3, 4, 5))
    nx, ny, nz = int(x.max()), int(y.max()), int(z.max())
    phase = np.zeros((nz, ny, nx), dtype=int)
    phase[z - 1, y - 1, x - 1] = arr[:, 7].astype(int)
    return nx, ny, nz, phase


def face_indices(phase: np.ndarray) -> tuple[int, int, int, int]:
    """Cell indices of the outermost solid layers on the x and y sides: the gas layers are
    counted along the centre lines of the middle z plane (calc_utils.get_face_idx)."""
    nz, ny, nx = phase.shape
    gas = phase == GAS_PHASE
    ixmin = int(gas[nz // 2, ny // 2, 0: nx // 2].sum())
    ixmax = nx - int(gas[nz // 2, ny // 2, nx // 2:].sum()) - 1
    iymin = int(gas[nz // 2, 0: ny // 2, nx // 2].sum())
    iymax = ny - int(gas[nz // 2, ny // 2:, nx // 2].sum()) - 1
    return ixmin, ixmax, iymin, iymax


def read_points_slip(path, nx: int, ny: int, nz: int) -> tuple[np.ndarray, np.ndarray]:
    """Node coordinates [nz+1, ny+1, nx+1, 3] and accumulated slip [nz, ny, nx] of one VTK file."""
    nnodes, ncells = (nz + 1) * (ny + 1) * (nx + 1), nz * ny * nx
    points = slip = None
    with open(path) as f:
        for line in f:
            s = line.strip()
            if s.startswith("POINTS"):
                points = np.loadtxt(f, max_rows=nnodes, dtype=np.float64).reshape(nz + 1, ny + 1, nx + 1, 3)
            elif s.startswith("gamdot_acum"):
                slip = np.loadtxt(f, max_rows=ncells, dtype=np.float64).reshape(nz, ny, nx)
                break
    if points is None or slip is None:
        raise ValueError(f"{path}: no POINTS or gamdot_acum block")
    return points, slip


def _faces(ixmin, ixmax, iymin, iymax, node):
    return (ixmin, ixmax + 1, iymin, iymax + 1) if node else (ixmin, ixmax, iymin, iymax)


def surface_height(points: np.ndarray, faces) -> np.ndarray:
    """Heights of the side-face nodes (zero elsewhere), corner columns averaged over their faces."""
    ixmin, ixmax, iymin, iymax = _faces(*faces, node=True)
    h = np.zeros(points.shape[:3])
    hx0 = -(points[:, :, ixmin, 0] - points[:, :, ixmin, 0].mean())
    hy0 = -(points[:, iymin, :, 1] - points[:, iymin, :, 1].mean())
    hx1 = points[:, :, ixmax, 0] - points[:, :, ixmax, 0].mean()
    hy1 = points[:, iymax, :, 1] - points[:, iymax, :, 1].mean()
    h[:, :, ixmin] = hx0
    h[:, :, ixmax] = hx1
    h[:, iymin, :] = hy0
    h[:, iymax, :] = hy1
    h[:, iymin, ixmin] = (hx0[:, 0] + hy0[:, 0]) / 2
    h[:, iymin, ixmax] = (hx1[:, 0] + hy0[:, -1]) / 2
    h[:, iymax, ixmin] = (hx0[:, -1] + hy1[:, 0]) / 2
    h[:, iymax, ixmax] = (hx1[:, -1] + hy1[:, -1]) / 2
    return h


def face_metrics(points: np.ndarray, slip: np.ndarray, faces) -> dict:
    """Sa, Sz (node heights) and the largest and mean accumulated slip (cells) of the four faces,
    each as (x min, x max, y min, y max)."""
    h = surface_height(points, faces)
    nx0, nx1, ny0, ny1 = _faces(*faces, node=True)
    cx0, cx1, cy0, cy1 = _faces(*faces, node=False)
    hn = (h[:, :, nx0], h[:, :, nx1], h[:, ny0, :], h[:, ny1, :])
    sc = (slip[:, :, cx0], slip[:, :, cx1], slip[:, cy0, :], slip[:, cy1, :])
    return {
        "sa": np.array([np.abs(a).mean() for a in hn]),
        "sz": np.array([a.max() - a.min() for a in hn]),
        "max_slip": np.array([a.max() for a in sc]),
        "mean_slip": np.array([a.mean() for a in sc]),
    }


def vtk_sweep(out_dir, micro_path) -> dict:
    """Metrics of every VTK file of a solve, in file-name order: macrostep numbers and arrays
    [4, nfiles] of Sa, Sz, max and mean slip (the rows of the reference's vtk_sweep result)."""
    nx, ny, nz, phase = read_micro_phase(micro_path)
    faces = face_indices(phase)
    files = sorted(Path(out_dir).glob("*.vtk"))
    steps, rows = [], {k: [] for k in ("sa", "sz", "max_slip", "mean_slip")}
    for f in files:
        steps.append(int(re.findall(r"_(\d+)\.vtk$", f.name)[0]))
        pts, slip = read_points_slip(f, nx, ny, nz)
        m = face_metrics(pts, slip, faces)
        for k in rows:
            rows[k].append(m[k])
    out = {k: np.array(v).T for k, v in rows.items()}
    out["macrostep"] = np.array(steps, dtype=int)
    return out
