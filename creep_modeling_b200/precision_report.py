"""Error and speed of the mixed-precision path against the plain FP64 path.

Runs the two-phase creep configuration (periodic Voronoi polycrystal plus
5 vol % stiff elastic spheres, creep at each requested stress) twice per
stress, plain FP64 and mixed precision (FP32 spectrum, FFTs and Green
operator; FP64 local Newton, reductions and F/rotation updates), and prints
one JSON document:

* per tensor curve of results.csv (average strain, stress, plastic strain,
  elastic strain, velocity gradient, plastic strain rate): the largest
  difference over the run relative to the tensor's largest magnitude;
* the creep-strain curve epav33(t) and the stress sav33(t) on their own scale;
* the per-voxel von Mises stress at the last increment, relative to its maximum;
* device time, equilibrium iterations and voxel-iters/s of each run.

    python -m creep_modeling_b200.precision_report --n 128 --ngrains 2000 --steps 300
"""
from __future__ import annotations

import argparse
import json
import tempfile
from pathlib import Path

import numpy as np

from . import decks
from .solver import RESULTS_COLS, Solve

TENSORS = {"eav": 7, "sav": 13, "epav": 19, "eelav": 25, "vgrad": 31, "edotp": 37}


def _run(fft: Path, precision: int, nsteps: int) -> dict:
    s = Solve(fft, mix=1, modal=0, precision=precision)
    rows = []
    for _ in range(nsteps):
        if s.advance(1) != 1:
            break
        rows.append(s.rows()[0])
    st = s.stats()
    sg = s.field("sg").reshape(-1, 3, 3)
    s.close()
    dev = sg - np.trace(sg, axis1=1, axis2=2)[:, None, None] * np.eye(3) / 3.0
    vm = np.sqrt(1.5 * np.einsum("nij,nij->n", dev, dev))
    return {"rows": np.array(rows), "vm": vm, "gpu_s": st.gpu_s, "iters": st.equilibrium_iters,
            "voxel_iters": st.voxel_iters}


def compare(fft: Path, nsteps: int) -> dict:
    a, b = _run(fft, 0, nsteps), _run(fft, 1, nsteps)
    ra, rb = a["rows"], b["rows"]
    m = min(len(ra), len(rb))
    ra, rb = ra[:m], rb[:m]
    curves = {}
    for name, c0 in TENSORS.items():
        scale = float(np.max(np.abs(ra[:, c0:c0 + 6])))
        curves[name] = float(np.max(np.abs(rb[:, c0:c0 + 6] - ra[:, c0:c0 + 6])) / scale) if scale > 0 else 0.0
    own = {}
    for col in ("epav33", "eav33", "sav33"):
        i = RESULTS_COLS.index(col)
        scale = float(np.max(np.abs(ra[:, i])))
        own[col] = float(np.max(np.abs(rb[:, i] - ra[:, i])) / scale) if scale > 0 else 0.0
    return {
        "increments": m, "curve_err_by_tensor": curves, "curve_err_own_scale": own,
        "vm_field_err": float(np.max(np.abs(b["vm"] - a["vm"])) / np.max(a["vm"])),
        "fp64": {"gpu_s": a["gpu_s"], "iters": a["iters"], "voxel_iters_per_s": a["voxel_iters"] / max(a["gpu_s"], 1e-30)},
        "mixed": {"gpu_s": b["gpu_s"], "iters": b["iters"], "voxel_iters_per_s": b["voxel_iters"] / max(b["gpu_s"], 1e-30)},
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--ngrains", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--stresses", default="100,150,200")
    ap.add_argument("--out", default="", help="also write the JSON here")
    args = ap.parse_args(argv)
    res = {"config": {"n": args.n, "ngrains": args.ngrains, "increments": args.steps, "phase2": "5 vol% spheres r 2-4, "
                      "E=400 GPa nu=0.3, tau0=1e8 (elastic)", "dt_s": 10.0}, "stress": {}}
    with tempfile.TemporaryDirectory() as td:
        for sv in [float(x) for x in args.stresses.split(",")]:
            case = decks.case_c3(stress33=sv, nsteps=args.steps, n=args.n, ngrains=args.ngrains)
            fft = decks.write_case(case, Path(td) / f"s{int(sv)}")
            res["stress"][str(int(sv))] = compare(fft, args.steps)
            print(json.dumps({str(int(sv)): res["stress"][str(int(sv))]}), flush=True)
    txt = json.dumps(res, indent=1)
    if args.out:
        Path(args.out).write_text(txt)
    print(txt)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
