"""Generate the calibration-client fixtures from the reference's own Python.

Writes, next to this file:
  calib_creep.csv, calib_srj.csv   synthetic experimental stand-ins (creep_modeling_b200.calibration)
  calib_golden.npz                 what the reference's loaders and metrics return on them

The reference's ``utils/`` package imports ``skopt`` (absent here) from
``config.py`` only for a search-space type that the loaders and metrics never
use; a stub module satisfies that import.  The reference checkout is named by
the first argument or by the EVP_REFERENCE environment variable:

    python tests/golden/make_calibration_golden.py PATH/TO/creep_modeling
"""
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from creep_modeling_b200 import calibration  # noqa: E402


def _import_reference(ref: Path):
    sk, sp = types.ModuleType("skopt"), types.ModuleType("skopt.space")

    class Real:  # only constructed by config.py's search-space table
        def __init__(self, *a, **k):
            pass

    sp.Real = Real
    sk.space = sp
    sys.modules.setdefault("skopt", sk)
    sys.modules.setdefault("skopt.space", sp)
    sys.path.insert(0, str(ref / "utils"))
    import calc_utils
    import data_utils

    return calc_utils, data_utils


def main(ref: str) -> None:
    calc_utils, data_utils = _import_reference(Path(ref))
    creep = calibration.synthetic_creep_csv(HERE / "calib_creep.csv", seed=7)
    srj = calibration.synthetic_srj_csv(HERE / "calib_srj.csv", seed=7)
    out = {}
    cd = data_utils.CreepData.load(csv_path=creep, skip_roughness=True)
    for load in calibration.LOADS:
        v = cd.get_load_vals(load)
        out[f"creep{load}_time"] = v["time"][1:]
        out[f"creep{load}_mps"] = v["mean_plastic_strain"]
    sd = data_utils.SrjData.load(csv_path=srj)
    out["srj_time"], out["srj_stress"], out["srj_strain"] = sd.time, sd.mean_stress, sd.mean_strain
    rng = np.random.default_rng(11)
    for k in range(4):
        sim_x = np.sort(rng.uniform(0, 100, 37))
        exp_x = np.sort(rng.uniform(-5, 105, 23))
        sim_y = rng.uniform(0.5, 2.0, 37)
        exp_y = rng.uniform(0.5, 2.0, 23)
        out[f"m{k}_sim_x"], out[f"m{k}_sim_y"], out[f"m{k}_exp_x"], out[f"m{k}_exp_y"] = sim_x, sim_y, exp_x, exp_y
        out[f"m{k}_idx"] = calc_utils.nearest_indices(exp_x, sim_x)
        kw = dict(sim_x=sim_x, sim_y=sim_y, exp_x=exp_x, exp_y=exp_y)
        out[f"m{k}_mae"] = calc_utils.mean_abs_error_aligned(**kw)
        out[f"m{k}_mse"] = calc_utils.mean_sq_error_aligned(**kw)
        out[f"m{k}_mre"] = calc_utils.mean_rel_err_aligned(**kw)
    np.savez(HERE / "calib_golden.npz", **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    import os

    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EVP_REFERENCE")
    if not ref:
        sys.exit("usage: make_calibration_golden.py PATH/TO/reference (or set EVP_REFERENCE)")
    main(ref)
