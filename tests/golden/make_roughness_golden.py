"""Generate the surface-roughness fixture from the reference's own post-processing.

The oracle (oracle/, the CPU FP64 restatement of the solver) writes the VTK files of
the free-surface creep case of tests/roughness_case.py; the reference's ``vtk_sweep``
(``utils/data_utils.py:934-1004``, on a copy of those files, since it appends fields
to them) computes Sa, Sz and the largest and mean accumulated slip of the four side
faces from them.  Its results go to roughness_golden.npz, which
tests/test_roughness_cpu.py holds the package's restatement
(creep_modeling_b200/roughness.py) to.  The reference's ``config.py`` imports ``skopt``
only for a search-space type; a stub module satisfies that import.  The reference
checkout is named by the first argument or by EVP_REFERENCE:

    python tests/golden/make_roughness_golden.py PATH/TO/creep_modeling
"""
import os
import shutil
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def _import_reference(ref: Path):
    sk, sp = types.ModuleType("skopt"), types.ModuleType("skopt.space")

    class Real:  # only constructed by config.py's search-space tables
        def __init__(self, *a, **k):
            pass

    sp.Real = Real
    sk.space = sp
    sys.modules.setdefault("skopt", sk)
    sys.modules.setdefault("skopt.space", sp)
    sys.path.insert(0, str(ref / "utils"))
    import data_utils

    return data_utils


def main(ref: str) -> None:
    import oracle
    from tests import roughness_case

    data_utils = _import_reference(Path(ref))
    td = Path(tempfile.mkdtemp())
    fft, micro = roughness_case.write_case(td / "deck")
    o = oracle.OracleSolve(fft, out_dir=str(td / "out"), mix=1, modal=0, write_files=True)
    o.run()
    o.close()
    work = td / "ref_copy"
    shutil.copytree(td / "out", work)
    res = np.loadtxt(td / "out" / "results.csv", delimiter=",", skiprows=1, ndmin=2)
    sim_time = np.concatenate([[0.0], res[:, 3]])
    info = data_utils.MicrostructureInfo.load(micro)
    steps, times, sa, sz, mx, mn = data_utils.vtk_sweep(work, sim_time, info)
    np.savez(HERE / "roughness_golden.npz", macrostep=np.asarray(steps), time=np.asarray(times), sa=np.asarray(sa),
             sz=np.asarray(sz), max_slip=np.asarray(mx), mean_slip=np.asarray(mn))
    print("wrote roughness_golden.npz:", np.asarray(sa).shape)


if __name__ == "__main__":
    r = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EVP_REFERENCE")
    if not r:
        sys.exit("usage: make_roughness_golden.py PATH/TO/reference (or set EVP_REFERENCE)")
    main(r)
