"""Record the shell command that the reference's utils/run.py:run_solver (169-196) issues.

The reference launches its solver through ``run.os_system(cmd)``; this script imports the
reference's ``run`` module (with a stub for the ``skopt`` import its config needs), replaces
``os_system`` by a recorder, calls ``run_solver`` with placeholder paths and writes the
command to run_solver_cmd.txt with the solver path, deck, output directory, wisdom file and
log file replaced by @EXE@, @FFT@, @OUT@, @WISDOM@ and @LOG@.  tests/test_gpu_dropin.py runs
that command, with the placeholders filled in and @EXE@ pointing at this repository's
LS-EVPFFT, exactly as run.py would.  The reference checkout is named by the first argument
or by EVP_REFERENCE:

    python tests/golden/make_run_solver_cmd.py PATH/TO/creep_modeling
"""
import os
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref: str) -> None:
    sk, sp = types.ModuleType("skopt"), types.ModuleType("skopt.space")

    class Real:  # only constructed by config.py's search-space tables
        def __init__(self, *a, **k):
            pass

    sp.Real = Real
    sk.space = sp
    sys.modules.setdefault("skopt", sk)
    sys.modules.setdefault("skopt.space", sp)
    sys.path.insert(0, str(Path(ref) / "utils"))
    import run

    seen = []
    run.os_system = lambda cmd: seen.append(cmd) or 0
    cfg = types.SimpleNamespace(nthreads=4, fft="@FFT@", evpfft_dir="@OUT@", fftw_save="@WISDOM@", mix=1, modal=0,
                                out_txt="@LOG@")
    assert run.run_solver(cfg) == 0 and len(seen) == 1
    cmd = seen[0].replace(str(run.SOLVER_EXE), "@EXE@")
    (HERE / "run_solver_cmd.txt").write_text(cmd + "\n")
    print(cmd)


if __name__ == "__main__":
    r = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EVP_REFERENCE")
    if not r:
        sys.exit("usage: make_run_solver_cmd.py PATH/TO/reference (or set EVP_REFERENCE)")
    main(r)
