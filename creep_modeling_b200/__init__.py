"""B200-native LS-EVPFFT crystal-plasticity solver (drop-in for gdebrun2/creep_modeling's lsevpfft/LS-EVPFFT).

The compute path is the sm_100a library ``_build/libevp_b200.so`` (C ABI in
``include/evp.h``); this package is the thin Python host over it.
"""
from .solver import Batch, Solve, run_solver, solve_files, load_results, RESULTS_COLS, DIAG_COLS  # noqa: F401
from ._lib import EvpError  # noqa: F401

__all__ = ["Batch", "Solve", "run_solver", "solve_files", "load_results", "RESULTS_COLS", "DIAG_COLS", "EvpError"]
