"""Python front end of the B200 LS-EVPFFT solver.

Mirrors the reference's solver interface: the executable ``lsevpfft/LS-EVPFFT``
(flags of ``lsevpfft/src/LS-EVPFFT.f90:87-142``) as launched by
``utils/run.py:169-196`` (``run_solver``), and the files it writes.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _lib

RESULTS_COLS = (
    "iter,macrostep,ipr,sim_time,wall_time,tdot,tdot_ref,eav11,eav22,eav33,eav23,eav13,eav12,sav11,sav22,sav33,"
    "sav23,sav13,sav12,epav11,epav22,epav33,epav23,epav13,epav12,eelav11,eelav22,eelav33,eelav23,eelav13,"
    "eelav12,vgrad11,vgrad22,vgrad33,vgrad23,vgrad13,vgrad12,edotp11,edotp22,edotp33,edotp23,edotp13,edotp12,"
    "evm,evmp,dvm,dvmp,svm,gamma,g,geff").split(",")

DIAG_COLS = (
    "iter,macrostep,ipr,sim_time,wall_time,tdot,vm_max_inc,tdotref,erre,errs,errsbc,s33_target,s33,s33_sol,"
    "detF_min_sol,detF_min_gas,detF_min_sol_rel,detF_min_gas_rel,volinc_max_sol,volinc_max_gas,volinc_max_sol_rel,"
    "volinc_max_gas_rel,stretchinc_max_sol,stretchinc_max_gas,stretchinc_max_sol_rel,stretchinc_max_gas_rel,"
    "rotang_max_sol,rotang_max_gas,dL_step_rms_sol,dL_step_rms_gas,dL_step_rms,dL_step_max_sol,dL_step_max_gas,"
    "dL_step_max,dvelgradavg_mag,cond_c066mod_max_sol,cond_c066mod_max_gas,cond_cgas_max,imin_sol_i,imin_sol_j,"
    "imin_sol_k,imin_gas_i,imin_gas_j,imin_gas_k").split(",")

WRITE_FILES = 1
VERBOSE = 2
WRITE_CSV = 4
PROFILE = 8
MIXED = 16


def run_solver(fft_in, out_dir="evpfft_outputs/", nthreads=0, fftw_save="", mix=1, modal=1) -> _lib.Report:
    """One whole solve, as one ``LS-EVPFFT --in ... --out ...`` process would do it.

    Raises ``EvpError`` with the library's status code on failure."""
    L = _lib.load()
    rep = _lib.Report()
    rc = L.evp_solve_file(str(fft_in).encode(), str(out_dir).encode(), int(nthreads), str(fftw_save).encode(), int(mix),
                          int(modal), ctypes.byref(rep))
    _lib.check(rc)
    return rep


def tune_cache(path) -> None:
    """Tile cache of the FFT passes for every later solve in this process (``evp_tune_cache``):
    grids not in the file are timed on the device at open and appended; None or "": no cache."""
    _lib.check(_lib.load().evp_tune_cache(str(path).encode() if path else b""))


class Solve:
    """A device-resident solve advanced macrostep by macrostep."""

    def __init__(self, fft_in, out_dir="", mix=1, modal=1, write_files=False, verbose=False, csv_only=False,
                 profile=False, precision=0):
        """precision 0: plain FP64; 1: mixed (FP32 spectrum, FFTs and Green operator in the
        equilibrium iteration; FP64 local Newton, reductions and F/rotation updates)."""
        L = _lib.load()
        h = ctypes.c_void_p()
        flags = ((WRITE_FILES if write_files else 0) | (VERBOSE if verbose else 0) | (WRITE_CSV if csv_only else 0)
                 | (PROFILE if profile else 0) | (MIXED if precision else 0))
        _lib.check(L.evp_open(str(fft_in).encode(), str(out_dir).encode(), int(mix), int(modal), flags, ctypes.byref(h)))
        self._h = h
        rep = self.stats()
        self.shape = (rep.n1, rep.n2, rep.n3)
        self.nvox = rep.n1 * rep.n2 * rep.n3

    def advance(self, nmacro: int = 1) -> int:
        done = ctypes.c_int(0)
        _lib.check(_lib.load().evp_advance(self._h, int(nmacro), ctypes.byref(done)))
        return done.value

    def run(self) -> list:
        rows = []
        while self.advance(1) == 1:
            rows.append(self.rows()[0])
        return rows

    def rows(self):
        r = np.zeros(51)
        d = np.zeros(44)
        _lib.load().evp_last_rows(self._h, r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return r, d

    def field(self, name: str) -> np.ndarray:
        cap = self.nvox * 128 + 3 * (self.shape[0] + 1) * (self.shape[1] + 1) * (self.shape[2] + 1)
        buf = np.zeros(cap)
        n = ctypes.c_longlong(0)
        _lib.check(_lib.load().evp_get_field(self._h, name.encode(), buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap,
                                             ctypes.byref(n)))
        return buf[: n.value].copy()

    def kernel_times(self) -> dict:
        """{kernel: (launches, total ms)} recorded under ``profile=True``."""
        cap = 64
        names = ctypes.create_string_buffer(32 * cap)
        launches = (ctypes.c_longlong * cap)()
        ms = (ctypes.c_double * cap)()
        n = _lib.load().evp_kernel_times(self._h, names, launches, ms, cap)
        out = {}
        for i in range(max(n, 0)):
            nm = names.raw[32 * i: 32 * i + 32].split(b"\0", 1)[0].decode()
            out[nm] = (int(launches[i]), float(ms[i]))
        return out

    def launches(self) -> int:
        """Kernels launched by this solve so far."""
        return int(_lib.load().evp_kernel_launches(self._h))

    def newton_stats(self) -> dict:
        """Activity counters of the local Newton kernel (profiled solves only)."""
        v = (ctypes.c_longlong * 6)()
        _lib.check(_lib.load().evp_newton_stats(self._h, v))
        keys = ("eval_passes", "evaluations", "newton_steps", "hardening_updates", "voxels", "newton_passes")
        return dict(zip(keys, (int(x) for x in v)))

    def stats(self) -> _lib.Report:
        rep = _lib.Report()
        _lib.check(_lib.load().evp_stats(self._h, ctypes.byref(rep)))
        return rep

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().evp_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_results(path) -> np.ndarray:
    """results.csv as a float array (columns RESULTS_COLS)."""
    return np.loadtxt(Path(path), delimiter=",", skiprows=1, ndmin=2)


class Batch:
    """Many solves advanced together (``evp_batch_*`` of ``include/evp.h``): one launch per pass
    of every equilibrium iteration over all running members, a device-side controller for each
    member's serial tail, the iterations replayed as a CUDA graph.  Members start and finish
    increments independently; each member's results equal those of its solve alone."""

    def __init__(self):
        L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(L.evp_batch_open(ctypes.byref(h)))
        self._h = h

    def add(self, fft_in, out_dir="", mix=1, modal=0, write_files=False, csv_only=True, precision=0) -> int:
        """Open one solve as a member; returns its slot.  Raises EvpError on a deck or start-up error."""
        flags = (WRITE_FILES if write_files else 0) | (WRITE_CSV if csv_only else 0) | (MIXED if precision else 0)
        slot = ctypes.c_int(-1)
        _lib.check(_lib.load().evp_batch_add(self._h, str(fft_in).encode(), str(out_dir).encode(), int(mix), int(modal),
                                             flags, ctypes.byref(slot)))
        return int(slot.value)

    def step(self, rounds: int = 1) -> int:
        """Advance every running member by a few rounds of iterations; returns how many still run."""
        n = ctypes.c_int(0)
        _lib.check(_lib.load().evp_batch_step(self._h, int(rounds), ctypes.byref(n)))
        return int(n.value)

    def run(self) -> None:
        while self.step(16) > 0:
            pass

    def status(self, slot: int) -> dict:
        st, rep = ctypes.c_int(0), _lib.Report()
        msg = ctypes.create_string_buffer(512)
        _lib.check(_lib.load().evp_batch_status(self._h, int(slot), ctypes.byref(st), ctypes.byref(rep), msg, 512))
        return {"state": "done" if st.value == 1 else "running", "status": rep.status, "macrosteps": rep.macrosteps,
                "equilibrium_iters": rep.equilibrium_iters, "voxel_iters": rep.voxel_iters, "wall_s": rep.wall_s,
                "grid": (rep.n1, rep.n2, rep.n3), "error": msg.value.decode(errors="replace")}

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().evp_batch_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_files(ffts, out_dirs, mix=1, modal=0, csv_only=False, precision=0) -> list:
    """Run every deck to its end as one batch (``evp_solve_files``); one Report per deck."""
    n = len(ffts)
    arr_in = (ctypes.c_char_p * n)(*[str(f).encode() for f in ffts])
    arr_out = (ctypes.c_char_p * n)(*[str(o).encode() for o in out_dirs])
    reps = (_lib.Report * n)()
    flags = (WRITE_CSV if csv_only else WRITE_FILES) | (MIXED if precision else 0)
    rc = _lib.load().evp_solve_files(n, arr_in, arr_out, int(mix), int(modal), flags, reps)
    out = [reps[i] for i in range(n)]
    if rc != 0 and all(r.status == 0 for r in out):
        _lib.check(rc)
    return out
