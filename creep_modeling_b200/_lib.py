"""ctypes binding of ``libevp_b200.so`` (the C ABI declared in ``include/evp.h``).

There is no CPU fallback: if the library cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_build" / "libevp_b200.so"

EXPORTED = (
    "evp_solve_file", "evp_open", "evp_advance", "evp_get_field", "evp_last_rows", "evp_stats", "evp_close",
    "evp_kernel_times", "evp_green_apply", "evp_green_apply_noalloc", "evp_last_error", "evp_version",
    "evp_server_open", "evp_submit", "evp_submit_deadline", "evp_poll", "evp_wait", "evp_server_close",
    "evp_set_deadline", "evp_kernel_launches", "evp_newton_stats",
    "evp_tune_cache", "evp_batch_open", "evp_batch_add", "evp_batch_step", "evp_batch_status", "evp_batch_close", "evp_solve_files",
)

STATUS = {
    0: "ok", -1: "deck or input-file error", -2: "deck feature not supported", -3: "singular matrix",
    -4: "non-convergence or non-finite state", -5: "output-file error", -6: "CUDA error or no device",
    -7: "bad argument", -8: "deadline exceeded",
}


class EvpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}: {STATUS.get(code, 'error')}] {msg}")
        self.code = code


class Report(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("macrosteps", ctypes.c_int),
        ("equilibrium_iters", ctypes.c_longlong),
        ("voxel_iters", ctypes.c_longlong),
        ("wall_s", ctypes.c_double),
        ("gpu_s", ctypes.c_double),
        ("n1", ctypes.c_int),
        ("n2", ctypes.c_int),
        ("n3", ctypes.c_int),
        ("h2d_bytes", ctypes.c_longlong),
        ("d2h_bytes", ctypes.c_longlong),
    ]


class Status(ctypes.Structure):
    """evp_status: the state of one served request."""

    _fields_ = [
        ("state", ctypes.c_int),
        ("status", ctypes.c_int),
        ("macrosteps", ctypes.c_int),
        ("n1", ctypes.c_int),
        ("n2", ctypes.c_int),
        ("n3", ctypes.c_int),
        ("voxel_iters", ctypes.c_longlong),
        ("queued_s", ctypes.c_double),
        ("run_s", ctypes.c_double),
        ("latency_s", ctypes.c_double),
        ("footprint_bytes", ctypes.c_ulonglong),
        ("error", ctypes.c_char * 256),
    ]


_lib = None


def load(path: Path | str | None = None):
    """Load the library (building it first when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        from . import build as _build

        _build.build()
    L = ctypes.CDLL(str(p))
    c_dp = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    L.evp_solve_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(Report)]
    L.evp_solve_file.restype = ctypes.c_int
    L.evp_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.evp_open.restype = ctypes.c_int
    L.evp_advance.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.evp_advance.restype = ctypes.c_int
    L.evp_get_field.argtypes = [vp, ctypes.c_char_p, c_dp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    L.evp_get_field.restype = ctypes.c_int
    L.evp_last_rows.argtypes = [vp, c_dp, c_dp]
    L.evp_last_rows.restype = ctypes.c_int
    L.evp_stats.argtypes = [vp, ctypes.POINTER(Report)]
    L.evp_stats.restype = ctypes.c_int
    L.evp_close.argtypes = [vp]
    L.evp_close.restype = ctypes.c_int
    L.evp_kernel_times.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong), c_dp, ctypes.c_int]
    L.evp_kernel_times.restype = ctypes.c_int
    L.evp_newton_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.evp_newton_stats.restype = ctypes.c_int
    L.evp_tune_cache.argtypes = [ctypes.c_char_p]
    L.evp_tune_cache.restype = ctypes.c_int
    ip = ctypes.POINTER(ctypes.c_int)
    L.evp_batch_open.argtypes = [ctypes.POINTER(vp)]
    L.evp_batch_open.restype = ctypes.c_int
    L.evp_batch_add.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip]
    L.evp_batch_add.restype = ctypes.c_int
    L.evp_batch_step.argtypes = [vp, ctypes.c_int, ip]
    L.evp_batch_step.restype = ctypes.c_int
    L.evp_batch_status.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(Report), ctypes.c_char_p, ctypes.c_int]
    L.evp_batch_status.restype = ctypes.c_int
    L.evp_batch_close.argtypes = [vp]
    L.evp_batch_close.restype = ctypes.c_int
    L.evp_solve_files.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_char_p),
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Report)]
    L.evp_solve_files.restype = ctypes.c_int
    L.evp_kernel_launches.argtypes = [vp]
    L.evp_kernel_launches.restype = ctypes.c_longlong
    L.evp_green_apply.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp, c_dp, vp]
    L.evp_green_apply.restype = ctypes.c_int
    L.evp_green_apply_noalloc.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp, c_dp, vp]
    L.evp_green_apply_noalloc.restype = ctypes.c_int
    L.evp_last_error.argtypes = []
    L.evp_last_error.restype = ctypes.c_char_p
    L.evp_version.argtypes = []
    L.evp_version.restype = ctypes.c_int
    u64 = ctypes.c_ulonglong
    L.evp_server_open.argtypes = [u64, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(vp)]
    L.evp_server_open.restype = ctypes.c_int
    L.evp_submit.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.POINTER(u64)]
    L.evp_submit.restype = ctypes.c_int
    L.evp_submit_deadline.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, ctypes.POINTER(u64)]
    L.evp_submit_deadline.restype = ctypes.c_int
    L.evp_set_deadline.argtypes = [vp, ctypes.c_double]
    L.evp_set_deadline.restype = ctypes.c_int
    L.evp_poll.argtypes = [vp, u64, ctypes.POINTER(Status)]
    L.evp_poll.restype = ctypes.c_int
    L.evp_wait.argtypes = [vp, u64, ctypes.c_double, ctypes.POINTER(Status)]
    L.evp_wait.restype = ctypes.c_int
    L.evp_server_close.argtypes = [vp]
    L.evp_server_close.restype = ctypes.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != 0:
        raise EvpError(rc, (load().evp_last_error() or b"").decode())
