"""Serving: one resident solver process per GPU that takes solve requests.

The reference answers every request with a new ``LS-EVPFFT`` process
(``utils/run.py:169-196``); ``calibrate.py`` runs two or three of them at once
(``calibrate.py:1053-1057``).  Here a :class:`Server` (the ``evp_server_*``
entry points of ``include/evp.h``) keeps the GPU busy with many solves at once:
requests queue in arrival order, are admitted while their device-memory
estimates fit the budget, and run concurrently, each on its own CUDA stream,
writing the same files as the executable.

``python -m creep_modeling_b200.serve --socket PATH`` hosts a server behind a
local Unix socket.  With ``EVP_SERVER_SOCKET=PATH`` in its environment the
``LS-EVPFFT`` shim submits its solve there and blocks until the files are
written, so concurrent shim processes (calibrate.py's) share one GPU.  The
socket has no authentication: any local user who can open it can submit decks,
so create it in a directory only the intended users can reach.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import threading
from pathlib import Path

from . import _lib

STATE = {0: "queued", 1: "running", 2: "done"}


def _status_dict(st: _lib.Status) -> dict:
    return {
        "state": STATE.get(st.state, str(st.state)), "status": st.status, "macrosteps": st.macrosteps,
        "grid": (st.n1, st.n2, st.n3), "voxel_iters": st.voxel_iters, "queued_s": st.queued_s, "run_s": st.run_s,
        "latency_s": st.latency_s, "footprint_bytes": st.footprint_bytes, "error": st.error.decode(errors="replace"),
    }


class Server:
    """A resident request loop on the current GPU.

    hbm_budget_bytes: device memory the running solves may hold together (0: 85 %
    of the free memory); max_inflight: solves running at once."""

    def __init__(self, hbm_budget_bytes: int = 0, max_inflight: int = 16):
        L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(L.evp_server_open(int(hbm_budget_bytes), int(max_inflight), None, ctypes.byref(h)))
        self._h = h
        self._lock = threading.Lock()

    def submit(self, fft_in, out_dir, mix: int = 1, modal: int = 0, precision: int = 0, csv_only: bool = False) -> int:
        """Queue one solve; returns its ticket.  csv_only: results/diagnostics without VTK."""
        L = _lib.load()
        t = ctypes.c_ulonglong()
        flags = 4 if csv_only else 1  # EVP_WRITE_CSV / EVP_WRITE_FILES
        _lib.check(L.evp_submit(self._h, str(fft_in).encode(), str(out_dir).encode(), int(mix), int(modal),
                                int(precision), flags, ctypes.byref(t)))
        return int(t.value)

    def poll(self, ticket: int) -> dict:
        st = _lib.Status()
        _lib.check(_lib.load().evp_poll(self._h, int(ticket), ctypes.byref(st)))
        return _status_dict(st)

    def wait(self, ticket: int, timeout: float | None = None) -> dict:
        """Block until the request is done (or timeout seconds pass; then its state is not "done")."""
        st = _lib.Status()
        rc = _lib.load().evp_wait(self._h, int(ticket), -1.0 if timeout is None else float(timeout), ctypes.byref(st))
        if rc < 0:
            _lib.check(rc)
        return _status_dict(st)

    def close(self) -> None:
        """Let queued and running solves finish, then release the server."""
        if self._h:
            _lib.load().evp_server_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------- local socket front end
def serve_socket(path: str, backend, stop: threading.Event | None = None) -> None:
    """Accept requests on a Unix socket and answer each with its final status.

    A request is a dict {"in", "out", "mix", "modal", "precision", "csv_only"};
    the answer is the status dict of :meth:`Server.wait`, or {"status": -7,
    "error": ...} for a malformed request.  ``backend`` is a :class:`Server`
    (anything with its submit/wait methods).  Each connection is served on its
    own thread, so a client blocks only on its own solve."""
    from multiprocessing.connection import Listener

    if os.path.exists(path):
        os.unlink(path)
    listener = Listener(path, family="AF_UNIX")

    def handle(conn):
        try:
            req = conn.recv()
            try:
                t = backend.submit(req["in"], req["out"], int(req.get("mix", 1)), int(req.get("modal", 0)),
                                   int(req.get("precision", 0)), bool(req.get("csv_only", False)))
            except _lib.EvpError as e:
                conn.send({"state": "done", "status": e.code, "error": str(e)})
                return
            except (KeyError, TypeError, ValueError) as e:
                conn.send({"state": "done", "status": -7, "error": f"bad request: {e}"})
                return
            conn.send(backend.wait(t))
        except EOFError:
            pass
        finally:
            conn.close()

    try:
        while stop is None or not stop.is_set():
            try:
                conn = listener.accept()
            except OSError:
                break
            threading.Thread(target=handle, args=(conn,), daemon=True).start()
    finally:
        listener.close()


def submit_via_socket(path: str, fft_in, out_dir, mix: int = 1, modal: int = 0, precision: int = 0,
                      csv_only: bool = False) -> dict:
    """Send one request to a socket server and wait for its final status."""
    from multiprocessing.connection import Client

    with Client(path, family="AF_UNIX") as c:
        c.send({"in": str(fft_in), "out": str(out_dir), "mix": int(mix), "modal": int(modal), "precision": int(precision),
                "csv_only": bool(csv_only)})
        return c.recv()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Host an LS-EVPFFT solve server on this GPU behind a Unix socket.")
    ap.add_argument("--socket", required=True, help="socket path (clients: EVP_SERVER_SOCKET=PATH LS-EVPFFT ...)")
    ap.add_argument("--budget-gb", type=float, default=0.0, help="device memory for running solves (0: 85%% of free)")
    ap.add_argument("--max-inflight", type=int, default=16)
    args = ap.parse_args(argv)
    with Server(int(args.budget_gb * 2**30), args.max_inflight) as srv:
        try:
            serve_socket(str(Path(args.socket)), srv)
        except KeyboardInterrupt:
            pass
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
