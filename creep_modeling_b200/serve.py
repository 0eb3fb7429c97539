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
written, so concurrent shim processes (calibrate.py's) share one GPU.  Requests
and answers are JSON (never pickled objects), every request field is checked,
and the socket file is created with mode 0600: only its owner can connect.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import socket
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
    of the free memory); max_inflight: solves running at once; tune_cache: the FFT
    passes' tile cache file (see solver.tune_cache)."""

    def __init__(self, hbm_budget_bytes: int = 0, max_inflight: int = 16, tune_cache=None):
        L = _lib.load()
        h = ctypes.c_void_p()
        tc = str(tune_cache).encode() if tune_cache else None
        _lib.check(L.evp_server_open(int(hbm_budget_bytes), int(max_inflight), tc, ctypes.byref(h)))
        self._h = h
        self._lock = threading.Lock()

    def submit(self, fft_in, out_dir, mix: int = 1, modal: int = 0, precision: int = 0, csv_only: bool = False,
               deadline_s: float | None = None) -> int:
        """Queue one solve; returns its ticket.  csv_only: results/diagnostics without VTK.
        deadline_s: wall-clock budget from admission; an overrunning solve ends with status -8."""
        L = _lib.load()
        t = ctypes.c_ulonglong()
        flags = 4 if csv_only else 1  # EVP_WRITE_CSV / EVP_WRITE_FILES
        _lib.check(L.evp_submit_deadline(self._h, str(fft_in).encode(), str(out_dir).encode(), int(mix), int(modal),
                                         int(precision), flags, float(deadline_s or 0.0), ctypes.byref(t)))
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
# Wire format: one JSON object per connection in each direction, terminated by a
# newline.  JSON carries only data (no pickled objects), requests are checked
# field by field, and the socket file is created with mode 0600 so only its
# owner can connect.
MAX_REQUEST_BYTES = 64 * 1024
_FIELDS = {"in": str, "out": str, "mix": int, "modal": int, "precision": int, "csv_only": bool}


def _read_line(sock, limit: int = MAX_REQUEST_BYTES) -> bytes:
    buf = bytearray()
    while b"\n" not in buf:
        chunk = sock.recv(4096)
        if not chunk:
            break
        buf += chunk
        if len(buf) > limit:
            raise ValueError(f"request longer than {limit} bytes")
    return bytes(buf.split(b"\n", 1)[0])


def parse_request(raw: bytes) -> dict:
    """Decode and check one request: {"in": str, "out": str} plus optional mix, modal,
    precision (ints) and csv_only (bool).  Raises ValueError on anything else."""
    try:
        req = json.loads(raw.decode("utf-8"))
    except (UnicodeDecodeError, json.JSONDecodeError) as e:
        raise ValueError(f"not a JSON object: {e}") from None
    if not isinstance(req, dict):
        raise ValueError("request must be a JSON object")
    extra = set(req) - set(_FIELDS)
    if extra:
        raise ValueError(f"unknown fields {sorted(extra)}")
    for key in ("in", "out"):
        if key not in req:
            raise ValueError(f"missing field {key!r}")
    out = {"mix": 1, "modal": 0, "precision": 0, "csv_only": False}
    for key, typ in _FIELDS.items():
        if key not in req:
            continue
        v = req[key]
        ok = isinstance(v, typ) and not (typ is int and isinstance(v, bool))
        if not ok or (typ is str and (not v or "\0" in v)):
            raise ValueError(f"field {key!r} must be a {typ.__name__}")
        out[key] = v
    return out


def serve_socket(path: str, backend, stop: threading.Event | None = None) -> None:
    """Accept requests on a Unix socket and answer each with its final status.

    A request is the JSON object {"in", "out", "mix", "modal", "precision",
    "csv_only"}; the answer is the status dict of :meth:`Server.wait`, or
    {"status": -7, "error": ...} for a malformed request.  ``backend`` is a
    :class:`Server` (anything with its submit/wait methods).  Each connection is
    served on its own thread, so a client blocks only on its own solve."""
    if os.path.exists(path):
        os.unlink(path)
    lsock = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
    old = os.umask(0o177)  # the socket file is created owner read/write only
    try:
        lsock.bind(path)
    finally:
        os.umask(old)
    os.chmod(path, 0o600)
    lsock.listen(64)

    def answer(conn, obj):
        conn.sendall(json.dumps(obj).encode() + b"\n")

    def handle(conn):
        try:
            try:
                req = parse_request(_read_line(conn))
            except ValueError as e:
                answer(conn, {"state": "done", "status": -7, "error": f"bad request: {e}"})
                return
            try:
                t = backend.submit(req["in"], req["out"], req["mix"], req["modal"], req["precision"], req["csv_only"])
            except _lib.EvpError as e:
                answer(conn, {"state": "done", "status": e.code, "error": str(e)})
                return
            answer(conn, backend.wait(t))
        except OSError:
            pass
        finally:
            conn.close()

    try:
        while stop is None or not stop.is_set():
            try:
                conn, _ = lsock.accept()
            except OSError:
                break
            threading.Thread(target=handle, args=(conn,), daemon=True).start()
    finally:
        lsock.close()


def submit_via_socket(path: str, fft_in, out_dir, mix: int = 1, modal: int = 0, precision: int = 0,
                      csv_only: bool = False) -> dict:
    """Send one request to a socket server and wait for its final status."""
    with socket.socket(socket.AF_UNIX, socket.SOCK_STREAM) as c:
        c.connect(path)
        req = {"in": str(fft_in), "out": str(out_dir), "mix": int(mix), "modal": int(modal), "precision": int(precision),
               "csv_only": bool(csv_only)}
        c.sendall(json.dumps(req).encode() + b"\n")
        raw = _read_line(c, 1 << 20)
    return json.loads(raw.decode()) if raw else {"state": "done", "status": -7, "error": "server closed the connection"}


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
