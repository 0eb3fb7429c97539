"""Serving front end on the CPU: the socket protocol and the shim's serving mode.

The GPU server itself is covered by tests/test_gpu_server.py; here a fake
backend with the server's submit/wait methods stands in, so the request
routing, error mapping and the LS-EVPFFT shim's client path run without a GPU.
"""
import ctypes
import os
import threading
import time

import pytest

from creep_modeling_b200 import _lib, cli, serve


class FakeBackend:
    """Records requests; answers like Server.wait; deck 'bad.in' fails like a deck error."""

    def __init__(self):
        self.requests = []

    def submit(self, fft_in, out_dir, mix, modal, precision, csv_only):
        if str(fft_in).endswith("bad.in"):
            raise _lib.EvpError(-1, "cannot open bad.in")
        self.requests.append((str(fft_in), str(out_dir), mix, modal, precision, csv_only))
        return len(self.requests)

    def wait(self, ticket):
        return {"state": "done", "status": 0, "macrosteps": 3, "voxel_iters": 4096 * ticket, "latency_s": 0.01,
                "error": ""}


@pytest.fixture
def fake_server(tmp_path):
    path = str(tmp_path / "evp.sock")
    backend, stop = FakeBackend(), threading.Event()
    th = threading.Thread(target=serve.serve_socket, args=(path, backend, stop), daemon=True)
    th.start()
    for _ in range(200):
        if os.path.exists(path):
            break
        time.sleep(0.01)
    yield path, backend
    stop.set()
    try:  # wake the accept loop so it sees the stop flag
        serve.submit_via_socket(path, "x.in", "o")
    except Exception:
        pass
    th.join(timeout=5)


def test_socket_round_trip(fake_server):
    path, backend = fake_server
    st = serve.submit_via_socket(path, "a/fft.in", "out1", mix=1, modal=0, csv_only=True)
    assert st["status"] == 0 and st["macrosteps"] == 3
    assert backend.requests[0] == ("a/fft.in", "out1", 1, 0, 0, True)


def test_socket_concurrent_clients(fake_server):
    path, backend = fake_server
    res = [None] * 6

    def go(i):
        res[i] = serve.submit_via_socket(path, f"d{i}/fft.in", f"o{i}")

    ths = [threading.Thread(target=go, args=(i,)) for i in range(6)]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=10)
    assert all(r is not None and r["status"] == 0 for r in res)
    assert sorted(r[0] for r in backend.requests) == sorted(f"d{i}/fft.in" for i in range(6))


def test_socket_maps_errors(fake_server):
    path, _ = fake_server
    st = serve.submit_via_socket(path, "bad.in", "o")
    assert st["status"] == -1 and "bad.in" in st["error"]


def test_shim_uses_the_server(fake_server, monkeypatch, capsys):
    path, backend = fake_server
    monkeypatch.setenv("EVP_SERVER_SOCKET", path)
    assert cli.main(["--in", "deck/fft.in", "--out", "res/", "--mix", "1", "--modal", "0"]) == 0
    assert "(served)" in capsys.readouterr().out
    assert backend.requests[-1][:4] == ("deck/fft.in", "res/", 1, 0)
    assert cli.main(["--in", "bad.in", "--out", "res/"]) == 1


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_server_open_without_device():
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.evp_server_open(0, 4, None, ctypes.byref(h)) == -6
    assert b"CUDA" in L.evp_last_error()


def test_socket_file_is_owner_only(fake_server):
    import stat

    path, _ = fake_server
    assert stat.S_IMODE(os.stat(path).st_mode) == 0o600


@pytest.mark.parametrize("raw", [
    b"not json",
    b"[1, 2]",
    b'{"in": "a"}',
    b'{"in": "a", "out": "b", "mix": "1"}',
    b'{"in": "a", "out": "b", "mix": true}',
    b'{"in": 3, "out": "b"}',
    b'{"in": "a", "out": "b", "cmd": "x"}',
    b'{"in": "", "out": "b"}',
])
def test_malformed_requests_are_refused(raw):
    with pytest.raises(ValueError):
        serve.parse_request(raw)


def test_malformed_request_answered_with_status(fake_server):
    import json
    import socket as so

    path, backend = fake_server
    n0 = len(backend.requests)
    with so.socket(so.AF_UNIX, so.SOCK_STREAM) as c:
        c.connect(path)
        c.sendall(b'{"in": "a", "out": "b", "precision": "1"}\n')
        st = json.loads(serve._read_line(c).decode())
    assert st["status"] == -7 and "precision" in st["error"]
    assert len(backend.requests) == n0
