"""Command line with the reference executable's flags (``lsevpfft/src/LS-EVPFFT.f90:87-142``).

    LS-EVPFFT --in FILE --out DIR --nthreads n --fftw_save PATH --mix 0/1 --modal 0/1

Unknown flags print the reference's message and stop.  Exit status: 0 on
success, 1 on a solver error (the reference's ``stop 1`` paths); a deck error
also exits 1 here, where the Fortran ``stop 'msg'`` exits 0 (callers treat
both through the missing/short results.csv path).  With ``EVP_SERVER_SOCKET``
naming a running ``python -m creep_modeling_b200.serve`` socket, the solve is
submitted there instead of running in this process.
"""
from __future__ import annotations

import os
import sys


HELP = """Optional inputs:
--in FILE | name of input file (fft.in by default)
--out DIR | output directory (evpfft_outputs by default)
--nthreads n | number of threads to run with (# physical cpu cores by default)
--save FILE | path to FFTW wisdom file (default: <outdir>/fftw_wisdom.save)
--modal 0-1 | toggle modified AL (default 1)"""


def parse(argv):
    opts = {"in": "fft.in", "out": "evpfft_outputs/", "nthreads": 0, "fftw_save": "", "mix": 1, "modal": 1}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a in ("-h", "--help"):
            print(HELP)
            return None
        key = {"--in": "in", "--out": "out", "--nthreads": "nthreads", "--fftw_save": "fftw_save", "--mix": "mix",
               "--modal": "modal"}.get(a)
        if key is None:
            print(f'Unknown command-line option: "{a}" use -h or --help for argument list')
            return None
        val = argv[i + 1] if i + 1 < len(argv) else ""
        if key in ("nthreads", "mix", "modal"):
            v = int(val)
            opts[key] = (1 if v != 0 else 0) if key in ("mix", "modal") else v
        else:
            opts[key] = val
        i += 2
    return opts


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    opts = parse(argv)
    if opts is None:
        return 0
    from . import solver
    from ._lib import EvpError

    sock = os.environ.get("EVP_SERVER_SOCKET")
    if sock and os.path.exists(sock):  # serving mode: the resident server runs the solve
        from .serve import submit_via_socket

        st = submit_via_socket(sock, opts["in"], opts["out"], opts["mix"], opts["modal"])
        if st.get("status", -7) != 0:
            print(f"\n[{st.get('status')}] {st.get('error', '')}", file=sys.stderr)
            return 1
        print(f"\nMACROSTEPS={st['macrosteps']} VOXEL_ITERS={st['voxel_iters']} LATENCY={st['latency_s']:.3f}s (served)")
        return 0
    try:
        rep = solver.run_solver(opts["in"], opts["out"], opts["nthreads"], opts["fftw_save"], opts["mix"], opts["modal"])
    except EvpError as e:
        print(f"\n{e}", file=sys.stderr)
        return 1
    print(f"\nMACROSTEPS={rep.macrosteps} ITERS={rep.equilibrium_iters} VOXEL_ITERS={rep.voxel_iters} "
          f"GPU={rep.gpu_s:.3f}s WALL={rep.wall_s:.3f}s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
