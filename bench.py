#!/usr/bin/env python3
"""Throughput benchmark of the B200 LS-EVPFFT solve (plain FP64 path).

Workload (one B200): large-strain strain-rate-controlled tension, 64^3 voxels,
500 periodic-Voronoi grains (seed 2), FCC power law n=20, udot33=1e-3/s,
dt=0.5 s increments with lattice rotation and grid update (iupdate=1).
Synthetic seeded inputs in the reference's file grammar stand in for the
reference's (unshipped) microstructures.  A "step" is one macrostep
(increment): every equilibrium iteration it needs plus the large-strain
updates.  Metric: voxel-iters/s = voxels x equilibrium iterations / device
seconds (CUDA events on the solver's stream, max over ranks).  The state
(~2 kB/voxel, 0.5 GB) is larger than the 126 MB L2, so no flush is needed.
The line's "batch" object times the calibration sweep batched against one solve
after another (batch_sample), and its "serving" object the served request stream
against the plain path (serving_stream).

--gpus N > 1 runs N independent replicas (the solve does not shard), one
process per GPU, and sums their voxel-iters.
--impl reference times the CPU oracle (a C++ restatement of the reference
Fortran/OpenMP solver; the Fortran build itself cannot be compiled here) on
the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "voxel-iters/s"
# Algorithmic HBM bytes per voxel and launch of the equilibrium-iteration kernels
# (FP64 state, 12 slip systems; spectrum terms scale with (n1/2+1)/n1).
def algorithmic_bytes(n1: int, nsys: int = 12) -> dict:
    half = (n1 // 2 + 1) / n1
    spec = 9 * 16 * half  # one pass over the 9-component half spectrum, per voxel
    return {
        "k_sgavg": 7 * 8,
        "k_fft_x_fwd": 16 * 8 + spec,
        "k_fft_y_fwd": 2 * spec,
        "k_fft_z_green": 2 * spec,
        "k_fft_y_inv": 2 * spec,
        "k_fft_x_inv": spec + (9 + 1 + 9) * 8,
        "k_corr": (9 * 4 + 1) * 8 + 1 + 9 * 2 * 8,
        # velgrad 9, sg 6, sgt 6, wgtc 1, trialtau 2n, gacumgr 1, crss 2n, sch 5n, C~ 36, S 36 | sg 6, edotp 6, gamdot n, trialtau 2n
        "k_newton": (9 + 6 + 6 + 1 + 2 * nsys + 1 + 2 * nsys + 5 * nsys + 36 + 36 + 6 + 6 + nsys + 2 * nsys) * 8 + 2,
    }


# Counted FP64 arithmetic of k_newton6p (12 slip systems; a fused multiply-add counts 2, a division
# 1, the integer power |x|^(n-1) by binary powering 8): one constitutive evaluation (resolved shear,
# power law, plastic strain rate, residual rho and C~ rho, their norm) 612; one Newton step (the
# tangent dd, the rows of H, Gauss-Jordan on the 6x6 system, the update and its norm) 1000; one
# hardening update (Voce increment, the 12 x 12 latent-hardening product, the resistance change) 780.
NEWTON_FLOPS = {"evaluation": 612, "newton_step": 1000, "hardening_update": 780}


def fp64_peak_tflops(dev) -> float:
    """Measured FP64 rate of this GPU: cuBLAS DGEMM (torch float64 matmul, 8192^3), best of 5."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(5):
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or not f[0].isdigit() or int(f[0]) != self.index:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def aggregate_replicas(pg, seconds: float, voxel_iters: float, device) -> tuple[float, float]:
    """Whole-job figures of N independent replicas (one solve per rank, no data exchange): the
    slowest rank's device time and the voxel-iterations of all ranks.  pg is torch.distributed
    (or None for one process); the two reductions run in the same order on every rank."""
    if pg is None:
        return float(seconds), float(voxel_iters)
    import torch

    t = torch.tensor([float(seconds), float(voxel_iters)], dtype=torch.float64, device=device)
    tmax = t.clone()
    pg.all_reduce(tmax, op=pg.ReduceOp.MAX)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(tmax[0]), float(t[1])


def make_deck(root: Path, n: int, nsteps: int, ngrains: int) -> Path:
    from creep_modeling_b200 import decks

    case = decks.case_c2(nsteps=nsteps, n=n, ngrains=ngrains)
    return decks.write_case(case, root)


WORKLOAD = "tension {n}^3, {g} grains, n=20, udot33=1e-3/s, dt=0.5 s, iupdate=1"


def cpu_baseline(fft: Path, warmup: int, nmacro: int, budget_s: float) -> dict:
    """The oracle on all host cores, on a bounded sample of the same workload: the increments
    after the warm-up ones, as the device figure times them, until nmacro are done or
    budget_s of timed CPU work has passed."""
    import oracle

    threads = os.cpu_count() or 1
    s = oracle.OracleSolve(fft, mix=1, modal=0, nthreads=threads)
    for _ in range(warmup):
        s.advance(1)
    done = 0
    iters0 = s.total_iters()
    t0 = time.perf_counter()
    while done < nmacro:
        if s.advance(1) != 1:
            break
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    vi = (s.total_iters() - iters0) * s.nvox
    s.close()
    return {"value": vi / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"increments {warmup + 1}-{warmup + done} of the same {s.shape[0]}^3 tension deck "
                      f"({vi} voxel-iters, {dt:.1f} s)"}


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    n = args.n
    with tempfile.TemporaryDirectory() as td:
        fft = make_deck(Path(td), n, args.warmup + args.steps + 1, args.ngrains)
        import oracle

        threads = os.cpu_count() or 1
        s = oracle.OracleSolve(fft, mix=1, modal=0, nthreads=threads)
        budget = args.ref_budget
        t_all = time.perf_counter()
        for _ in range(args.warmup):  # the same untimed increments as the device arm
            s.advance(1)
        it0 = s.total_iters()
        t0 = time.perf_counter()
        done = 0
        for _ in range(args.steps):
            s.advance(1)
            done += 1
            if time.perf_counter() - t_all > budget:
                break
        dt = time.perf_counter() - t0
        vi = (s.total_iters() - it0) * s.nvox
        value = vi / dt
        sample = (f"increments {args.warmup + 1}-{args.warmup + done} (after {args.warmup} untimed) of the {n}^3 "
                  f"tension deck on {threads} host threads (C++ FP64 restatement of the reference Fortran solver)")
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": done,
                "warmup": args.warmup, "ms_per_step": dt / max(done, 1) * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD.format(n=n, g=args.ngrains), "voxels": n ** 3,
                           "increments_timed": f"{args.warmup + 1}-{args.warmup + done}",
                           "l2": "state larger than L2"},
                "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    return 0


def fft_vs_cufft(kd: dict, iters: int, n: int, dev) -> dict:
    """The five FFT passes of one equilibrium iteration (PK1 prologue, x R2C, y, z with the
    Green-operator product, y inverse, x C2R with the correction epilogue; their average
    device time per iteration from the profiled increments) beside cuFFT (through
    torch.fft) doing only the real-to-complex and complex-to-real 3-D transforms of the
    same nine FP64 fields, timed with CUDA events.  A timing comparison, not a product path."""
    import torch

    ours = sum(kd.get(k, (0, 0.0))[1] for k in ("k_fft_x_fwd", "k_fft_y_fwd", "k_fft_z_green", "k_fft_y_inv",
                                                 "k_fft_x_inv")) / max(iters, 1)
    x = torch.randn(9, n, n, n, dtype=torch.float64, device=dev)
    for _ in range(3):
        y = torch.fft.irfftn(torch.fft.rfftn(x, dim=(1, 2, 3)), s=(n, n, n), dim=(1, 2, 3))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    torch.cuda.synchronize(dev)
    a.record()
    for _ in range(reps):
        y = torch.fft.irfftn(torch.fft.rfftn(x, dim=(1, 2, 3)), s=(n, n, n), dim=(1, 2, 3))
    b.record()
    torch.cuda.synchronize(dev)
    cu = a.elapsed_time(b) / reps
    del y
    return {"grid": f"{n}^3 x 9 fields FP64", "ours_five_passes_ms": ours, "cufft_r2c_c2r_ms": cu,
            "ratio_cufft_over_ours": cu / ours if ours else None,
            "note": "ours includes the PK1 prologue, the Green-operator product and the correction epilogue; "
                    "cuFFT does the transforms only (torch.fft)"}


def _curves(path: Path):
    import numpy as np

    return np.loadtxt(path, delimiter=",", skiprows=1, ndmin=2)


def _curve_err(a, b) -> float:
    """Largest difference of the results.csv tensor curves (eav, sav, epav, eelav, vgrad, edotp), each
    relative to its tensor's largest magnitude over the run."""
    import numpy as np

    if a.shape != b.shape:
        return float("inf")
    err = 0.0
    for g in range(6):
        cols = list(range(7 + 6 * g, 13 + 6 * g))
        scale = float(np.max(np.abs(b[:, cols])))
        if scale > 1e-30:
            err = max(err, float(np.max(np.abs(a[:, cols] - b[:, cols])) / scale))
    return err


def _plain_solve(fft, out):
    """One solve through the plain single-solve path (evp_open / evp_advance / evp_close, the
    steps of evp_solve_file) writing results.csv and diagnostics.csv, as the batched and served
    legs do; returns its report."""
    from creep_modeling_b200 import solver as S

    s = S.Solve(fft, out_dir=str(out), mix=1, modal=0, csv_only=True)
    s.run()
    rep = s.stats()
    s.close()
    return rep


def batch_sample(k: int, nsteps: int) -> dict:
    """The calibration sweep (configuration 4: grids 16^3-64^3, tau0, n and theta0 drawn per solve, creep
    at 120 MPa) on its first k solves at the full increment count: all of them as one batch
    (evp_solve_files) against one after the other through the plain single-solve path (as the
    reference's callers run one solver process per solve).  Same decks; both write results.csv and
    diagnostics.csv only; the batch members' results.csv must equal the one-by-one ones."""
    from creep_modeling_b200 import decks
    from creep_modeling_b200 import solver as S

    td = Path(tempfile.mkdtemp(prefix="evp_batch_"))
    cases = [decks.case_c4(i, nsteps) for i in range(k)]
    ffts = [decks.write_case(c, td / f"d{i}") for i, c in enumerate(cases)]
    t0 = time.perf_counter()
    reps = S.solve_files(ffts, [td / f"b{i}" for i in range(k)], mix=1, modal=0, csv_only=True)
    tb = time.perf_counter() - t0
    # the configuration's FP32/FP64 split: the same batch with FP32 spectra (mixed precision)
    t0 = time.perf_counter()
    repm = S.solve_files(ffts, [td / f"m{i}" for i in range(k)], mix=1, modal=0, csv_only=True, precision=1)
    tm = time.perf_counter() - t0
    t0 = time.perf_counter()
    seq = [_plain_solve(f, td / f"s{i}") for i, f in enumerate(ffts)]
    ts = time.perf_counter() - t0
    same = all(_curve_err(_curves(td / f"b{i}" / "results.csv"), _curves(td / f"s{i}" / "results.csv")) == 0.0
               for i in range(k))
    errm = max(_curve_err(_curves(td / f"m{i}" / "results.csv"), _curves(td / f"s{i}" / "results.csv"))
               for i in range(k) if repm[i].status == 0) if any(r.status == 0 for r in repm) else None
    vb = sum(r.voxel_iters for r in reps)
    vm = sum(r.voxel_iters for r in repm)
    vs = sum(r.voxel_iters for r in seq)
    return {"config": "calibration sweep (configuration 4)", "solves": k, "increments": nsteps,
            "edges": [c.n for c in cases], "status": [r.status for r in reps],
            "batched": {"wall_s": tb, "solves_per_hour": k / tb * 3600.0, "voxel_iters_per_s": vb / tb},
            "batched_mixed": {"wall_s": tm, "solves_per_hour": k / tm * 3600.0, "voxel_iters_per_s": vm / tm,
                              "status": [r.status for r in repm], "max_curve_rel_err_vs_fp64": errm},
            "one_by_one": {"wall_s": ts, "solves_per_hour": k / ts * 3600.0, "voxel_iters_per_s": vs / ts},
            "speedup": ts / tb, "speedup_mixed": ts / tm, "results_identical": bool(same),
            "sample": f"first {k} of the 256 sweep solves, all {nsteps} increments; batched in plain FP64 "
                      f"(bit-identical to one by one) and in the FP32/FP64 split; one by one in plain FP64"}


def serving_stream(k: int, rate: float) -> dict:
    """The served request stream (configuration 5: grid edges 16-96, Arrhenius-scaled gamma0 at
    475/525/575, creep 80-220 MPa, 50-400 increments) on its first k requests at their full increment
    counts, arriving as a Poisson stream of `rate` per s.  Served: one resident server, mixed precision,
    every admitted solve in one batch (continuous batching); latency = arrival -> files written.
    Plain: the FP64 single-solve path, one solve after the other in arrival order (as the reference's
    run.py runs one process per request), latency = arrival -> its solve's end.  Both write
    results.csv and diagnostics.csv only.
    Error: largest curve difference of every served (mixed) result against its plain FP64 result."""
    import numpy as np

    from creep_modeling_b200 import decks
    from creep_modeling_b200 import solver as S
    from creep_modeling_b200.serve import Server

    td = Path(tempfile.mkdtemp(prefix="evp_serve_"))
    cases = [decks.case_c5(i) for i in range(k)]
    ffts = [decks.write_case(c, td / f"r{i}") for i, c in enumerate(cases)]  # untimed
    arr = decks.stream_arrivals(k, rate)
    # served
    with Server(0, 64) as srv:
        t0 = time.perf_counter()
        tickets = []
        for i, f in enumerate(ffts):
            dt = arr[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            tickets.append(srv.submit(f, td / f"o{i}", mix=1, modal=0, precision=1, csv_only=True))
        sts = [srv.wait(t) for t in tickets]
        span = time.perf_counter() - t0
    ok = [i for i, s in enumerate(sts) if s["status"] == 0]
    lat = np.array([sts[i]["latency_s"] for i in ok])
    served = {"completed": len(ok), "makespan_s": span, "solves_per_hour": len(ok) / span * 3600.0,
              "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
              "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
              "voxel_iters_per_s": sum(sts[i]["voxel_iters"] for i in ok) / span,
              "failed": [{"request": i, "status": s["status"], "error": s["error"][:120]} for i, s in enumerate(sts)
                         if s["status"] != 0]}
    # plain FP64, one by one in arrival order
    t0 = time.perf_counter()
    ends, vi, pok = [], 0, 0
    for i, f in enumerate(ffts):
        dt = arr[i] - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        try:
            r = _plain_solve(f, td / f"p{i}")
            vi += r.voxel_iters
            pok += 1
        except Exception:
            pass
        ends.append(time.perf_counter() - t0)
    pspan = time.perf_counter() - t0
    plat = np.array([ends[i] - arr[i] for i in range(k)])
    plain = {"completed": pok, "makespan_s": pspan, "solves_per_hour": pok / pspan * 3600.0,
             "p50_s": float(np.percentile(plat, 50)), "p99_s": float(np.percentile(plat, 99)),
             "voxel_iters_per_s": vi / pspan}
    errs = [_curve_err(_curves(td / f"o{i}" / "results.csv"), _curves(td / f"p{i}" / "results.csv")) for i in ok]
    return {"config": "served request stream (configuration 5)", "requests": k, "arrival_rate_per_s": rate,
            "edges": [c.n for c in cases], "increments": [c.processes[0].nsteps for c in cases],
            "served_mixed_batched": served, "plain_fp64_one_by_one": plain,
            "solves_per_hour_ratio": served["solves_per_hour"] / plain["solves_per_hour"],
            "max_curve_rel_err_vs_fp64": max(errs) if errs else None,
            "sample": f"first {k} requests of the seeded stream, full increment counts, Poisson arrivals {rate}/s"}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64, help="grid edge (default: the 64^3 configuration)")
    ap.add_argument("--ngrains", type=int, default=500)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--cpu-budget", type=float, default=25.0, help="seconds of timed CPU work in the cpu_baseline leg")
    ap.add_argument("--ref-budget", type=float, default=300.0, help="seconds of CPU time for --impl reference")
    ap.add_argument("--serve-requests", type=int, default=12, help="requests of the served stream (0: skip)")
    ap.add_argument("--batch-solves", type=int, default=8, help="solves of the calibration-sweep batch (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=150, help="increments of each sweep solve")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)

    import torch

    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    else:
        torch.cuda.set_device(0)
    from creep_modeling_b200 import Solve

    dev = torch.device("cuda", local if ws > 1 else 0)
    n = args.n
    td = tempfile.mkdtemp(prefix=f"evp_bench_r{rank}_")
    fft = make_deck(Path(td), n, args.warmup + args.steps + 1, args.ngrains)

    # 1. the device figure: increments W+1..W+K, CUDA events on the solver's stream, no per-kernel timers
    s = Solve(fft, mix=1, modal=0)
    for _ in range(args.warmup):
        s.advance(1)
    clocks = ClockSampler(local if ws > 1 else 0)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    st0 = s.stats()
    l0 = s.launches()
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.advance(1)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    if pg:
        pg.barrier()
    st1 = s.stats()
    launches = s.launches() - l0
    s.close()
    gpu_s = st1.gpu_s - st0.gpu_s
    vi = (st1.equilibrium_iters - st0.equilibrium_iters) * (n ** 3)
    iters = st1.equilibrium_iters - st0.equilibrium_iters
    gpu_s_max, vi_tot = aggregate_replicas(pg, gpu_s, vi, dev)
    value = vi_tot / gpu_s_max

    # 2. end to end through the C ABI on the same increments: a second solve of the same deck
    #    writing results.csv and diagnostics.csv, host wall clock around its K increments (every
    #    increment uploads its reference-medium constants and reads its sums and rows back)
    e2e = None
    try:
        out = Path(td) / "e2e_out"
        s2 = Solve(fft, out_dir=out, mix=1, modal=0, csv_only=True)
        for _ in range(args.warmup):
            s2.advance(1)
        r0 = s2.stats()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s2.advance(1)
        torch.cuda.synchronize(dev)
        we = time.perf_counter() - t0
        r1 = s2.stats()
        s2.close()
        vi2 = (r1.equilibrium_iters - r0.equilibrium_iters) * (n ** 3)
        e2e = {"value": vi2 / we, "unit": METRIC,
               "h2d_bytes_per_step": int((r1.h2d_bytes - r0.h2d_bytes) / max(args.steps, 1)),
               "d2h_bytes_per_step": int((r1.d2h_bytes - r0.d2h_bytes) / max(args.steps, 1)),
               "increments": f"{args.warmup + 1}-{args.warmup + args.steps}",
               "same_iterations_as_device": bool(vi2 == vi),
               "note": "evp_advance through the C ABI with results/diagnostics CSV written, host wall clock"}
        # the whole solve as a caller runs it: deck files -> evp_solve_file -> output files
        from creep_modeling_b200 import solver as _solver

        t0 = time.perf_counter()
        rep = _solver.run_solver(fft, Path(td) / "whole_out", mix=1, modal=0)
        wt = time.perf_counter() - t0
        e2e["whole_solve"] = {"value": rep.voxel_iters / wt, "unit": METRIC, "increments": rep.macrosteps,
                              "wall_s": wt, "note": "evp_solve_file: deck parse + upload + every increment + "
                                                    "results, diagnostics and VTK files"}
    except Exception as exc:  # pragma: no cover - reported, not hidden
        e2e = {"value": None, "unit": METRIC, "error": str(exc)}

    # 3. per-kernel device times on the same increments of a third, profiled solve (an event pair
    #    around every launch): the roofline of the dominant kernel and the kernel shares
    sp = Solve(fft, mix=1, modal=0, profile=True)
    for _ in range(args.warmup):
        sp.advance(1)
    kt0, p0, ns0 = sp.kernel_times(), sp.stats(), sp.newton_stats()
    for _ in range(args.steps):
        sp.advance(1)
    kt1, p1, ns1 = sp.kernel_times(), sp.stats(), sp.newton_stats()
    sp.close()
    nst = {k: ns1[k] - ns0[k] for k in ns1}
    kd = {}
    for k, (cnt, ms) in kt1.items():
        c0, m0 = kt0.get(k, (0, 0.0))
        kd[k] = (cnt - c0, ms - m0)
    piters = p1.equilibrium_iters - p0.equilibrium_iters

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return 0

    peak, peak_kind = load_peaks()
    ab = algorithmic_bytes(n)
    dom = max(kd, key=lambda k: kd[k][1]) if kd else None
    roof = None
    if dom:
        cnt, ms = kd[dom]
        avg_s = ms / 1e3 / max(cnt, 1)
        bytes_launch = ab.get(dom, 0.0) * n ** 3
        ach = bytes_launch / avg_s / 1e9 if bytes_launch else None
        traffic = None
        tp = ROOT / "profiles" / f"{dom}_traffic.json"
        if tp.exists():
            try:
                traffic = json.loads(tp.read_text()).get("bytes_per_launch_scaled")
            except Exception:
                traffic = None
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": (ach / peak if ach else None), "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                "avg_launch_ms": avg_s * 1e3, "algorithmic_bytes_per_launch": bytes_launch,
                "timing": "CUDA events around each launch in a separate profiled solve over the same increments",
                "kernel_share": {k: round(v[1] / max(sum(x[1] for x in kd.values()), 1e-30), 4) for k, v in
                                 sorted(kd.items(), key=lambda kv: -kv[1][1])}}
        if dom == "k_newton" and nst.get("eval_passes"):
            flops = (nst["evaluations"] * NEWTON_FLOPS["evaluation"] + nst["newton_steps"] * NEWTON_FLOPS["newton_step"]
                     + nst["hardening_updates"] * NEWTON_FLOPS["hardening_update"])
            try:
                fpk = fp64_peak_tflops(dev)
            except Exception:  # pragma: no cover
                fpk = None
            ach_tf = flops / (ms / 1e3) / 1e12
            roof["fp64"] = {
                "counted_flops_per_launch": flops / max(cnt, 1), "achieved_tflops": ach_tf,
                "peak_tflops": fpk, "peak_source": "measured cuBLAS DGEMM (torch float64 matmul 8192^3)",
                "frac": (ach_tf / fpk if fpk else None), "flops_model": NEWTON_FLOPS,
                "per_voxel": {"evaluations": nst["evaluations"] / max(nst["voxels"], 1),
                              "newton_steps": nst["newton_steps"] / max(nst["voxels"], 1),
                              "hardening_updates": nst["hardening_updates"] / max(nst["voxels"], 1)},
                "active_slot_fraction": nst["evaluations"] / (5.0 * nst["eval_passes"]),
                "active_slot_fraction_newton": nst["newton_steps"] / (5.0 * max(nst["newton_passes"], 1)),
                "note": "voxel slots: five six-lane groups per warp; a slot idles while the warp waits for its "
                        "slowest voxel"}

    cpu = None
    if not args.no_cpu:
        try:
            cpu = cpu_baseline(fft, args.warmup, args.cpu_steps, args.cpu_budget)
        except Exception as exc:  # pragma: no cover
            cpu = {"value": None, "error": str(exc)}

    fftcmp = None
    try:
        fftcmp = fft_vs_cufft(kd, piters, n, dev)
    except Exception as exc:  # pragma: no cover
        fftcmp = {"error": str(exc)}

    batch = None
    if args.batch_solves > 0:
        try:
            batch = batch_sample(args.batch_solves, args.batch_steps)
        except Exception as exc:  # pragma: no cover - reported, not hidden
            batch = {"error": str(exc)}
    serving = None
    if args.serve_requests > 0:
        try:
            serving = serving_stream(args.serve_requests, 20.0)
        except Exception as exc:  # pragma: no cover - reported, not hidden
            serving = {"error": str(exc)}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": gpu_s_max / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.format(n=n, g=args.ngrains), "voxels": n ** 3, "equilibrium_iters": int(iters),
                   "increments_timed": f"{args.warmup + 1}-{args.warmup + args.steps}", "precision": "plain FP64",
                   "parallelism": f"replicas x{ws}", "l2": "state (~460 MB) larger than L2; no flush"},
        "wall_s": wall, "gpu_launches": int(launches), "clocks": clk, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
        "fft_vs_cufft": fftcmp, "batch": batch, "serving": serving,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
