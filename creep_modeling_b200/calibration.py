"""Calibration evaluations as one batch of solves on a resident server.

The reference's calibration loop (``utils/calibrate.py``) scores one candidate
parameter set at a time: ``run_one`` (calibrate.py:980-1040) writes a deck,
runs one ``LS-EVPFFT`` process, loads ``results.csv`` and scores it against
experimental curves; ``run_srj_creep`` (1043-1077) and ``run_multi_load``
(1080-1132) run two or three such solves at once as separate processes.

Unchanged, those calls already share one GPU: with ``EVP_SERVER_SOCKET`` set,
every ``LS-EVPFFT`` shim process submits to the same resident server, which
admits them together and runs them concurrently.  :func:`evaluate_batch` is the
batched form for a caller that owns the loop (for example an optimiser asking
for several candidates per round): all candidate x load solves go to one
:class:`~creep_modeling_b200.serve.Server` at once and are scored with the
reference's objectives when they finish.

Restated from the reference (parity fixtures in ``tests/golden/``):

* aligned error metrics MAE / MSE / MRE and ``nearest_indices``
  (``utils/calc_utils.py:35-105``);
* the experimental-curve loaders ``CreepData.load`` and ``SrjData.load``
  (``utils/data_utils.py:516-640, 723-770``; true strain ``ln(1+e)``, true
  stress ``s(1+e)``, plastic strain by subtracting the second sample,
  ``calc_utils.py:21-32, 318-325``);
* the objectives ``_creep_objective`` (calibrate.py:824-864) and
  ``_srj_objective`` (calibrate.py:755-821), and the per-evaluation loss
  ``base + w_iters * mean(iter)`` (calibrate.py:1027).

The experimental CSVs the reference loads at import (calibrate.py:976-977,
``data/creep_int_95_105_115.csv`` and ``data/CPValidation_316L/StrainRateJump.csv``)
are not part of the reference repository.  :func:`synthetic_creep_csv` and
:func:`synthetic_srj_csv` write clearly synthetic stand-ins with the loaders'
column schema (every creep data column name starts with ``synthetic``); they
are smooth model curves with seeded noise, not measurements.
"""
from __future__ import annotations

import dataclasses
from pathlib import Path

import numpy as np

LOADS = (475, 525, 575)  # creep load levels of the experiment (columns ending a, b, c)
SRJ_SECTION_COLS = ("Section1Strain", "Section2Strain", "Section3Strain", "Section4Strain", "Section5Strain")
SRJ_OFFSET = 5.25  # s, utils/config.py:52
SRJ_ROWS = 643  # the SRJ sample broke after this row (data_utils.py:729)


# ---------------------------------------------------------------- metrics (calc_utils.py:35-105)
def nearest_indices(query_x: np.ndarray, ref_x: np.ndarray) -> np.ndarray:
    """Index into ref_x of the closest entry to each query_x (first one on ties)."""
    query_x = np.asarray(query_x, dtype=float)
    ref_x = np.asarray(ref_x, dtype=float)
    if ref_x.ndim != 1 or query_x.ndim != 1:
        raise ValueError("nearest_indices expects 1D arrays")
    if len(ref_x) == 0:
        raise ValueError("ref_x must be non-empty")
    return np.array([int(np.argmin(np.abs(ref_x - x))) for x in query_x], dtype=int)


def mean_abs_error_aligned(*, sim_x, sim_y, exp_x, exp_y) -> float:
    """Mean of |exp - sim| / max(exp), sim taken at the nearest sim_x of each exp_x."""
    if len(exp_x) == 0 or len(sim_x) == 0:
        return np.inf
    y = np.asarray(sim_y)[nearest_indices(exp_x, sim_x)]
    return float((np.abs(exp_y - y) / np.max(exp_y)).mean())


def mean_sq_error_aligned(*, sim_x, sim_y, exp_x, exp_y) -> float:
    """Mean of ((exp - sim) / max(exp))^2, sim taken at the nearest sim_x of each exp_x."""
    if len(exp_x) == 0 or len(sim_x) == 0:
        return np.inf
    y = np.asarray(sim_y)[nearest_indices(exp_x, sim_x)]
    r = (exp_y - y) / np.max(exp_y)
    return float((r ** 2).mean())


def mean_rel_err_aligned(*, sim_x, sim_y, exp_x, exp_y, eps: float = 1e-12) -> float:
    """Mean of |sim - exp| / max(|sim|, |exp|).  The reference passes its eps
    array as the third positional argument of np.maximum, which numpy takes as
    the output buffer, so no eps floor applies; this keeps that behaviour (0/0
    where both values are zero gives nan, as there)."""
    if len(exp_x) == 0 or len(sim_x) == 0:
        return np.inf
    y = np.asarray(sim_y)[nearest_indices(exp_x, sim_x)]
    a = np.abs(y - exp_y)
    b = np.maximum(np.abs(y), np.abs(exp_y))
    return float(np.mean(a / b))


METRICS = {"MAE": mean_abs_error_aligned, "MSE": mean_sq_error_aligned, "MRE": mean_rel_err_aligned}


# ---------------------------------------------------------------- experimental curves
@dataclasses.dataclass
class CreepTarget:
    """Mean plastic strain history of one creep load (time in s, first sample dropped)."""
    load: int
    time: np.ndarray
    mean_plastic_strain: np.ndarray


@dataclasses.dataclass
class SrjTarget:
    """Strain-rate-jump test: mean true stress and true strain over the sections."""
    time: np.ndarray
    mean_stress: np.ndarray
    mean_strain: np.ndarray


def load_creep_target(csv_path, load: int) -> CreepTarget:
    """CreepData.load + get_load_vals (data_utils.py:516-640, 642-700) for one load level."""
    import pandas as pd

    df = pd.read_csv(csv_path, dtype=float)
    df.columns = df.columns.str.strip()
    time = df["Time"].values * 3600
    groups = {"a": [], "b": [], "c": []}
    for col in df.columns.values:
        if col != "Time" and col[-1:] in groups:
            groups[col[-1]].append(df[col].values)
    stacked = {k: np.vstack(v).T for k, v in groups.items()}
    bad = np.all(np.isnan(stacked["a"]), axis=1)  # the same row for all loads
    key = {475: "a", 525: "b", 575: "c"}[int(load)]
    s = stacked[key][~bad, :]
    time = time[~bad]
    plastic = s[1:] - s[1]
    return CreepTarget(int(load), time[1:].copy(), np.nanmean(plastic, axis=1))


def load_srj_target(csv_path) -> SrjTarget:
    """SrjData.load (data_utils.py:723-770)."""
    import pandas as pd

    df = pd.read_csv(csv_path, dtype=float).iloc[:SRJ_ROWS]
    df.columns = df.columns.str.strip()
    stress = df["Stress(MPa)"].values
    st = np.vstack([stress * (1.0 + df[c].values) for c in SRJ_SECTION_COLS])
    se = np.vstack([np.log1p(df[c].values) for c in SRJ_SECTION_COLS])
    return SrjTarget(df["Time"].values, np.mean(st, axis=0), np.mean(se, axis=0))


# ---------------------------------------------------------------- objectives
def _overlap_error(err_func, sim_x, sim_y, exp_x, exp_y) -> float:
    if len(sim_x) == 0 or len(exp_x) == 0:
        return float("inf")
    lo = max(np.min(sim_x), np.min(exp_x))
    hi = min(np.max(sim_x), np.max(exp_x))
    e_ok = (exp_x >= lo) & (exp_x <= hi)
    s_ok = (sim_x >= lo) & (sim_x <= hi)
    return err_func(sim_x=sim_x[s_ok], sim_y=sim_y[s_ok], exp_x=exp_x[e_ok], exp_y=exp_y[e_ok])


def creep_objective(results, target: CreepTarget, metric: str = "MAE") -> float:
    """_creep_objective (calibrate.py:824-864): epav33(sim_time) vs the mean plastic strain."""
    if metric not in METRICS:
        raise ValueError(f"Unknown metric: {metric}")
    return _overlap_error(METRICS[metric], np.asarray(results["sim_time"], float), np.asarray(results["epav33"], float),
                          target.time, target.mean_plastic_strain)


def srj_objective(results, target: SrjTarget, metric: str = "MAE", align: str = "strain") -> float:
    """_srj_objective (calibrate.py:755-821): sav33 vs the mean true stress, aligned on strain or time."""
    if metric not in METRICS:
        raise ValueError(f"Unknown metric: {metric}")
    et = target.time - SRJ_OFFSET
    st = np.asarray(results["sim_time"], float) - SRJ_OFFSET
    em, sm = et > 0, st > 0
    exp_y = target.mean_stress[em]
    sim_y = np.asarray(results["sav33"], float)[sm]
    if align == "strain":
        exp_x, sim_x = target.mean_strain[em], np.asarray(results["eav33"], float)[sm]
    elif align == "time":
        exp_x, sim_x = et[em], st[sm]
    else:
        raise ValueError(f"Unknown srj_align: {align}")
    return _overlap_error(METRICS[metric], sim_x, sim_y, exp_x, exp_y)


def read_results(out_dir) -> dict:
    """The results.csv columns the objectives use, as float arrays, cut before the first
    diverged increment (non-finite eav33, sav33 or epav33), as SimResults.load does
    (data_utils.py:261-296)."""
    import pandas as pd

    df = pd.read_csv(Path(out_dir) / "results.csv")
    df.columns = df.columns.str.strip()
    out = {c: df[c].to_numpy(dtype=float) for c in ("iter", "sim_time", "epav33", "sav33", "eav33")}
    ok = np.isfinite(out["eav33"]) & np.isfinite(out["sav33"]) & np.isfinite(out["epav33"])
    bad = np.where(~ok)[0]
    if len(bad) > 0:
        out = {c: a[: bad[0]] for c, a in out.items()}
    return out


# ---------------------------------------------------------------- the batch
@dataclasses.dataclass
class Job:
    """One solve of a calibration evaluation.

    fft_in/out_dir: the deck and where its files go; target: a CreepTarget or
    SrjTarget to score against (None: no score, only the solve)."""
    fft_in: Path
    out_dir: Path
    target: object = None
    metric: str = "MAE"
    srj_align: str = "strain"


def evaluate_batch(server, jobs, w_iters: float = 0.0, mix: int = 1, modal: int = 0, precision: int = 0) -> list[dict]:
    """Submit every job to ``server`` at once, wait for all, and score each.

    Returns per job {"loss", "base", "avg_iters", "status", "error", "latency_s"}.
    A failed solve gets loss = inf (the reference's caller turns a failed
    solver into its worst loss)."""
    tickets = [server.submit(j.fft_in, j.out_dir, mix=mix, modal=modal, precision=precision, csv_only=True) for j in jobs]
    out = []
    for j, t in zip(jobs, tickets):
        st = server.wait(t)
        rec = {"status": st["status"], "error": st["error"], "latency_s": st["latency_s"], "loss": float("inf"),
               "base": float("inf"), "avg_iters": float("nan")}
        if st["status"] == 0:
            res = read_results(j.out_dir)
            rec["avg_iters"] = float(np.mean(res["iter"]))
            if isinstance(j.target, CreepTarget):
                base = creep_objective(res, j.target, j.metric)
            elif isinstance(j.target, SrjTarget):
                base = srj_objective(res, j.target, j.metric, j.srj_align)
            else:
                base = 0.0
            rec["base"] = base
            rec["loss"] = base + w_iters * rec["avg_iters"]
        out.append(rec)
    return out


# ---------------------------------------------------------------- synthetic stand-ins for the experimental CSVs
def synthetic_creep_csv(path, seed: int = 0, hours: float = 200.0, rows: int = 81, samples: int = 3) -> Path:
    """Write a synthetic creep-curve CSV in the schema CreepData.load reads.

    Columns: Time (h), then ``synthetic<k><a|b|c>`` engineering strains of
    ``samples`` specimens per load (a: 475, b: 525, c: 575 MPa): elastic
    step + primary (power of time) + secondary (linear) creep, rate rising with
    the load, with 2 % seeded specimen scatter.  A first all-NaN row mimics a
    blank line of a spreadsheet export (the loader drops it)."""
    import pandas as pd

    rng = np.random.default_rng(seed)
    t = np.linspace(0.0, hours, rows)
    cols = {"Time": np.concatenate([[np.nan], t])}
    for key, load in zip("abc", LOADS):
        r = (load / 525.0) ** 6
        for k in range(samples):
            f = 1.0 + 0.02 * rng.standard_normal()
            e = load / 2.0e5 + f * r * (2.0e-3 * (t / hours) ** 0.4 + 4.0e-3 * t / hours)
            cols[f"synthetic{k + 1}{key}"] = np.concatenate([[np.nan], e])
    path = Path(path)
    pd.DataFrame(cols).to_csv(path, index=False, float_format="%.9g")
    return path


def synthetic_srj_csv(path, seed: int = 0, rows: int = 700) -> Path:
    """Write a synthetic strain-rate-jump CSV in the schema SrjData.load reads.

    Columns: Time (s), Stress(MPa), and five section engineering strains
    ``Section<k>Strain``; the strain rate jumps 1e-4 -> 1e-3 -> 1e-4 /s and the
    stress follows a Voce curve with a rate-sensitivity term.  Rows beyond 643
    are written on purpose (the loader truncates there)."""
    import pandas as pd

    rng = np.random.default_rng(seed)
    t = np.arange(rows, dtype=float)
    rate = np.where((t > 250) & (t <= 450), 1e-3, 1e-4)
    e = np.concatenate([[0.0], np.cumsum(rate[1:] * np.diff(t))])
    stress = 250.0 + 200.0 * (1.0 - np.exp(-e / 0.02)) + 15.0 * np.log10(rate / 1e-4)
    cols = {"Time": t, "Stress(MPa)": stress}
    for c in SRJ_SECTION_COLS:
        cols[c] = e * (1.0 + 0.03 * rng.standard_normal())
    path = Path(path)
    pd.DataFrame(cols).to_csv(path, index=False, float_format="%.9g")
    return path
