"""Calibration client on the GPU: a batch of candidate x load creep solves on one server,
scored with the reference's creep objective."""
import dataclasses

import pytest

from creep_modeling_b200 import calibration as cal, decks
from creep_modeling_b200.serve import Server

pytestmark = pytest.mark.gpu

LOADS = (140.0, 150.0, 160.0)


def _jobs(root, target=None):
    jobs = []
    for c, tau0 in enumerate((90.0, 110.0)):
        for load in LOADS:
            case = decks.case_c1(nsteps=4)
            case.n = 12
            case.ngrains = 16
            case.material = dataclasses.replace(case.material, tau0f=tau0, tau0b=tau0)
            case.processes[0].stress33 = load
            d = root / f"cand{c}" / f"creep{int(load)}"
            jobs.append(cal.Job(decks.write_case(case, d), d / "out", target))
    return jobs


def test_batch_scores_every_candidate_and_load(tmp_path):
    with Server(0, 8) as srv:
        first = cal.evaluate_batch(srv, _jobs(tmp_path / "a"))
        assert [r["status"] for r in first] == [0] * 6
        # the candidate-0 150 MPa curve as the "experiment": that solve scores 0, the others do not
        ref = cal.read_results(tmp_path / "a" / "cand0" / "creep150" / "out")
        assert (ref["epav33"] > 0).all()
        tgt = cal.CreepTarget(150, ref["sim_time"], ref["epav33"])
        res = cal.evaluate_batch(srv, _jobs(tmp_path / "b", tgt), w_iters=1e-3)
    assert [r["status"] for r in res] == [0] * 6
    # solves are independent of what else was in flight: the second batch repeats the first bit for bit
    strip = lambda rows: [",".join(r.split(",")[:4] + r.split(",")[5:]) for r in rows]  # wall_time differs
    for c in range(2):
        for load in LOADS:
            a = (tmp_path / "a" / f"cand{c}" / f"creep{int(load)}" / "out" / "results.csv").read_text().splitlines()
            b = (tmp_path / "b" / f"cand{c}" / f"creep{int(load)}" / "out" / "results.csv").read_text().splitlines()
            assert strip(a) == strip(b), (c, load)
    base = [r["base"] for r in res]
    assert base[1] == 0.0
    assert all(b > 0.0 for i, b in enumerate(base) if i != 1)
    # plastic strain rate ~ stress^n with n = 10: the 160 MPa curve departs further from the
    # 150 MPa one than the 140 MPa curve does
    assert base[0] < base[2]
    for r in res:
        assert r["loss"] == pytest.approx(r["base"] + 1e-3 * r["avg_iters"], rel=1e-12)


def test_batch_scores_match_the_oracle(tmp_path, oracle_lib):
    """Every candidate x load solve of the served batch against the CPU FP64 oracle on the same
    deck: the results.csv rows within the parity bar (identical iteration counts, 1e-8 per
    column) and the creep objective of each solve within 1e-8 of the oracle's."""
    import numpy as np

    from creep_modeling_b200.solver import load_results
    from tests import parity

    with Server(0, 8) as srv:
        ref_jobs = _jobs(tmp_path / "a")
        assert [r["status"] for r in cal.evaluate_batch(srv, ref_jobs)] == [0] * 6
        ref = cal.read_results(tmp_path / "a" / "cand0" / "creep150" / "out")
        tgt = cal.CreepTarget(150, ref["sim_time"], ref["epav33"])
        jobs = _jobs(tmp_path / "b", tgt)
        res = cal.evaluate_batch(srv, jobs)
    for job, r in zip(jobs, res):
        odir = job.out_dir.parent / "oracle"
        o = oracle_lib.OracleSolve(job.fft_in, out_dir=str(odir), mix=1, modal=0, write_files=True)
        o.run()
        o.close()
        rg, ro = load_results(job.out_dir / "results.csv"), load_results(odir / "results.csv")
        dg = np.loadtxt(job.out_dir / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
        do = np.loadtxt(odir / "diagnostics.csv", delimiter=",", skiprows=1, ndmin=2)
        parity.assert_rows_match(rg, ro, dg, do)
        base_o = cal.creep_objective(cal.read_results(odir), tgt)
        # the objective is a mean absolute difference of plastic-strain curves: compare it on the curves' scale
        scale = float(np.max(np.abs(ref["epav33"])))
        assert abs(r["base"] - base_o) <= 1e-8 * scale, (r["base"], base_o)
