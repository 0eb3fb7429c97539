"""Calibration client: loaders, metrics and objectives pinned to the reference's own
Python (fixtures made by tests/golden/make_calibration_golden.py), and the batch
logic against a fake server (no GPU)."""
from pathlib import Path

import numpy as np
import pytest

from creep_modeling_b200 import calibration as cal

G = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def golden():
    return np.load(G / "calib_golden.npz")


@pytest.mark.parametrize("load", cal.LOADS)
def test_creep_loader_matches_reference(golden, load):
    t = cal.load_creep_target(G / "calib_creep.csv", load)
    np.testing.assert_array_equal(t.time, golden[f"creep{load}_time"])
    np.testing.assert_array_equal(t.mean_plastic_strain, golden[f"creep{load}_mps"])


def test_srj_loader_matches_reference(golden):
    t = cal.load_srj_target(G / "calib_srj.csv")
    assert len(t.time) == cal.SRJ_ROWS
    np.testing.assert_array_equal(t.time, golden["srj_time"])
    np.testing.assert_array_equal(t.mean_stress, golden["srj_stress"])
    np.testing.assert_array_equal(t.mean_strain, golden["srj_strain"])


@pytest.mark.parametrize("k", range(4))
def test_metrics_match_reference(golden, k):
    kw = dict(sim_x=golden[f"m{k}_sim_x"], sim_y=golden[f"m{k}_sim_y"], exp_x=golden[f"m{k}_exp_x"], exp_y=golden[f"m{k}_exp_y"])
    np.testing.assert_array_equal(cal.nearest_indices(kw["exp_x"], kw["sim_x"]), golden[f"m{k}_idx"])
    assert cal.mean_abs_error_aligned(**kw) == float(golden[f"m{k}_mae"])
    assert cal.mean_sq_error_aligned(**kw) == float(golden[f"m{k}_mse"])
    assert cal.mean_rel_err_aligned(**kw) == float(golden[f"m{k}_mre"])


def test_metrics_empty_inputs():
    e = np.zeros(0)
    assert cal.mean_abs_error_aligned(sim_x=e, sim_y=e, exp_x=np.ones(2), exp_y=np.ones(2)) == np.inf
    with pytest.raises(ValueError):
        cal.nearest_indices(np.ones(2), e)


def _results(t, epav33, sav33=None, eav33=None, it=None):
    n = len(t)
    return {"sim_time": np.asarray(t, float), "epav33": np.asarray(epav33, float),
            "sav33": np.zeros(n) if sav33 is None else np.asarray(sav33, float),
            "eav33": np.zeros(n) if eav33 is None else np.asarray(eav33, float),
            "iter": np.full(n, 10.0) if it is None else np.asarray(it, float)}


def test_creep_objective_is_zero_on_the_target_and_respects_the_overlap():
    tgt = cal.load_creep_target(G / "calib_creep.csv", 525)
    r = _results(tgt.time, tgt.mean_plastic_strain)
    assert cal.creep_objective(r, tgt, "MAE") == 0.0
    assert cal.creep_objective(r, tgt, "MSE") == 0.0
    # a simulation covering only the first half of the test is scored on that half only
    h = len(tgt.time) // 2
    r2 = _results(tgt.time[:h], tgt.mean_plastic_strain[:h] * 1.1)
    exp_ok = tgt.time <= tgt.time[h - 1]
    want = np.mean(np.abs(tgt.mean_plastic_strain[exp_ok] * 0.1) / tgt.mean_plastic_strain[exp_ok].max())
    assert cal.creep_objective(r2, tgt, "MAE") == pytest.approx(want, rel=1e-12)
    with pytest.raises(ValueError):
        cal.creep_objective(r, tgt, "RMS")


def test_srj_objective_alignment_modes():
    tgt = cal.load_srj_target(G / "calib_srj.csv")
    r = _results(tgt.time, np.zeros(len(tgt.time)), sav33=tgt.mean_stress, eav33=tgt.mean_strain)
    assert cal.srj_objective(r, tgt, "MAE", "strain") == 0.0
    assert cal.srj_objective(r, tgt, "MAE", "time") == 0.0
    with pytest.raises(ValueError):
        cal.srj_objective(r, tgt, "MAE", "stress")


class _FakeServer:
    """Records submissions; 'solves' by writing a results.csv that follows the target."""

    def __init__(self, tgt, fail=()):
        self.tgt, self.fail, self.sub = tgt, set(fail), []

    def submit(self, fft_in, out_dir, mix=1, modal=0, precision=0, csv_only=False):
        self.sub.append((Path(fft_in), Path(out_dir), csv_only))
        return len(self.sub) - 1

    def wait(self, t):
        fft_in, out, _ = self.sub[t]
        if t in self.fail:
            return {"status": -5, "error": "did not converge", "latency_s": 0.1}
        out.mkdir(parents=True, exist_ok=True)
        scale = float(fft_in.name.split("_")[1])
        import pandas as pd

        pd.DataFrame({"iter": np.arange(len(self.tgt.time)) % 5 + 1, "sim_time": self.tgt.time,
                      "epav33": self.tgt.mean_plastic_strain * scale, "sav33": 0.0, "eav33": 0.0}).to_csv(out / "results.csv", index=False)
        return {"status": 0, "error": "", "latency_s": 0.1}


def test_evaluate_batch_submits_everything_before_waiting(tmp_path):
    tgt = cal.load_creep_target(G / "calib_creep.csv", 475)
    srv = _FakeServer(tgt, fail={2})
    jobs = [cal.Job(tmp_path / f"fft_{s}_.in", tmp_path / f"out{i}", tgt) for i, s in enumerate((1.0, 1.2, 0.9))]
    res = cal.evaluate_batch(srv, jobs, w_iters=0.01)
    assert len(srv.sub) == 3 and all(c for _, _, c in srv.sub)
    assert res[0]["base"] == pytest.approx(0.0, abs=1e-12)
    assert res[0]["avg_iters"] == pytest.approx(np.mean(np.arange(len(tgt.time)) % 5 + 1))
    assert res[0]["loss"] == pytest.approx(0.01 * res[0]["avg_iters"], rel=1e-9)
    assert res[1]["base"] > 0.0
    assert res[2]["status"] == -5 and res[2]["loss"] == np.inf


def test_read_results_stops_at_the_first_diverged_increment(tmp_path):
    import pandas as pd

    pd.DataFrame({"iter": [3, 4, 5, 6], "sim_time": [1.0, 2.0, 3.0, 4.0], "epav33": [1e-6, 2e-6, float("nan"), 4e-6],
                  "sav33": [100.0, 100.0, 100.0, 100.0], "eav33": [1e-3, 1e-3, 1e-3, 1e-3]}).to_csv(tmp_path / "results.csv",
                                                                                            index=False)
    r = cal.read_results(tmp_path)
    assert list(r["sim_time"]) == [1.0, 2.0] and list(r["iter"]) == [3.0, 4.0]
