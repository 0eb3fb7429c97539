"""Helpers that run the CUDA solve and the CPU oracle on the same deck and compare them."""
from __future__ import annotations

import numpy as np

RTOL = 1e-8  # FP64 plain path vs oracle: curves and fields
COND_RTOL = 1e-6  # diagnostic 1-norm condition estimates
WALL_COL = 4  # wall_time column of results.csv / diagnostics.csv
DIAG_COND_COLS = (35, 36, 37)
DIAG_INDEX_COLS = tuple(range(38, 44))


def run_both(fft_in, nmacro, mix=1, modal=0, nthreads=0):
    import oracle
    from creep_modeling_b200 import Solve

    g = Solve(fft_in, mix=mix, modal=modal)
    o = oracle.OracleSolve(fft_in, mix=mix, modal=modal, nthreads=nthreads)
    rg, ro, dg, do = [], [], [], []
    for _ in range(nmacro):
        a = g.advance(1)
        b = o.advance(1)
        assert a == b
        if a == 0:
            break
        r1, d1 = g.rows()
        r2, d2 = o.rows()
        rg.append(r1); ro.append(r2); dg.append(d1); do.append(d2)
    return g, o, np.array(rg), np.array(ro), np.array(dg), np.array(do)


# results.csv tensor groups (eav, sav, epav, eelav, vgrad, edotp): each component is
# compared relative to the magnitude of its tensor, so components that the
# boundary conditions pin to zero (pure round-off) are judged on the tensor scale.
RESULT_GROUPS = [list(range(7 + 6 * g, 13 + 6 * g)) for g in range(6)]


def rel_err_cols(a, b, skip=(), groups=()):
    """Per-column max |a-b| / scale over the run; scale = column max, or the group max for grouped columns."""
    gscale = {}
    for grp in groups:
        s = float(np.max(np.abs(b[:, grp])))
        for c in grp:
            gscale[c] = s
    out = {}
    for c in range(b.shape[1]):
        if c in skip:
            continue
        scale = gscale.get(c, np.max(np.abs(b[:, c])))
        if scale == 0.0:
            out[c] = float(np.max(np.abs(a[:, c])))
        else:
            out[c] = float(np.max(np.abs(a[:, c] - b[:, c])) / scale)
    return out


def assert_rows_match(rg, ro, dg, do, rtol=RTOL):
    assert rg.shape == ro.shape and rg.shape[0] > 0
    np.testing.assert_array_equal(rg[:, 0], ro[:, 0], err_msg="equilibrium iteration counts differ")
    er = rel_err_cols(rg, ro, skip=(WALL_COL,), groups=RESULT_GROUPS)
    bad = {c: e for c, e in er.items() if e > rtol}
    assert not bad, f"results.csv columns beyond {rtol}: {bad}"
    ed = rel_err_cols(dg, do, skip=(WALL_COL,) + DIAG_COND_COLS + DIAG_INDEX_COLS)
    bad = {c: e for c, e in ed.items() if e > 1e-6}
    assert not bad, f"diagnostics.csv columns beyond 1e-6: {bad}"
    ec = rel_err_cols(dg[:, list(DIAG_COND_COLS)], do[:, list(DIAG_COND_COLS)])
    assert max(ec.values()) <= COND_RTOL, f"condition estimates differ: {ec}"


def field_rel_err(g, o, name):
    a = g.field(name)
    b = o.field(name)
    assert a.shape == b.shape, (name, a.shape, b.shape)
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))
