"""Host SLP driver (restatement of I/StrSLP.m): LP subproblem solvers and a
short optimisation with the oracle solve path (CPU)."""
import numpy as np
import pytest

from oracle_solver import OracleSolver
from tosp import problems as P
from tosp import slp


@pytest.mark.parametrize("seed", range(5))
def test_knapsack_lp_matches_dual_simplex(seed):
    rng = np.random.default_rng(seed)
    n = 300
    g = rng.standard_normal(n)
    a = rng.uniform(0.5, 2.0, n)
    lo = -rng.uniform(0, 0.1, n)
    hi = rng.uniform(0, 0.1, n)
    c = float(a @ np.where(g < 0, hi, lo)) * rng.uniform(-0.5, 0.5)
    s1, f1, l1, ok1 = slp.lp_knapsack(g, a, c, lo, hi)
    s2, f2, l2, ok2, _ = slp.lp_highs(g, a, c, lo, hi)
    assert ok1 and ok2
    assert abs(f1 - f2) <= 1e-10 * max(1.0, abs(f2))
    assert abs(l1 - l2) <= 1e-8 * max(1.0, abs(l2))
    assert a @ s1 <= c + 1e-10 and np.all(s1 >= lo - 1e-15) and np.all(s1 <= hi + 1e-15)


def test_knapsack_slack_constraint_and_infeasible():
    g = np.array([1.0, -1.0, 2.0])
    a = np.ones(3)
    s, f, lam, ok = slp.lp_knapsack(g, a, 10.0, -np.ones(3), np.ones(3))
    assert ok and lam == 0.0 and np.array_equal(s, [-1.0, 1.0, -1.0])
    s, f, lam, ok = slp.lp_knapsack(g, a, -5.0, -np.ones(3), np.ones(3))
    assert not ok


def test_grad_proj_rounds_to_volume():
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 1, 1000)
    g = rng.standard_normal(1000)
    velem = np.full(1000, 1.0)
    out = slp.grad_proj(x, g, slp.PrjParams(op=True), 400.0, velem)
    assert np.all((out >= 0) & (out <= 1))
    assert np.all(out[x <= 0.05] == 0.0)
    assert out[x >= 0.95].min() == 1.0


def test_slp_oracle_decreases_compliance():
    pb = P.cantilever(12, 6, 6)
    sol = OracleSolver(pb, ngrids=2, cycle=0, omega=0.6, rmin=1.5)
    res = slp.str_slp(sol, pb, 0.3, np.full(pb.nelem, 0.3), slp.SlpParams(maxiter=5))
    Fs = [h["F"] for h in res.history if h["it"] > 0]
    assert res.iters == 5
    assert res.F < res.history[0]["F"] + 1e-12 or res.F < Fs[0]
    assert abs(np.full(pb.nelem, 1.0) @ res.xstar / pb.nelem - 0.3) < 0.02


def _knapsack_by_sort(g, a, c, lo, hi, rtol=1e-9):
    """Sort-based statement of the same LP (all candidates sorted by cost per
    unit of constraint), used to check the selection-based solver."""
    s = np.where(g < 0, hi, lo).astype(np.float64)
    excess = a @ s - c
    if excess <= 0:
        return s
    cand = np.nonzero((g < 0) & (hi > lo))[0]
    ratio = -g[cand] / a[cand]
    srt = np.argsort(ratio, kind="stable")
    order, ratio = cand[srt], ratio[srt]
    red = a[order] * (hi[order] - lo[order])
    newgrp = np.ones(order.size, dtype=bool)
    newgrp[1:] = ratio[1:] - ratio[:-1] > rtol * np.abs(ratio[1:])
    gid = np.cumsum(newgrp) - 1
    gred = np.bincount(gid, weights=red)
    gcum = np.cumsum(gred)
    k = int(np.searchsorted(gcum, excess))
    s[order[gid < k]] = lo[order[gid < k]]
    frac = (excess - (gcum[k - 1] if k > 0 else 0.0)) / gred[k]
    grp = order[gid == k]
    s[grp] = hi[grp] - frac * (hi[grp] - lo[grp])
    return s


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_knapsack_selection_matches_sort(seed):
    """The selection-based knapsack equals the full-sort statement, with
    exact ties (mirrored entries) and near ties inside the 1e-9 group rule."""
    rng = np.random.default_rng(seed)
    n = 20000
    g = rng.standard_normal(n)
    g[n // 2:] = g[:n // 2]                                  # exact ties
    g[:50] = g[50:100] * (1 + 1e-12)                         # near ties
    a = rng.uniform(0.5, 2.0, n)
    a[n // 2:] = a[:n // 2]
    lo = np.zeros(n)
    hi = rng.uniform(0.2, 1.0, n)
    hi[n // 2:] = hi[:n // 2]
    for c in (0.05 * (a @ hi), 0.3 * (a @ hi), 0.9 * (a @ hi)):
        s1, f1, lam, ok = slp.lp_knapsack(g, a, c, lo, hi)
        s2 = _knapsack_by_sort(g, a, c, lo, hi)
        assert ok
        assert np.abs(s1 - s2).max() <= 1e-9
        assert a @ s1 <= c * (1 + 1e-12)


def test_heaviside_projection_keeps_volume():
    """HeavisideProj (I/HeavisideProj.m): eta is chosen so that the projected
    volume equals the requested one; the map is monotone, fixes 0 and 1 and
    sharpens towards 0/1 as beta grows."""
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 1.0, 5000)
    velem = np.full(x.size, 1.0 / x.size)
    prj = slp.PrjParams(op=True)
    vol = float(velem @ x)
    prev_gray = np.inf
    for _ in range(6):
        xs, prj = slp.heaviside_proj(x, prj, velem, vol, vol, True)
        assert abs(velem @ xs - vol) <= 1e-10
        o = np.argsort(x)
        assert np.all(np.diff(xs[o]) >= -1e-15)
        gray = float(np.mean((xs > 0.05) & (xs < 0.95)))
        assert gray <= prev_gray + 1e-12
        prev_gray = gray
    c = np.tanh(prj.beta * prj.eta)
    d = 1.0 / (c + np.tanh(prj.beta * (1.0 - prj.eta)))
    assert abs((c + np.tanh(prj.beta * (0.0 - prj.eta))) * d) <= 1e-15
    assert abs((c + np.tanh(prj.beta * (1.0 - prj.eta))) * d - 1.0) <= 1e-15
    assert prj.beta == 64.0


def test_two_oracle_paths_give_identical_thresholded_designs():
    """The tie rule of GradProj: the same SLP loop on the NumPy/SciPy oracle
    and on its C/OpenMP restatement (solutions equal to rounding) thresholds
    to identical 0/1 designs."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    pytest.importorskip("oracle.cpu_assembled")
    from oracle_solver import AssembledOracleSolver, OracleSolver
    from tosp import problems as P
    pb = P.cantilever(16, 8, 8)
    x0 = np.full(pb.nelem, 0.3)
    params = slp.SlpParams(maxiter=6, lp="knapsack")
    r1 = slp.str_slp(AssembledOracleSolver(pb, ngrids=3, omega=0.6, rmin=1.5, maxiter=5000, nthreads=4), pb, 0.3,
                     x0, params, prj=slp.PrjParams(op=True))
    r2 = slp.str_slp(OracleSolver(pb, ngrids=3, cycle=0, omega=0.6, rmin=1.5, maxiter=5000), pb, 0.3, x0, params,
                     prj=slp.PrjParams(op=True))
    assert [h["it"] for h in r1.history] == [h["it"] for h in r2.history]
    assert abs(r1.F - r2.F) <= 1e-10 * abs(r2.F)
    assert np.array_equal(r1.xstar, r2.xstar) and 0 < r1.xstar.sum() < r1.xstar.size
