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
