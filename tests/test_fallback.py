"""Host logic of tosp.FallbackSolver (mixed-precision solves finished in FP64
when they stall), on a fake solve handle: no GPU needed."""
import numpy as np
import pytest

import tosp


class FakeHandle:
    """Stands in for tosp.Solver: the mixed handle follows a script of
    outcomes ('ok', 'stall', 'breakdown', 'oom'); the FP64 one converges."""

    made = []
    script = []

    def __init__(self, pb, mg, precision, **kw):
        self.precision, self.mg, self.kw = precision, mg, kw
        self.setups, self.solves = [], []
        FakeHandle.made.append(self)

    def SetupGMG(self, x):
        self.setups.append(np.array(x))

    def SolveMG(self, x, f):
        self.solves.append(np.array(x))
        if self.precision == tosp.PREC_MIXED:
            mode = FakeHandle.script.pop(0)
            if mode == "breakdown":
                raise tosp.TospError(tosp.TOSP_ERR_BREAKDOWN, "breakdown")
            if mode == "oom":
                raise tosp.TospError(-3, "out of memory")
            return np.asarray(x) + 1.0, 10, 1e-9 if mode == "ok" else 1e-5, 0 if mode == "ok" else 1
        return np.asarray(x) + 2.0, 5, 1e-9, 0

    def Grad(self, u, return_unfiltered=False):
        return ("grad", self.precision)

    def ApplyFilter(self, x, trans=False):
        return np.asarray(x) * 2.0

    def Compliance(self, f, u):
        return float(np.dot(f, u))

    def close(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    FakeHandle.made = []
    FakeHandle.script = []
    monkeypatch.setattr(tosp, "Solver", FakeHandle)
    return FakeHandle


def make(maxstall=100, sticky=1):
    mg = tosp.default_mg(ngrids=3, cycle=1, omega=0.5, tolMG=1e-8, maxiterMG=500)
    return tosp.FallbackSolver(object(), mg, mr_n=2, maxstall=maxstall, sticky=sticky)


def test_converged_mixed_solve_needs_no_fp64_handle(fake):
    fake.script = ["ok"]
    fs = make()
    mixed = fake.made[0]
    assert mixed.precision == tosp.PREC_MIXED and mixed.mg.maxstall == 100 and mixed.mg.flexible == 1
    fs.SetupGMG(np.full(4, 0.5))
    u, it, rr, rc = fs.SolveMG(np.zeros(3), np.ones(3))
    assert rc == 0 and it == 10 and np.all(u == 1.0)
    assert fs.fp64 is None and fs.fallbacks == 0 and len(fake.made) == 1
    assert fs.Grad(np.zeros(3)) == ("grad", tosp.PREC_MIXED)


def test_stalled_solve_is_finished_in_fp64_from_the_mixed_iterate(fake):
    fake.script = ["stall"]
    fs = make()
    x = np.linspace(0.1, 0.9, 4)
    fs.SetupGMG(x)
    u, it, rr, rc = fs.SolveMG(np.zeros(3), np.ones(3))
    f64 = fs.fp64
    assert f64 is not None and f64.precision == tosp.PREC_FP64
    assert f64.mg.maxstall == 0 and f64.mg.flexible == 0 and f64.mg.cycle == 1
    assert np.array_equal(f64.setups[-1], x)            # set up with the current densities
    assert np.all(f64.solves[-1] == 1.0)                # started from the mixed iterate
    assert rc == 0 and it == 15 and np.all(u == 3.0)    # iterations of both solves
    assert fs.fallbacks == 1 and fs.use_fp64
    # sticky: the next design is set up and solved in FP64 only
    mixed = fake.made[0]
    n_mixed_setups = len(mixed.setups)
    fs.SetupGMG(x * 0.5)
    u2, it2, _, rc2 = fs.SolveMG(u, np.ones(3))
    assert len(mixed.setups) == n_mixed_setups and len(mixed.solves) == 1
    assert rc2 == 0 and it2 == 5 and np.array_equal(f64.setups[-1], x * 0.5)
    assert fs.Grad(np.zeros(3)) == ("grad", tosp.PREC_FP64)


def test_breakdown_falls_back_from_the_starting_iterate(fake):
    fake.script = ["breakdown"]
    fs = make()
    fs.SetupGMG(np.full(4, 0.5))
    x0 = np.array([0.25, 0.5, 0.75])
    u, it, rr, rc = fs.SolveMG(x0, np.ones(3))
    assert rc == 0 and it == 5 and np.allclose(u, x0 + 2.0) and fs.fallbacks == 1


def test_other_errors_are_not_hidden(fake):
    fake.script = ["oom"]
    fs = make()
    fs.SetupGMG(np.full(4, 0.5))
    with pytest.raises(tosp.TospError) as e:
        fs.SolveMG(np.zeros(3), np.ones(3))
    assert e.value.code == -3 and fs.fp64 is None


def test_sticky_two_retries_mixed_once_more(fake):
    fake.script = ["stall", "ok"]
    fs = make(sticky=2)
    fs.SetupGMG(np.full(4, 0.5))
    fs.SolveMG(np.zeros(3), np.ones(3))
    assert fs.fallbacks == 1 and not fs.use_fp64
    fs.SetupGMG(np.full(4, 0.4))
    u, it, _, rc = fs.SolveMG(np.zeros(3), np.ones(3))
    assert rc == 0 and it == 10 and fs.fallbacks == 1      # the mixed path answered
