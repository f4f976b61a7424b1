"""Serving loop: continuous admission by slots and HBM budget; each result is
the same alone and in the mix.

Tolerance: requests solve to ||f - K u|| <= 1e-8 ||f||; run alone or among
others (different streams, different summation order of the atomics, FP32
V-cycle) the iterates may take a different path, so results agree to the
solve tolerance: compliance within 1e-7 relative, displacement within 1e-5,
sensitivities within 1e-5 (relative to their max).
"""
import numpy as np
import pytest

from tosp import problems as P
from tosp import workloads as W

pytestmark = pytest.mark.gpu


def _reqs():
    pool = W.FieldPool(seed=3)
    out = []
    for nx, n, bc in ((16, 2, "cantilever"), (16, 1, "bridge"), (32, 1, "torsion"), (16, 2, "bridge"),
                      (32, 2, "cantilever")):
        pb = W.serving_problem(nx, bc)
        x = pool.field(nx, n, 0, 0.5)
        out.append((pb, n, x, W.serving_levels(nx)))
    return out


def _submit(tosp, srv, pb, n, x, ng, precision):
    mg = tosp.default_mg(ngrids=ng, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=1000, flexible=1)
    return srv.submit(pb, x, mg=mg, precision=precision, mr_n=n, p=3.0, emin=1e-9, rmin=1.0 if n > 1 else 1.5)


@pytest.mark.parametrize("precision", [0, 1])
def test_same_result_alone_and_in_the_mix(tosp_mod, precision):
    reqs = _reqs()
    alone = []
    srv = tosp_mod.Server(max_slots=1, hbm_budget_bytes=8 << 30)
    for pb, n, x, ng in reqs:
        rid = _submit(tosp_mod, srv, pb, n, x, ng, precision)
        srv.wait(rid)
        alone.append(srv.result(rid))
    srv.close()
    srv = tosp_mod.Server(max_slots=4, hbm_budget_bytes=8 << 30)
    ids = [_submit(tosp_mod, srv, pb, n, x, ng, precision) for pb, n, x, ng in reqs * 2]
    mixed = []
    for rid in ids:
        srv.wait(rid)
        mixed.append(srv.result(rid))
    srv.close()
    for k, (pb, n, x, ng) in enumerate(reqs):
        ua, ga, sa = alone[k]
        for um, gm, sm in (mixed[k], mixed[k + len(reqs)]):
            assert sa["status"] == 0 and sm["status"] == 0
            assert sa["relres"] <= 1e-8 and sm["relres"] <= 1e-8
            Fa, Fm = pb.f @ ua, pb.f @ um
            assert abs(Fa - Fm) <= 1e-7 * abs(Fa)
            assert np.linalg.norm(ua - um) <= 1e-5 * np.linalg.norm(ua)
            assert np.abs(ga - gm).max() <= 1e-5 * np.abs(ga).max()


def test_matches_single_handle_solver(tosp_mod):
    pb, n, x, ng = _reqs()[0]
    srv = tosp_mod.Server(max_slots=2, hbm_budget_bytes=4 << 30)
    rid = _submit(tosp_mod, srv, pb, n, x, ng, 0)
    srv.wait(rid)
    u, g, st = srv.result(rid)
    srv.close()
    s = tosp_mod.Solver(pb, tosp_mod.default_mg(ngrids=ng, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=1000,
                                                flexible=1), precision=0, mr_n=n, p=3.0, emin=1e-9, rmin=1.0)
    s.SetupGMG(x)
    u2, it2, _, _ = s.SolveMG(np.zeros(pb.f.size), pb.f)
    assert abs(st["it"] - it2) <= 1
    assert abs(pb.f @ u - pb.f @ u2) <= 1e-9 * abs(pb.f @ u2)


def test_admission_by_budget_and_cancel(tosp_mod):
    reqs = _reqs()
    pb, n, x, ng = reqs[4]                       # the largest request
    srv = tosp_mod.Server(max_slots=4, hbm_budget_bytes=100 << 20)
    ids = [_submit(tosp_mod, srv, pb, n, x, ng, 1) for _ in range(3)]
    info = srv.info()
    assert info["used_bytes"] <= 100 << 20
    cancelled = srv.cancel(ids[-1])              # queued (or already running -> -6)
    assert cancelled in (0, -6)
    for rid in ids[:-1]:
        srv.wait(rid)
        u, g, st = srv.result(rid)
        assert st["status"] == 0
    srv.close()
    with pytest.raises(tosp_mod.TospError):      # can never fit
        srv2 = tosp_mod.Server(max_slots=1, hbm_budget_bytes=1 << 20)
        _submit(tosp_mod, srv2, pb, n, x, ng, 1)


@pytest.mark.parametrize("small", [0, 65536])
@pytest.mark.parametrize("precision,cgp", [(0, 0), (1, 0), (1, 1)])
def test_batched_requests_match_standalone_solves(tosp_mod, precision, cgp, small):
    """Requests of one shape in flight together run as one batch, one CG
    iteration per tick; with mg.small_cycle_max > 0 every visit to the small
    levels is one persistent launch for all of them; with mg.cg_product = 1
    the runner replaces each member's residual after its tick.  Supports,
    loads and densities differ between members; each result equals the
    standalone solve of its request (same parameters) to the solve
    tolerance."""
    pool = W.FieldPool(seed=5)
    items = []
    for k, bc in enumerate(("cantilever", "bridge", "torsion", "cantilever", "bridge", "torsion")):
        pb = W.serving_problem(32, bc)
        items.append((pb, pool.field(32, 1, k % 3, 0.45 + 0.02 * k)))
    mg = tosp_mod.default_mg(ngrids=3, cycle=1, omega=0.5, tolMG=1e-8, maxiterMG=1000, flexible=1,
                             small_cycle_max=small, cg_product=cgp)
    srv = tosp_mod.Server(max_slots=6, hbm_budget_bytes=8 << 30)
    srv.prepare(items[0][0], count=6, mg=mg, precision=precision)
    ids = [srv.submit(pb, x, mg=mg, precision=precision, mr_n=1, p=3.0, emin=1e-9, rmin=1.5) for pb, x in items]
    res = []
    for rid in ids:
        srv.wait(rid)
        res.append(srv.result(rid))
    cnt = srv.counters()
    srv.close()
    assert cnt["max_batch"] >= 2, cnt
    for (pb, x), (u, g, st) in zip(items, res):
        s = tosp_mod.Solver(pb, mg, precision=precision, mr_n=1, p=3.0, emin=1e-9, opfilter=1, rmin=1.5)
        s.SetupGMG(x)
        u0, it0, rr0, rc0 = s.SolveMG(np.zeros(pb.f.size), pb.f)
        uf = np.zeros(3 * pb.nnodes)
        uf[pb.freedofs] = u0
        g0 = s.Grad(uf)
        s.close()
        assert st["status"] == 0 and rc0 == 0 and st["relres"] <= 1e-8
        assert abs(pb.f @ u - pb.f @ u0) <= 1e-7 * abs(pb.f @ u0)
        assert np.linalg.norm(u - u0) <= 1e-5 * np.linalg.norm(u0)
        assert np.abs(g - g0).max() <= 1e-5 * np.abs(g0).max()
