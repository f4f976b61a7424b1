"""Failure detection with faults injected on the host: bad densities, a zero
load, a stalling mixed-precision solve that the serving loop re-runs in FP64,
and requests that can never be admitted.  Nothing here faults, traps or hangs
the GPU: every failure is a status code read back by the host."""
import numpy as np
import pytest

from tosp import problems as P
from tosp import workloads as W

pytestmark = pytest.mark.gpu


def _solver(tosp, pb, n=1, prec=0, **kw):
    mg = dict(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=500)
    mg.update(kw)
    return tosp.Solver(pb, tosp.default_mg(**mg), precision=prec, mr_n=n, p=3.0, emin=1e-9, opfilter=1,
                       rmin=1.0 if n > 1 else 1.5)


@pytest.mark.parametrize("bad", [np.nan, -0.5])
def test_invalid_densities_stop_at_setup(tosp_mod, bad):
    """A NaN or negative density gives a non-positive coarsest pivot: SetupGMG
    reports TOSP_ERR_BREAKDOWN instead of producing a meaningless hierarchy."""
    pb = P.cantilever(8, 4, 4)
    x = np.full(pb.nelem, 0.5)
    x[:] = bad
    s = _solver(tosp_mod, pb)
    with pytest.raises(tosp_mod.TospError) as e:
        s.SetupGMG(x)
    assert e.value.code == -4                       # TOSP_ERR_BREAKDOWN


def test_zero_load_returns_the_start(tosp_mod):
    """With f = 0 the reference's loop condition is false from the start
    (I/SolveMG.m:30): the iterate is returned unchanged after no iteration."""
    pb = P.cantilever(8, 4, 4)
    s = _solver(tosp_mod, pb)
    s.SetupGMG(np.full(pb.nelem, 0.5))
    u, it, rr, rc = s.SolveMG(np.zeros(pb.f.size), np.zeros(pb.f.size))
    assert rc == 0 and it == 1
    assert not np.any(u)


def test_stalled_mixed_request_falls_back_to_fp64(tosp_mod):
    """A mixed-precision request whose residual does not halve within maxstall
    iterations is re-run in FP64 by the serving loop and still converges."""
    pb = W.serving_problem(16, "cantilever")
    x = W.FieldPool(seed=3).field(16, 2, 0, 0.5)
    srv = tosp_mod.Server(max_slots=1, hbm_budget_bytes=4 << 30)
    mg = tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=1000, flexible=1, maxstall=1)
    rid = srv.submit(pb, x, mg=mg, precision=1, mr_n=2, p=3.0, emin=1e-9, rmin=1.0)
    srv.wait(rid)
    u, g, st = srv.result(rid)
    srv.close()
    assert st["status"] == 0
    assert st["precision"] == 0          # finished in FP64
    assert st["relres"] <= 1e-8


def test_unadmittable_request_is_rejected(tosp_mod):
    """A request larger than the whole HBM budget is refused at submission."""
    pb = W.serving_problem(32, "bridge")
    x = W.FieldPool(seed=3).field(32, 2, 0, 0.5)
    srv = tosp_mod.Server(max_slots=2, hbm_budget_bytes=1 << 20)
    mg = tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=1000)
    with pytest.raises(tosp_mod.TospError) as e:
        srv.submit(pb, x, mg=mg, precision=1, mr_n=2, p=3.0, emin=1e-9, rmin=1.0)
    assert e.value.code == -3
    srv.close()


def test_fallback_solver_finishes_stalled_solves_in_fp64(tosp_mod):
    """FallbackSolver: a mixed solve that stalls (maxstall = 1 forces it) is
    finished in FP64 from its iterate, and the FP64 path then serves the next
    solve; the result matches a plain FP64 solve."""
    pb = P.cantilever(16, 8, 8)
    dens = np.random.default_rng(5).uniform(0.001, 1.0, pb.nelem * 8)
    mg = tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=500)
    fs = tosp_mod.FallbackSolver(pb, mg, mr_n=2, p=3.0, emin=1e-9, opfilter=1, rmin=1.0, maxstall=1)
    fs.SetupGMG(dens)
    u, it, rr, rc = fs.SolveMG(np.zeros(pb.f.size), pb.f)
    assert rc == 0 and rr <= 1e-8
    assert fs.fallbacks == 1 and fs.use_fp64
    ref = _solver(tosp_mod, pb, n=2, ngrids=3)
    ref.SetupGMG(dens)
    u64, _, _, _ = ref.SolveMG(np.zeros(pb.f.size), pb.f)
    assert abs(pb.f @ u - pb.f @ u64) <= 1e-6 * abs(pb.f @ u64)
    fs.SetupGMG(dens * 0.9 + 0.05)          # the next design goes straight to FP64
    u2, it2, rr2, rc2 = fs.SolveMG(u, pb.f)
    assert rc2 == 0 and rr2 <= 1e-8 and fs.fallbacks == 1
    uf = np.zeros(3 * pb.nnodes)
    uf[pb.freedofs] = u2
    ref.SetupGMG(dens * 0.9 + 0.05)
    go = ref.Grad(uf)
    assert np.abs(fs.Grad(uf) - go).max() <= 1e-12 * np.abs(go).max()
    fs.close()


def test_fallback_solver_keeps_converging_mixed_solves(tosp_mod):
    """Without a stall the mixed path answers and no FP64 handle is made."""
    pb = P.cantilever(16, 8, 8)
    dens = np.random.default_rng(6).uniform(0.001, 1.0, pb.nelem * 8)
    mg = tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=500)
    fs = tosp_mod.FallbackSolver(pb, mg, mr_n=2, p=3.0, emin=1e-9, opfilter=1, rmin=1.0, maxstall=100)
    fs.SetupGMG(dens)
    u, it, rr, rc = fs.SolveMG(np.zeros(pb.f.size), pb.f)
    assert rc == 0 and rr <= 1e-8
    assert fs.fallbacks == 0 and fs.fp64 is None
    fs.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_bounded_wait_runs_out_and_the_handle_recovers(tosp_mod, prec):
    """A bounded device wait that runs out: the persistent small-level cycle's
    grid barrier gets a short poll limit and one block skips its first
    arrival (tosp_inject_wait_fault), so the other blocks give up.  The cycle
    returns TOSP_ERR_TIMEOUT; the barrier state is reset, and the same handle
    then gives the same preconditioner output and solve as a handle that never
    saw the fault.  No kernel waits without bound, traps or faults."""
    import ctypes as C
    pb = P.cantilever(32, 16, 16)
    kw = dict(ngrids=4, cycle=0, omega=0.5, flexible=1 if prec else 0, maxiterMG=2000)
    s = _solver(tosp_mod, pb, n=1, prec=prec, small_cycle_max=16384, **kw)
    ref = _solver(tosp_mod, pb, n=1, prec=prec, small_cycle_max=16384, **kw)
    dens = np.random.default_rng(3).uniform(0.2, 1.0, pb.nelem)
    s.SetupGMG(dens)
    ref.SetupGMG(dens)
    nb = C.c_int32()
    assert tosp_mod._lib.tosp_small_cycle_blocks(s.h, C.byref(nb)) == 0
    assert nb.value >= 2, nb.value
    r = np.random.default_rng(4).standard_normal(pb.freedofs.size)
    assert tosp_mod._lib.tosp_inject_wait_fault(s.h, 4096, nb.value - 1) == 0
    with pytest.raises(tosp_mod.TospError) as e:
        s.MGCycle(r)
    assert e.value.code == -8                                 # TOSP_ERR_TIMEOUT
    assert "timed out" in str(e.value)
    tol = 1e-12 if prec == 0 else 5e-5
    assert rel_err(s.MGCycle(r), ref.MGCycle(r)) <= tol
    u1, it1, rr1, rc1 = s.SolveMG(np.zeros(pb.f.size), pb.f)
    u0, it0, rr0, rc0 = ref.SolveMG(np.zeros(pb.f.size), pb.f)
    assert rc1 == rc0 == 0 and rr1 <= 1e-8
    assert abs(pb.f @ u1 - pb.f @ u0) <= 1e-9 * abs(pb.f @ u0)


def rel_err(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_metrics_lines_and_nvtx_ranges(tmp_path):
    """With TOSP_METRICS set, every solve and every served request appends one
    JSON line (iterations, residual, times, status); the entry points' NVTX
    ranges cost nothing without a profiler.  Run in a child process, since the
    library reads the variable once."""
    import json
    import os
    import subprocess
    import sys
    log = tmp_path / "metrics.jsonl"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys; sys.path[:0] = [%r, %r]\n"
        "import numpy as np, tosp\n"
        "from tosp import problems as P\n"
        "pb = P.cantilever(16, 8, 8)\n"
        "s = tosp.Solver(pb, tosp.default_mg(ngrids=3, cycle=0, omega=0.6), mr_n=1)\n"
        "s.SetupGMG(np.full(pb.nelem, 0.5)); s.SolveMG(np.zeros(pb.f.size), pb.f)\n"
        "srv = tosp.Server(max_slots=2, hbm_budget_bytes=1 << 30)\n"
        "rid = srv.submit(pb, np.full(pb.nelem, 0.5), mg=tosp.default_mg(ngrids=3, cycle=0, omega=0.6))\n"
        "srv.wait(rid); srv.result(rid); srv.close()\n") % (root, os.path.join(root, "topopt-slp-3d_b200"))
    env = dict(os.environ, TOSP_METRICS=str(log))
    subprocess.run([sys.executable, "-c", code], check=True, env=env, timeout=300)
    lines = [json.loads(l) for l in log.read_text().splitlines()]
    events = [l["event"] for l in lines]
    assert "solve" in events and "request" in events
    solve = lines[events.index("solve")]
    assert solve["status"] == 0 and solve["relres"] <= 1e-8 and solve["it"] > 1
    req = lines[events.index("request")]
    assert req["status"] == 0 and req["mesh"] == [16, 8, 8] and req["ms_latency"] >= req["ms_run"]
