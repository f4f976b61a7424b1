"""GPU parity at the benchmark configurations, through the C ABI.

* Golden solutions (tests/golden/solutions.npz, NumPy/SciPy oracle): the FP64
  path with the reference's beta reproduces the reference's `it`, u and the
  sensitivities to 1e-9 relative (summation order only); the mixed path
  reaches a true relative residual <= 1e-8 and the compliance to 1e-7.
* 96x48x48 MR 2 (FP64 drop-in workload): GPU FP64 against the oracle's C/OpenMP
  restatement of the assembled path on the same densities: `it` within one,
  u and dF/drho to 1e-8 relative, F to 1e-9, true residual <= 1e-8.
* 192x96x96 MR 2 (mixed-precision workload, 5.4 M dofs): the mixed solves
  (FP64 CG product every iteration, and the tensor-core CG product with
  residual replacement) and the FP64 GPU solve against the CPU oracle's FP64
  solve: true residuals ||f - K u||/||f|| of the GPU solutions with the
  oracle's operator <= 1e-8 (to rounding of the residual itself), and the
  errors of u, F and dF/drho against the oracle <= 1e-6 relative (printed).
* 48x24x24 SLP loop (20 iterations, knapsack LP, GradProj at the end): GPU
  FP64 against the same loop on the oracle: identical accept/reject sequence,
  compliance history within 1e-9, identical thresholded designs.
"""
import os
import sys

import numpy as np
import pytest

from oracle_solver import AssembledOracleSolver
from tosp import problems as P
from tosp import slp
from tosp.workloads import build_workload

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_solutions as MS  # noqa: E402

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(HERE, "golden", "solutions.npz"))
P_SIMP, EMIN = 3.0, 1e-9


def golden(name):
    return {k.split("/", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(name + "/")}


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def full(pb, u):
    out = np.zeros(3 * pb.nnodes)
    out[pb.freedofs] = u
    return out


def gpu_solver(tosp, pb, n, prec, ngrids, omega, rmin, flexible=0, maxiter=1000, cg_product=0):
    mg = tosp.default_mg(ngrids=ngrids, cycle=0, omega=omega, smoothiter1=1, smoothiter2=1, tolMG=1e-8,
                         maxiterMG=maxiter, flexible=flexible, cg_product=cg_product)
    return tosp.Solver(pb, mg, precision=prec, mr_n=n, p=P_SIMP, emin=EMIN, opfilter=1, rmin=rmin)


@pytest.mark.parametrize("name", list(MS.CASES))
def test_golden_solutions(tosp_mod, name):
    spec = MS.CASES[name]
    pb = MS.case_problem(name)
    gd = golden(name)
    n = spec["n"]
    dens = gd["dens"] if "dens" in gd else np.full(pb.nelem * n ** 3, 0.3)
    orc = AssembledOracleSolver(pb, n=n, ngrids=MS.NGRIDS, omega=spec["omega"], rmin=spec["rmin"])
    orc.SetupGMG(dens)
    nf = np.linalg.norm(pb.f)
    for prec in (tosp_mod.PREC_FP64, tosp_mod.PREC_MIXED):
        s = gpu_solver(tosp_mod, pb, n, prec, MS.NGRIDS, spec["omega"], spec["rmin"],
                       flexible=1 if prec == tosp_mod.PREC_MIXED else 0)
        s.SetupGMG(dens)
        u, it, rr, rc = s.SolveMG(np.zeros(pb.f.size), pb.f)
        g = s.Grad(full(pb, u))
        s.close()
        assert rc == 0
        rtrue = np.linalg.norm(pb.f - orc.KelemProd(u)) / nf
        F = pb.f @ u
        if prec == tosp_mod.PREC_FP64:
            assert abs(it - int(gd["it"][0])) <= 1, (it, gd["it"])
            assert rel_max(u, gd["u"]) <= 1e-9
            assert abs(F - gd["F"][0]) <= 1e-10 * abs(gd["F"][0])
            assert rel_max(g, gd["g"]) <= 1e-9
            assert rtrue <= 1e-8
        else:
            assert rtrue <= 1.001e-8, rtrue
            assert abs(F - gd["F"][0]) <= 1e-7 * abs(gd["F"][0])
            assert rel_max(g, gd["g"]) <= 1e-6


def test_config1_fp64_matches_oracle(tosp_mod):
    """96x48x48, MR 2 (698 691 dofs, 1 769 472 density elements), 4-grid V,
    omega 0.5, FP64 with the reference's beta."""
    pb = P.cantilever(96, 48, 48)
    n, ngrids, omega, rmin = 2, 4, 0.5, 1.0
    orc = AssembledOracleSolver(pb, n=n, ngrids=ngrids, omega=omega, rmin=rmin)
    pb, n, xfil, _ = build_workload("cantilever96x48x48_mr2", filter_fn=orc.ApplyFilter)
    orc.SetupGMG(xfil)
    uo, ito, rro, _ = orc.SolveMG(np.zeros(pb.f.size), pb.f)
    go = orc.Grad(full(pb, uo))
    s = gpu_solver(tosp_mod, pb, n, tosp_mod.PREC_FP64, ngrids, omega, rmin)
    s.SetupGMG(xfil)
    u, it, rr, rc = s.SolveMG(np.zeros(pb.f.size), pb.f)
    g = s.Grad(full(pb, u))
    s.close()
    assert rc == 0 and abs(it - ito) <= 1, (it, ito)
    rtrue = np.linalg.norm(pb.f - orc.KelemProd(u)) / np.linalg.norm(pb.f)
    eu, eF, eg = rel_max(u, uo), abs(pb.f @ u - pb.f @ uo) / abs(pb.f @ uo), rel_max(g, go)
    print(f"config 1 FP64 vs oracle: it {it} / {ito}, true relres {rtrue:.3e}, u {eu:.2e}, F {eF:.2e}, "
          f"dF/drho {eg:.2e}")
    assert rtrue <= 1e-8
    assert eu <= 1e-8 and eF <= 1e-9 and eg <= 1e-8


def test_config2_mixed_and_fp64_against_oracle(tosp_mod):
    """192x96x96, MR 2 (5 447 811 dofs, 14 155 776 density elements), the
    benchmark's 5-grid V-cycle with omega 0.5 and flexible beta, both
    precisions, against the CPU oracle's FP64 solve of the same densities."""
    pb, n, xfil, spec = build_workload("cantilever192x96x96_mr2")
    ngrids, omega, rmin = spec["ngrids"], spec["omega"], spec["rmin"]
    res = {}
    for key, prec, cgp in (("mixed", tosp_mod.PREC_MIXED, 0), ("mixed_cg32", tosp_mod.PREC_MIXED, 1),
                           ("fp64", tosp_mod.PREC_FP64, 0)):
        s = gpu_solver(tosp_mod, pb, n, prec, ngrids, omega, rmin, flexible=1, cg_product=cgp)
        s.SetupGMG(xfil)
        u, it, rr, rc = s.SolveMG(np.zeros(pb.f.size), pb.f)
        g = s.Grad(full(pb, u))
        s.close()
        assert rc == 0, (key, rc)
        res[key] = (u, it, rr, g)
    orc = AssembledOracleSolver(pb, n=n, ngrids=ngrids, omega=omega, rmin=rmin)
    orc.SetupGMG(xfil)
    uo, ito, rro, _ = orc.SolveMG(np.zeros(pb.f.size), pb.f)
    go = orc.Grad(full(pb, uo))
    nf = np.linalg.norm(pb.f)
    Fo = pb.f @ uo
    for key, (u, it, rr, g) in res.items():
        rtrue = np.linalg.norm(pb.f - orc.KelemProd(u)) / nf
        eu, eF, eg = rel_max(u, uo), abs(pb.f @ u - Fo) / abs(Fo), rel_max(g, go)
        print(f"config 2 {key}: it {it} (oracle {ito}), CG relres {rr:.3e}, true relres {rtrue:.3e}, "
              f"errors vs oracle: u {eu:.2e}, F {eF:.2e}, dF/drho {eg:.2e}")
        assert rtrue <= 1.001e-8, (key, rtrue)
        assert eu <= 1e-6 and eF <= 1e-6 and eg <= 1e-6, (key, eu, eF, eg)


def test_config0_slp_loop_matches_oracle(tosp_mod):
    """The 48x24x24 cantilever loop: 20 SLP iterations from uniform 0.3,
    volume fraction 0.3, filter radius 1.5, 3-grid V-cycle with omega 0.6,
    FP64, knapsack LP, GradProj thresholding at the end.  The iteration cap is
    the reference default (maxiterMG = 5000): with omega 0.6 some designs of
    this loop need more than 1000 PCG iterations, and an unconverged solve
    would make the two loops' trust-region decisions depend on rounding."""
    pb = P.cantilever(48, 24, 24)
    x0 = np.full(pb.nelem, 0.3)
    params = slp.SlpParams(maxiter=20, lp="knapsack")
    gpu = gpu_solver(tosp_mod, pb, 1, tosp_mod.PREC_FP64, 3, 0.6, 1.5, maxiter=5000)
    orc = AssembledOracleSolver(pb, n=1, ngrids=3, omega=0.6, rmin=1.5, maxiter=5000)
    r1 = slp.str_slp(gpu, pb, 0.3, x0, params, prj=slp.PrjParams(op=True))
    r2 = slp.str_slp(orc, pb, 0.3, x0, params, prj=slp.PrjParams(op=True))
    gpu.close()
    assert r1.iters == r2.iters == 20 and r1.rejected == r2.rejected
    assert all(st == 0 for st in r1.pcgstatus)
    assert [h["it"] for h in r1.history] == [h["it"] for h in r2.history]
    for h1, h2 in zip(r1.history, r2.history):
        assert abs(h1["F"] - h2["F"]) <= 1e-9 * abs(h2["F"])
    print(f"config 0 loop: F {r1.F:.12g} vs oracle {r2.F:.12g}, design max diff "
          f"{np.abs(r1.x - r2.x).max():.2e}, thresholded elements {int(r1.xstar.sum())}")
    assert np.array_equal(r1.xstar, r2.xstar)
    assert set(np.unique(r1.xstar)) <= {0.0, 1.0}
