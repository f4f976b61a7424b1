"""SLP loop on the GPU solve path against the same loop on the oracle
(I/StrSLP.m restated in tosp.slp).  Tolerance: every solve stops at
||f - K u|| <= 1e-8 ||f||, so the compliance histories agree to 1e-6
relative and the accept/reject decisions are identical."""
import numpy as np
import pytest

from oracle_solver import OracleSolver
from tosp import problems as P
from tosp import slp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lp", ["highs", "knapsack"])
def test_slp_gpu_matches_oracle(tosp_mod, lp):
    pb = P.cantilever(16, 8, 8)
    x0 = np.full(pb.nelem, 0.3)
    gpu = tosp_mod.Solver(pb, tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=1000),
                          precision=tosp_mod.PREC_FP64, mr_n=1, p=3.0, emin=1e-9, opfilter=1, rmin=1.5)
    orc = OracleSolver(pb, ngrids=3, cycle=0, omega=0.6, rmin=1.5)
    params = slp.SlpParams(maxiter=6, lp=lp)
    r1 = slp.str_slp(gpu, pb, 0.3, x0, params)
    r2 = slp.str_slp(orc, pb, 0.3, x0, params)
    assert r1.iters == r2.iters and r1.rejected == r2.rejected
    for h1, h2 in zip(r1.history, r2.history):
        assert h1["it"] == h2["it"]
        assert abs(h1["F"] - h2["F"]) <= 1e-6 * abs(h2["F"])
    assert np.abs(r1.x - r2.x).max() <= 1e-5
    assert r1.F < r1.history[0]["F"] or r1.iters == 0


def test_slp_mixed_precision_same_designs(tosp_mod):
    pb = P.cantilever(16, 8, 8)
    x0 = np.full(pb.nelem, 0.3)
    kw = dict(mr_n=1, p=3.0, emin=1e-9, opfilter=1, rmin=1.5)
    mg = tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=1000, flexible=1)
    r64 = slp.str_slp(tosp_mod.Solver(pb, mg, precision=0, **kw), pb, 0.3, x0, slp.SlpParams(maxiter=6))
    rmx = slp.str_slp(tosp_mod.Solver(pb, mg, precision=1, **kw), pb, 0.3, x0, slp.SlpParams(maxiter=6))
    assert abs(r64.F - rmx.F) <= 1e-6 * abs(r64.F)
    prj = slp.PrjParams(op=True)
    V = pb.l * pb.h * pb.w
    velem = np.full(pb.nelem, V / pb.nelem)
    t64 = slp.grad_proj(r64.xstar, np.ones(pb.nelem), prj, 0.3 * V, velem)
    tmx = slp.grad_proj(rmx.xstar, np.ones(pb.nelem), prj, 0.3 * V, velem)
    assert np.abs(r64.x - rmx.x).max() <= 1e-5
    # GradProj's tie rule (inputs snapped to 2^-30 of their scale) makes the
    # thresholded designs of the two precisions identical
    assert np.array_equal(t64, tmx)


def test_correct_function_value_matches_oracle(tosp_mod):
    """CorrectFunctionValue (I/CorrectFunctionValue.m): re-solve the MR design
    on the density mesh; against the oracle's assembled solve on that mesh."""
    import scipy.sparse.linalg as spla
    from oracle import fem
    pb = P.cantilever(8, 4, 4)
    n = 2
    x = np.random.default_rng(2).uniform(0.2, 1.0, pb.nelem * n ** 3)
    F, it, rr = slp.correct_function_value(pb, n, x, tosp_mod.default_mg(ngrids=3, cycle=1, omega=0.5))
    strT = slp.density_mesh_problem(pb, n)
    ks = fem.elem_stiff_gqmr(strT.el, strT.eh, strT.ew, strT.nu, 1)
    K = fem.global_stiff_matrix(strT.nelx, strT.nely, strT.nelz, ks, x, 3.0, 1e-9, strT.freedofs)
    u = spla.spsolve(K.tocsc(), strT.f)
    assert rr <= 1e-8
    assert abs(F - strT.f @ u) <= 1e-7 * abs(strT.f @ u)
