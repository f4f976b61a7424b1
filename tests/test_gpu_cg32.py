"""GPU: the CG's tensor-core product (mg.cg_product = 1) and the solve that
uses it, through the C ABI.

* The product (tensor cores, FP32 SIMP factors and vectors, blocks in three
  FP16 pieces) against the FP64 oracle product with FP32-rounded factors and
  input: max error <= 1e-6 of max |y| (FP32 accumulation), and within 2e-6 of
  the FP64 operator itself, for MR factors 1, 2, 3 on ragged meshes.
* Solves: the true relative residual ||f - K u|| / ||f|| with the oracle's
  operator <= 1e-8 (to rounding of the residual itself), the reported residual
  is that true residual, at least one replacement ran, compliance within 1e-8
  of the oracle's FP64 solve, and the iteration count close to the mixed
  solve with the FP64 CG product: within 10 % (at least 3) for MR factors 2
  and 3, within 25 % + 3 on the MR-1 mesh, whose i.i.d. densities put
  stiffness jumps of up to 1e9 between neighbouring elements (45 -> 53
  measured; smooth designs keep the FP64 count).  omega 0.5: with 0.6 the
  Jacobi sweep is not convergent on i.i.d. densities and neither solve
  converges on the MR-1 mesh.
* Refusals: cg_product 1 on FP64 handles or on meshes without the tensor-core
  operator (n * nely odd), and the product entry on other handles.
"""
import numpy as np
import pytest

from oracle import fem, gmg
from tosp import problems as P

pytestmark = pytest.mark.gpu

P_SIMP, EMIN = 3.0, 1e-9


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make(pb, n, seed=0, lo=0.001):
    return np.random.default_rng(seed).uniform(lo, 1, pb.nelem * n ** 3)


def solver(tosp, pb, n, prec=1, **mgkw):
    kw = dict(ngrids=3, cycle=0, omega=0.6, tolMG=1e-8, maxiterMG=500, flexible=1)
    kw.update(mgkw)
    return tosp.Solver(pb, tosp.default_mg(**kw), precision=prec, mr_n=n, p=P_SIMP, emin=EMIN, opfilter=1,
                       rmin=1.0 if n > 1 else 1.5)


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


@pytest.mark.parametrize("dims,n", [((8, 4, 4), 2), ((10, 9, 3), 2), ((12, 16, 6), 2), ((6, 10, 2), 1),
                                    ((9, 6, 5), 1), ((16, 8, 8), 1), ((4, 4, 4), 3), ((5, 6, 3), 3)])
def test_cg32_operator_parity(tosp_mod, dims, n):
    pb = P.cantilever(*dims)
    dens = make(pb, n, seed=sum(dims) + 7)
    s = solver(tosp_mod, pb, n, cg_product=1, omega=0.5)
    s.SetupGMG(dens)
    ks = fem.elem_stiff_gqmr(1, 1, 1, 0.3, n)
    x = np.random.default_rng(5).standard_normal(pb.freedofs.size)
    y = s.KelemProdCG32(x)
    xc = np.zeros(3 * pb.nnodes)
    xc[pb.freedofs] = f32(x)
    w = fem.simp(dens, P_SIMP, EMIN)
    yo = fem.kelem_prod_full(pb.nelx, pb.nely, pb.nelz, ks, f32(w), xc, n)[pb.freedofs]
    e32, e64 = rel(y, yo), rel(y, s.KelemProd(x))
    assert e32 <= 1e-6 and e64 <= 2e-6, (e32, e64)
    s.close()


@pytest.mark.parametrize("dims,n,seed", [((16, 8, 8), 2, 0), ((16, 8, 8), 2, 13), ((24, 12, 12), 1, 3),
                                         ((8, 6, 4), 3, 2)])
@pytest.mark.parametrize("cycle", [0, 1, 2])
def test_cg32_solve(tosp_mod, dims, n, seed, cycle):
    pb = P.cantilever(*dims)
    dens = make(pb, n, seed=seed)
    ks = fem.elem_stiff_gqmr(pb.el, pb.eh, pb.ew, pb.nu, n)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, P_SIMP, EMIN, pb.freedofs)
    ng = 3 if dims[2] >= 8 else 2
    H = gmg.setup_gmg(K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, ng, 0.5)
    uo, ito = gmg.solve_mg(H, np.zeros(pb.f.size), pb.f, cycle, 1, 1, 1e-8, 500)
    nf = np.linalg.norm(pb.f)
    its = {}
    for cgp in (0, 1):
        s = solver(tosp_mod, pb, n, ngrids=ng, cycle=cycle, omega=0.5, cg_product=cgp)
        s.SetupGMG(dens)
        u, it, relres, rc = s.SolveMG(np.zeros(pb.f.size), pb.f)
        st = s.stats()
        s.close()
        assert rc == 0
        rtrue = np.linalg.norm(pb.f - K @ u) / nf
        assert rtrue <= 1.0001e-8, (cgp, rtrue)
        assert abs(pb.f @ u - pb.f @ uo) <= 1e-8 * abs(pb.f @ uo)
        if cgp:
            assert st["replacements"] >= 1
            assert abs(relres - rtrue) <= 1e-3 * rtrue, (relres, rtrue)
        its[cgp] = it
    if n == 1:
        assert its[1] <= its[0] + its[0] // 4 + 3, its
    else:
        assert its[1] <= its[0] + max(3, its[0] // 10), its


def test_cg32_refusals(tosp_mod):
    pb = P.cantilever(8, 4, 4)
    with pytest.raises(tosp_mod.TospError) as e:
        solver(tosp_mod, pb, 2, prec=0, cg_product=1)
    assert e.value.code == -5
    with pytest.raises(tosp_mod.TospError) as e:
        solver(tosp_mod, P.cantilever(5, 7, 3), 1, cg_product=1)
    assert e.value.code == -5
    with pytest.raises(tosp_mod.TospError) as e:
        solver(tosp_mod, pb, 2, cg_product=2)
    assert e.value.code == -1
    s = solver(tosp_mod, pb, 2)
    s.SetupGMG(make(pb, 2))
    with pytest.raises(tosp_mod.TospError) as e:
        s.KelemProdCG32(np.ones(pb.freedofs.size))
    assert e.value.code == -6
    s.close()


def test_cg32_cap_and_warm_start(tosp_mod):
    """At the iteration cap the solve ends with TOSP_NOT_CONVERGED and reports
    the true residual of its iterate (a replacement runs at the end); a warm
    start from that iterate then converges with the true residual <= tolMG."""
    pb = P.cantilever(16, 8, 8)
    dens = make(pb, 2, seed=3)
    ks = fem.elem_stiff_gqmr(pb.el, pb.eh, pb.ew, pb.nu, 2)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, P_SIMP, EMIN, pb.freedofs)
    nf = np.linalg.norm(pb.f)
    s = solver(tosp_mod, pb, 2, omega=0.5, cg_product=1, maxiterMG=5)
    s.SetupGMG(dens)
    u, it, relres, rc = s.SolveMG(np.zeros(pb.f.size), pb.f)
    s.close()
    assert rc == 1 and it == 6
    rtrue = np.linalg.norm(pb.f - K @ u) / nf
    assert abs(relres - rtrue) <= 1e-6 * rtrue, (relres, rtrue)
    s = solver(tosp_mod, pb, 2, omega=0.5, cg_product=1)
    s.SetupGMG(dens)
    u2, it2, relres2, rc2 = s.SolveMG(u, pb.f)
    s.close()
    assert rc2 == 0 and np.linalg.norm(pb.f - K @ u2) <= 1.0001e-8 * nf
