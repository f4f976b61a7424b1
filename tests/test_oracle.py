"""CPU tests of the oracle: pins against the reference's closed-form element
matrix and its internal cross-implementations (I/ = Implementation/)."""
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle import fem, filt, gmg
from tosp import problems as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_gqmr_sum_equals_closed_form_ke():
    """sum_s KE_s (I/ElemStiffMatrixGQMR.m) == KE (I/ElemStiffMatrix.m) for n = 1, 2, 3."""
    d = np.load(os.path.join(GOLD, "ke_closed_form.npz"))
    for shape, ke in zip(d["shapes"], d["ke"]):
        for n in (1, 2, 3):
            ks = fem.elem_stiff_gqmr(*shape, n)
            assert np.abs(ks.sum(0) - ke).max() <= 1e-14 * np.abs(ke).max()


def test_ke_blocks_symmetric_psd_rigid_modes():
    ks = fem.elem_stiff_gqmr(1.0, 0.5, 2.0, 0.3, 2)
    for k in ks:
        assert np.array_equal(k, k.T)
    ev = np.linalg.eigvalsh(ks.sum(0))
    assert ev.min() > -1e-12
    assert np.sum(np.abs(ev) < 1e-10 * ev.max()) == 6     # 3 translations + 3 rotations


def test_numbering_conventions():
    dofs = fem.dof_table(3, 2, 2)
    # element 0: nodes (x0,y0,z0) (x0,y1,z0) (x1,y0,z0) (x1,y1,z0) ... (I/DegreesOfFreedom.m:24-38)
    ny, nx = 3, 4
    n0 = [0, 1, ny, ny + 1, nx * ny, nx * ny + 1, nx * ny + ny, nx * ny + ny + 1]
    assert dofs[0].tolist() == [3 * n + c for n in n0 for c in range(3)]
    # element order: y fastest, then x, then z
    assert dofs[1, 0] == 3 * 1 and dofs[2, 0] == 3 * ny
    didx = fem.density_table(2, 2, 1, 2)
    assert didx[0].tolist() == [0, 1, 4, 5, 16, 17, 20, 21]   # sub-elements y, x, z


@pytest.mark.parametrize("n", [1, 2, 3])
def test_kelem_prod_equals_assembled(n):
    """KelemProd (I/WOK/KelemProd.m) == GlobalStiffMatrix*x (I/GlobalStiffMatrix.m)."""
    pb = P.cantilever(4, 4, 2)
    ks = fem.elem_stiff_gqmr(1, 1, 1, 0.3, n)
    rng = np.random.default_rng(n)
    dens = rng.uniform(0.001, 1, pb.nelem * n ** 3)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, 3, 1e-9, pb.freedofs)
    x = rng.standard_normal(pb.freedofs.size)
    y = fem.kelem_prod(pb.nelx, pb.nely, pb.nelz, ks, dens, 3, 1e-9, pb.freedofs, x)
    assert np.abs(K @ x - y).max() <= 1e-13 * np.abs(y).max()


def test_prolongation_rowsums_and_coarse_free():
    fd = P.cantilever(4, 4, 4).freedofs
    Pm, fdc = gmg.prolongation(5, 5, 5, 3, 3, 3, fd)
    # interior fine rows of trilinear interpolation sum to 1
    full, _ = gmg.prolongation(5, 5, 5, 3, 3, 3, np.arange(375))
    assert np.allclose(np.asarray(full.sum(axis=1)).ravel(), 1.0)
    # coarse dofs on the fixed x = 0 face are removed
    assert fdc.size == 3 * 27 - 3 * 9


@pytest.mark.parametrize("cycle", [0, 1, 2])
def test_solve_mg_matches_direct(cycle):
    """SolveMG (I/SolveMG.m) reaches tolMG and agrees with a direct solve."""
    pb = P.cantilever(8, 4, 4)
    n = 2
    ks = fem.elem_stiff_gqmr(1, 1, 1, 0.3, n)
    dens = np.random.default_rng(0).uniform(0.001, 1, pb.nelem * n ** 3)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, 3, 1e-9, pb.freedofs)
    H = gmg.setup_gmg(K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, 3, 0.6)
    u, it = gmg.solve_mg(H, np.zeros(pb.f.size), pb.f, cycle, 1, 1, 1e-8, 500)
    ud = spla.spsolve(K.tocsc(), pb.f)
    assert np.linalg.norm(pb.f - K @ u) <= 1e-8 * np.linalg.norm(pb.f)
    assert abs(pb.f @ u - pb.f @ ud) <= 1e-6 * abs(pb.f @ ud)
    assert 2 <= it < 100


def test_level_rule():
    """I/StartStrSLP.m:107-133: configs' level counts."""
    assert gmg.gmg_levels(96, 48, 48, 4) == (4, 0)
    assert gmg.gmg_levels(192, 96, 96, 3) == (4, 0)          # 12675 coarse dofs <= 60000
    assert gmg.gmg_levels(160, 80, 40, 5)[0] == 4            # 40 limits to 2^3
    assert gmg.gmg_levels(30, 10, 10, 3)[0] == 2


def test_filter_matrix_symmetric_and_fixed_decoupled():
    W, w = filt.elem_neighborhood(6, 5, 4, 1, 1, 1, 1.5, 1, fixed=np.array([3, 17]))
    assert abs(W - W.T).max() == 0
    assert W[3, 3] == 1.0 and W[3].nnz == 1
    assert np.allclose(w, np.asarray(W.sum(axis=1)).ravel())
    # interior stencil of rmin = 1.5 on unit cells has 19 taps
    W2, _ = filt.elem_neighborhood(7, 7, 7, 1, 1, 1, 1.5, 1)
    assert W2[171].nnz == 19
    W3, _ = filt.elem_neighborhood(9, 9, 9, 1, 1, 1, 2.5, 2)
    assert W3[364].nnz == 81


def test_grad_finite_difference():
    """dF/drho of F = f'u (I/Grad.m) against central differences (no filter)."""
    pb = P.cantilever(4, 2, 2)
    n = 2
    ks = fem.elem_stiff_gqmr(1, 1, 1, 0.3, n)
    rng = np.random.default_rng(3)
    dens = rng.uniform(0.2, 1, pb.nelem * n ** 3)
    def compliance(d):
        K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, d, 3, 1e-9, pb.freedofs)
        u = spla.spsolve(K.tocsc(), pb.f)
        return pb.f @ u, u
    F, u = compliance(dens)
    uf = np.zeros(3 * pb.nnodes)
    uf[pb.freedofs] = u
    I = np.eye(dens.size)
    W = __import__("scipy.sparse", fromlist=["eye"]).eye(dens.size).tocsr()
    g, g0 = filt.grad(pb.nelx, pb.nely, pb.nelz, ks, uf, dens, 3, 1e-9, W, np.ones(dens.size), 1)
    for i in (0, 5, 17, 40):
        h = 1e-6
        fd = (compliance(dens + h * I[i])[0] - compliance(dens - h * I[i])[0]) / (2 * h)
        assert abs(fd - g0[i]) <= 1e-5 * abs(g0[i]) + 1e-12


def test_coarsest_pcg_branch_matches_direct_solve():
    """The oracle's opchol = 1 branch (I/VCycle.m:28-35: pcg with the diagonal
    preconditioner to tolPCG = 1e-8) gives the direct solve's cycle to within
    the PCG tolerance, and tighter as the tolerance shrinks."""
    import numpy as np
    from oracle import fem, gmg
    from tosp import problems as P
    pb = P.cantilever(12, 6, 6)
    dens = np.random.default_rng(3).uniform(0.001, 1, pb.nelem)
    ks = fem.elem_stiff_gqmr(pb.el, pb.eh, pb.ew, pb.nu, 1)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, 3.0, 1e-9, pb.freedofs)
    r = np.random.default_rng(5).standard_normal(pb.freedofs.size)
    Hd = gmg.setup_gmg(K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, 2, 0.5)
    zd = gmg.precondition(Hd, r, 0, 1, 1)
    errs = []
    for tol in (1e-6, 1e-10):
        Hp = gmg.setup_gmg(K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, 2, 0.5, opchol=1, tolPCG=tol)
        zp = gmg.precondition(Hp, r, 0, 1, 1)
        errs.append(np.abs(zp - zd).max() / np.abs(zd).max())
    assert errs[1] <= 1e-7 and errs[1] < errs[0]
