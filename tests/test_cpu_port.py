"""The C/OpenMP port of the matrix-free path (timed CPU baseline) agrees with
the NumPy oracle (assembled path)."""
import numpy as np
import pytest

from oracle import fem, filt, gmg
from tosp import problems as P

cpu_wok = pytest.importorskip("oracle.cpu_wok")


@pytest.fixture(scope="module")
def case():
    import __graft_entry__  # noqa: F401
    from oracle.cpu_wok import lib
    try:
        lib()
    except ImportError:
        import subprocess, sys, os
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        subprocess.check_call([sys.executable, os.path.join(root, "topopt-slp-3d_b200", "build.py"), "--oracle"])
    pb = P.cantilever(16, 8, 8)
    n = 2
    dens = np.random.default_rng(11).uniform(0.001, 1, pb.nelem * n ** 3)
    ks = fem.elem_stiff_gqmr(1, 1, 1, 0.3, n)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, 3, 1e-9, pb.freedofs)
    H = gmg.setup_gmg(K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, 3, 0.6)
    cw = cpu_wok.CpuWok(pb, n, 3, 0.6, nthreads=4)
    cw.setup(dens)
    return pb, n, dens, ks, K, H, cw


def test_kelem_and_cycle(case):
    pb, n, dens, ks, K, H, cw = case
    x = np.random.default_rng(0).standard_normal(pb.freedofs.size)
    xf = np.zeros(3 * pb.nnodes)
    xf[pb.freedofs] = x
    y = K @ x
    assert np.abs(cw.kelem(xf)[pb.freedofs] - y).max() <= 1e-13 * np.abs(y).max()
    s = gmg.precondition(H, x, 0, 1, 1)
    s2 = cw.vcycle(0, xf, np.zeros(xf.size))[pb.freedofs]
    assert np.abs(s - s2).max() <= 1e-11 * np.abs(s).max()


def test_solve_and_grad(case):
    pb, n, dens, ks, K, H, cw = case
    uo, ito = gmg.solve_mg(H, np.zeros(pb.f.size), pb.f, 0, 1, 1, 1e-8, 500)
    ff = pb.f_full()
    u, it, _ = cw.solve(np.zeros(ff.size), ff, 1e-8, 500)
    assert abs(it - ito) <= 1
    assert abs(ff @ u - pb.f @ uo) <= 1e-9 * abs(pb.f @ uo)
    W, w = filt.elem_neighborhood(32, 16, 16, 0.5, 0.5, 0.5, 1.0, 1)
    _, g0 = filt.grad(16, 8, 8, ks, u, dens, 3, 1e-9, W, w, 1)
    assert np.abs(cw.grad0(u) - g0).max() <= 1e-12 * np.abs(g0).max()


def test_assembled_port_matches_oracle(case):
    """The C/OpenMP port of the assembled path (GlobalStiffMatrix + SetupGMG +
    SolveMG + Grad, the timed reference arm) against the SciPy oracle: the
    product, one V-cycle, the full solve (iterations, compliance) and Grad
    with the transposed filter."""
    from oracle.cpu_assembled import CpuAssembled
    pb, n, dens, ks, K, H, cw = case
    ca = CpuAssembled(pb, n, 3, 0.6, rmin=1.0, nthreads=4)
    ca.setup(dens)
    x = np.random.default_rng(3).standard_normal(pb.freedofs.size)
    xf = np.zeros(3 * pb.nnodes)
    xf[pb.freedofs] = x
    y = K @ x
    assert np.abs(ca.apply(0, xf)[pb.freedofs] - y).max() <= 1e-13 * np.abs(y).max()
    s = gmg.precondition(H, x, 0, 1, 1)
    assert np.abs(ca.vcycle(0, xf)[pb.freedofs] - s).max() <= 1e-11 * np.abs(s).max()
    uo, ito = gmg.solve_mg(H, np.zeros(pb.f.size), pb.f, 0, 1, 1, 1e-8, 500)
    ff = pb.f_full()
    u, it, nr = ca.solve(np.zeros(ff.size), ff, 1e-8, 500)
    assert it == ito and nr <= 1e-8
    assert abs(ff @ u - pb.f @ uo) <= 1e-10 * abs(pb.f @ uo)
    W, w = filt.elem_neighborhood(32, 16, 16, 0.5, 0.5, 0.5, 1.0, 1)
    assert np.abs(ca.wsum - w).max() <= 1e-13 * w.max()
    go, _ = filt.grad(16, 8, 8, ks, u, dens, 3, 1e-9, W, w, 1)
    g, _ = ca.grad(u)
    assert np.abs(g - go).max() <= 1e-12 * np.abs(go).max()
    xr = np.random.default_rng(4).uniform(0, 1, dens.size)
    assert np.abs(ca.filter(xr) - filt.apply_filter(xr, W, w, 1, False)).max() <= 1e-14


def test_assembled_port_w_cycle_matches_oracle(case):
    """The C/OpenMP assembled path's WCycle (I/WCycle.m) against the SciPy
    oracle's: one preconditioner application and a full solve."""
    from oracle.cpu_assembled import CpuAssembled
    pb, n, dens, ks, K, H, cw = case
    ca = CpuAssembled(pb, n, 3, 0.6, rmin=1.0, nthreads=4, cycle=1)
    ca.setup(dens)
    x = np.random.default_rng(5).standard_normal(pb.freedofs.size)
    xf = np.zeros(3 * pb.nnodes)
    xf[pb.freedofs] = x
    s = gmg.precondition(H, x, 1, 1, 1)
    assert np.abs(ca.vcycle(0, xf)[pb.freedofs] - s).max() <= 1e-11 * np.abs(s).max()
    uo, ito = gmg.solve_mg(H, np.zeros(pb.f.size), pb.f, 1, 1, 1, 1e-8, 500)
    u, it, nr = ca.solve(np.zeros(3 * pb.nnodes), pb.f_full(), 1e-8, 500)
    assert it == ito and abs(pb.f_full() @ u - pb.f @ uo) <= 1e-10 * abs(pb.f @ uo)
