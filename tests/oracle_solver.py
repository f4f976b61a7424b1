"""Oracle-backed solve path with the interface of tosp.Solver (tests only):
assembled K (I/GlobalStiffMatrix.m), SetupGMG + SolveMG (I/SetupGMG.m,
I/SolveMG.m), Grad (I/Grad.m) and ApplyFilter (I/ApplyFilter.m) on the CPU."""
import numpy as np

from oracle import fem, filt, gmg


class OracleSolver:
    def __init__(self, pb, n=1, ngrids=3, cycle=0, omega=0.6, nu1=1, nu2=1, tol=1e-8, maxiter=1000, p=3.0,
                 emin=1e-9, opfilter=1, rmin=1.5, fixed=None):
        self.pb, self.n, self.ngrids, self.cycle, self.omega = pb, n, ngrids, cycle, omega
        self.nu1, self.nu2, self.tol, self.maxiter, self.p, self.emin = nu1, nu2, tol, maxiter, p, emin
        self.opfilter = opfilter
        self.ks = fem.elem_stiff_gqmr(pb.el, pb.eh, pb.ew, pb.nu, n)
        self.W, self.w = filt.elem_neighborhood(pb.nelx * n, pb.nely * n, pb.nelz * n, pb.el / n, pb.eh / n,
                                                pb.ew / n, rmin, opfilter, fixed=fixed)

    def ApplyFilter(self, x, trans=False):
        return filt.apply_filter(np.asarray(x, dtype=np.float64), self.W, self.w, self.opfilter, trans)

    def SetupGMG(self, xfil):
        pb = self.pb
        self.dens = np.asarray(xfil, dtype=np.float64).copy()
        self.K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, self.ks, self.dens, self.p, self.emin,
                                         pb.freedofs)
        self.H = gmg.setup_gmg(self.K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, self.ngrids, self.omega)

    def SolveMG(self, x, f):
        u, it = gmg.solve_mg(self.H, np.asarray(x, dtype=np.float64), f, self.cycle, self.nu1, self.nu2, self.tol,
                             self.maxiter)
        r = np.linalg.norm(f - self.K @ u) / np.linalg.norm(f)
        return u, it, r, 0

    def Grad(self, u_full):
        pb = self.pb
        g, _ = filt.grad(pb.nelx, pb.nely, pb.nelz, self.ks, u_full, self.dens, self.p, self.emin, self.W, self.w,
                         self.opfilter)
        return g


class AssembledOracleSolver:
    """The same interface on the C/OpenMP restatement of the assembled path
    (oracle/cpu_assembled.py; V-cycle, reference beta), which
    tests/test_cpu_port.py pins to the NumPy/SciPy oracle.  Fast enough for
    benchmark-size meshes and whole SLP loops."""

    def __init__(self, pb, n=1, ngrids=3, omega=0.6, tol=1e-8, maxiter=1000, p=3.0, emin=1e-9, opfilter=1,
                 rmin=1.5, nthreads=0):
        import os
        from oracle.cpu_assembled import CpuAssembled
        self.pb, self.tol, self.maxiter = pb, tol, maxiter
        self.ca = CpuAssembled(pb, n, ngrids, omega, p=p, emin=emin, rmin=rmin, opfilter=opfilter,
                               nthreads=nthreads or os.cpu_count())

    def ApplyFilter(self, x, trans=False):
        return self.ca.filter(x, trans)

    def SetupGMG(self, xfil):
        self.ca.setup(xfil)

    def _full(self, v):
        out = np.zeros(3 * self.pb.nnodes)
        out[self.pb.freedofs] = v
        return out

    def KelemProd(self, x):
        return self.ca.apply(0, self._full(x))[self.pb.freedofs]

    def SolveMG(self, x, f):
        u, it, nr = self.ca.solve(self._full(x), self._full(f), self.tol, self.maxiter)
        return u[self.pb.freedofs], it, nr, 0

    def Grad(self, u_full):
        return self.ca.grad(u_full)[0]
