"""Oracle (test infrastructure only): the reference's matrix-free MG-PCG on
the CPU, used as the timed CPU baseline and the ``--impl reference`` arm.

Restates ``I/WOK/SolveMGWOK.m:30-57`` (PCG), ``I/WOK/VCycleWOK.m:28-48``
(cycle), ``I/WOK/SmoothWOK.m:20-24`` (damped Jacobi, product taken even for a
zero start), ``I/WOK/AciProd.m:16-24`` (coarse product = prolong to the
finest grid, ``KelemProd``, restrict back) and ``I/WOK/KelemProd.m`` on top of
the C/OpenMP kernels in ``kelem_omp.c``.  The coarsest matrix ``An`` (built
in ``I/WOK/GlobalStiffMatrixWOK.m`` from batched P'KP products) is formed
from Galerkin element matrices - the same matrix - and factored with LAPACK
(``scipy.linalg.cho_factor``) in place of ``amd`` + ``chol``.  Vectors are
full length (3*nnodes) with zeros on fixed dofs.
"""
import ctypes as C
import os
import time

import numpy as np
import scipy.linalg as sla

from . import fem

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libkelem_omp.so")
        if not os.path.exists(path):
            raise ImportError("oracle/libkelem_omp.so not built (python topopt-slp-3d_b200/build.py --oracle)")
        L = C.CDLL(path)
        i, d, p = C.c_int, C.c_double, C.c_void_p
        L.kelem_prod_full.argtypes = [i, i, i, i, p, p, p, p, i]
        L.prolong_full.argtypes = [i, i, i, p, p, p, i, i]
        L.restrict_full.argtypes = [i, i, i, p, p, p, i]
        L.galerkin_fine.argtypes = [i, i, i, i, p, p, p, p, i]
        L.galerkin_coarse.argtypes = [i, i, i, p, p, p, i]
        L.dense_assemble.argtypes = [i, i, i, p, p, p]
        L.grad_full.argtypes = [i, i, i, i, p, p, p, p, d, d, d, p, i]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data


class CpuWok:
    def __init__(self, pb, n, ngrids, omega, nu1=1, nu2=1, p=3.0, emin=1e-9, nthreads=0):
        self.pb, self.n, self.ng, self.omega, self.nu1, self.nu2 = pb, n, ngrids, omega, nu1, nu2
        self.p, self.emin, self.nt = p, emin, nthreads
        self.dims = [(pb.nelx >> l, pb.nely >> l, pb.nelz >> l) for l in range(ngrids)]
        self.ndof = [3 * (a + 1) * (b + 1) * (c + 1) for a, b, c in self.dims]
        fm = np.zeros(self.ndof[0], dtype=np.uint8)
        fm[pb.freedofs] = 1
        self.fm = [fm]
        for l in range(1, ngrids):
            (fx, fy, fz), (cx, cy, cz) = self.dims[l - 1], self.dims[l]
            fmf = self.fm[-1].reshape(fz + 1, fx + 1, fy + 1, 3)
            self.fm.append(np.ascontiguousarray(fmf[::2, ::2, ::2, :]).ravel())
        self.ks = np.ascontiguousarray(fem.elem_stiff_gqmr(pb.el, pb.eh, pb.ew, pb.nu, n))

    # -- setup (SetupGMGWOK / GlobalStiffMatrixWOK) ----------------------------
    def setup(self, dens):
        L = lib()
        self.w = np.ascontiguousarray(fem.simp(dens, self.p, self.emin))
        self.dens = dens
        # diag of every level: M{l} = diag(A_l)/omega
        self.Ae = [None]
        nx, ny, nz = self.dims[0]
        Ae = np.zeros(((nx // 2) * (ny // 2) * (nz // 2), 576))
        L.galerkin_fine(nx, ny, nz, self.n, _p(self.ks), _p(self.w), _p(self.fm[0]), _p(Ae), self.nt)
        self.Ae.append(Ae)
        for l in range(2, self.ng):
            fx, fy, fz = self.dims[l - 1]
            Ac = np.zeros(((fx // 2) * (fy // 2) * (fz // 2), 576))
            L.galerkin_coarse(fx, fy, fz, _p(self.Ae[l - 1]), _p(self.fm[l - 1]), _p(Ac), self.nt)
            self.Ae.append(Ac)
        self.Minv = [self._fine_diag_inv()] + [self._coarse_diag_inv(l) for l in range(1, self.ng - 1)]
        cx, cy, cz = self.dims[-1]
        An = np.zeros((self.ndof[-1], self.ndof[-1]))
        L.dense_assemble(cx, cy, cz, _p(self.Ae[-1]), _p(self.fm[-1]), _p(An))
        self.chol = sla.cho_factor(An, lower=False)

    def _fine_diag_inv(self):
        nx, ny, nz = self.dims[0]
        dofs = fem.dof_table(nx, ny, nz)
        didx = fem.density_table(nx, ny, nz, self.n)
        kd = np.stack([np.diag(k) for k in self.ks])          # ns x 24
        de = self.w[didx] @ kd
        diag = np.bincount(dofs.ravel(), weights=de.ravel(), minlength=self.ndof[0])
        return np.where(self.fm[0] > 0, self.omega / np.where(diag == 0, 1, diag), 0.0)

    def _coarse_diag_inv(self, l):
        nx, ny, nz = self.dims[l]
        dofs = fem.dof_table(nx, ny, nz)
        de = self.Ae[l][:, ::25]                               # diagonal of each 24x24 block
        diag = np.bincount(dofs.ravel(), weights=de.ravel(), minlength=self.ndof[l])
        fm = self.fm[l]
        diag = np.where(fm > 0, diag, 0.0)
        return np.where(fm > 0, self.omega / np.where(diag == 0, 1, diag), 0.0)

    # -- products ------------------------------------------------------------------
    def kelem(self, x):
        nx, ny, nz = self.dims[0]
        y = np.zeros(self.ndof[0])
        lib().kelem_prod_full(nx, ny, nz, self.n, _p(self.ks), _p(self.w), _p(np.ascontiguousarray(x)), _p(y),
                              self.nt)
        y[self.fm[0] == 0] = 0.0
        return y

    def prolong(self, l, xc):          # level l+1 -> l
        cx, cy, cz = self.dims[l + 1]
        xf = np.zeros(self.ndof[l])
        lib().prolong_full(cx, cy, cz, _p(np.ascontiguousarray(xc)), _p(xf), _p(self.fm[l]), 0, self.nt)
        return xf

    def restrict(self, l, rf):         # level l -> l+1
        cx, cy, cz = self.dims[l + 1]
        bc = np.zeros(self.ndof[l + 1])
        lib().restrict_full(cx, cy, cz, _p(np.ascontiguousarray(rf)), _p(bc), _p(self.fm[l + 1]), self.nt)
        return bc

    def aci(self, l, x):
        """AciProd (I/WOK/AciProd.m:16-24)."""
        for i in range(l - 1, -1, -1):
            x = self.prolong(i, x)
        y = self.kelem(x)
        for i in range(l):
            y = self.restrict(i, y)
        return y

    # -- cycle and PCG ----------------------------------------------------------------
    def smooth(self, l, b, x, niter):
        for _ in range(niter):
            x = x + (b - self.aci(l, x)) * self.Minv[l]
        return x

    def vcycle(self, l, b, x0):
        x = self.smooth(l, b, x0, self.nu1)
        rH = self.restrict(l, b - self.aci(l, x))
        if l + 1 == self.ng - 1:
            eH = sla.cho_solve(self.chol, rH)
        else:
            eH = self.vcycle(l + 1, rH, np.zeros(rH.size))
        x = x + self.prolong(l, eH)
        return self.smooth(l, b, x, self.nu2)

    def solve(self, x, f, tol, maxiter, max_iterations=None):
        """SolveMGWOK; stops early after ``max_iterations`` (timing samples).
        Returns (x, it, seconds per iteration list)."""
        r = f - self.kelem(x)
        nf = np.linalg.norm(f)
        nr = np.linalg.norm(r) / nf
        it, times = 1, []
        d = gamma2 = None
        while nr > tol and it <= maxiter:
            if max_iterations is not None and it > max_iterations:
                break
            t0 = time.perf_counter()
            s = self.vcycle(0, r, np.zeros(r.size))
            rho = r @ s
            d = s if it == 1 else (rho / gamma2) * d + s
            q = self.kelem(d)
            alpha = rho / (d @ q)
            x = x + alpha * d
            r = r - alpha * q
            gamma2 = rho
            nr = np.linalg.norm(r) / nf
            it += 1
            times.append(time.perf_counter() - t0)
        return x, it, times

    def grad0(self, u_full, free_elem=None):
        nx, ny, nz = self.dims[0]
        g0 = np.zeros(self.w.size)
        fe = None if free_elem is None else np.ascontiguousarray(free_elem, dtype=np.uint8)
        lib().grad_full(nx, ny, nz, self.n, _p(self.ks), _p(np.ascontiguousarray(u_full)),
                        _p(np.ascontiguousarray(self.dens)), _p(fe) if fe is not None else None,
                        self.p, self.emin, 1.0, _p(g0), self.nt)
        return g0
