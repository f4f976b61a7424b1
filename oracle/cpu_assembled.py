"""Oracle (test infrastructure only): the reference's default assembled path
(``genK = true``) on the host cores, the timed CPU baseline of the benchmark.

Restates ``I/GlobalStiffMatrix.m:16-65`` (K on the free dofs),
``I/SetupGMG.m:16-77`` (A{l+1} = P'A{l}P, M{l} = diag(A{l})/omega, Cholesky
of the coarsest matrix), ``I/SolveMG.m:26-53`` (PCG, the reference's beta),
``I/VCycle.m:23-43`` / ``I/WCycle.m:23-44`` / ``I/Smooth.m:14-17`` (V- and
W-cycles, damped Jacobi),
``I/Grad.m:18-62`` (sensitivities, transposed filter) and
``I/ApplyFilter.m:74-81`` on top of the C/OpenMP kernels of
``assembled_omp.c`` and ``kelem_omp.c``.  The sparse matrices are stored as
node stencils (27 blocks of 3x3 per node: the non-zeros of MATLAB's sparse
K); P'AP is formed from Galerkin element matrices (the same matrix); the
coarsest system is factored with LAPACK (``scipy.linalg.cho_factor``) in
place of ``amd`` + ``chol``.  The first Jacobi sweep from a zero iterate
takes no product (b - A*0 = b).  Vectors are full length (3*nnodes) with
zeros on fixed dofs.
"""
import ctypes as C
import os

import numpy as np
import scipy.linalg as sla

from . import cpu_wok, fem, filt

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libassembled_omp.so")
        if not os.path.exists(path):
            raise ImportError("oracle/libassembled_omp.so not built (python topopt-slp-3d_b200/build.py --oracle)")
        L = C.CDLL(path)
        i, d, p, i64 = C.c_int, C.c_double, C.c_void_p, C.c_int64
        L.stencil_assemble.argtypes = [i, i, i, i, p, p, p, p, p, i]
        L.stencil_apply.argtypes = [i, i, i, p, p, p, p, p, i, i]
        L.stencil_minv.argtypes = [i, i, i, p, p, d, p]
        L.vec_axpby.argtypes = [i64, d, p, d, p, i]
        L.vec_dot.argtypes = [i64, p, p, i]
        L.vec_dot.restype = d
        L.vec_mul.argtypes = [i64, p, p, p, i]
        L.filter_taps_apply.argtypes = [i, i, i, i, p, p, p, p, p, p, i, i]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data


class CpuAssembled:
    def __init__(self, pb, n, ngrids, omega, nu1=1, nu2=1, p=3.0, emin=1e-9, rmin=1.5, opfilter=1, nthreads=0,
                 cycle=0):
        self.pb, self.n, self.ng, self.omega, self.nu1, self.nu2 = pb, n, ngrids, omega, nu1, nu2
        self.cycle = cycle   # 0 VCycle (I/VCycle.m), 1 WCycle (I/WCycle.m)
        self.p, self.emin, self.nt, self.opfilter = p, emin, nthreads, opfilter
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
        # filter taps of ElemNeighborhood on the density mesh and the row sums w
        self.dd = (pb.nelx * n, pb.nely * n, pb.nelz * n)
        taps = filt.filter_offsets(rmin, pb.el / n, pb.eh / n, pb.ew / n, opfilter) if opfilter else []
        self.off = np.ascontiguousarray(np.array([t[:3] for t in taps], dtype=np.int32).reshape(-1))
        self.tw = np.ascontiguousarray(np.array([t[3] for t in taps], dtype=np.float64))
        self.wsum = np.empty(self.dd[0] * self.dd[1] * self.dd[2])
        if opfilter:
            lib().filter_taps_apply(*self.dd, len(taps), _p(self.off), _p(self.tw), None, None, None,
                                    _p(self.wsum), 0, self.nt)
        self.st = [None] * (ngrids - 1)
        self.minv = [None] * (ngrids - 1)

    # -- GlobalStiffMatrix + SetupGMG --------------------------------------------------
    def setup(self, dens):
        L, W = lib(), cpu_wok.lib()
        self.dens = np.ascontiguousarray(dens, dtype=np.float64)
        self.w = np.ascontiguousarray(fem.simp(self.dens, self.p, self.emin))
        Ae = None
        for l in range(self.ng - 1):
            nx, ny, nz = self.dims[l]
            if self.st[l] is None:
                self.st[l] = np.empty((nx + 1) * (ny + 1) * (nz + 1) * 243)
                self.minv[l] = np.empty(self.ndof[l])
            if l == 0:
                L.stencil_assemble(nx, ny, nz, self.n, _p(self.ks), _p(self.w), None, _p(self.fm[0]),
                                   _p(self.st[0]), self.nt)
            else:
                L.stencil_assemble(nx, ny, nz, 1, None, None, _p(Ae), _p(self.fm[l]), _p(self.st[l]), self.nt)
            L.stencil_minv(nx, ny, nz, _p(self.st[l]), _p(self.fm[l]), self.omega, _p(self.minv[l]))
            # P'AP of this level as Galerkin element matrices of the next one
            Ac = np.zeros(((nx // 2) * (ny // 2) * (nz // 2), 576))
            if l == 0:
                W.galerkin_fine(nx, ny, nz, self.n, _p(self.ks), _p(self.w), _p(self.fm[0]), _p(Ac), self.nt)
            else:
                W.galerkin_coarse(nx, ny, nz, _p(Ae), _p(self.fm[l]), _p(Ac), self.nt)
            Ae = Ac
        cx, cy, cz = self.dims[-1]
        An = np.zeros((self.ndof[-1], self.ndof[-1]))
        W.dense_assemble(cx, cy, cz, _p(Ae), _p(self.fm[-1]), _p(An))
        self.chol = sla.cho_factor(An, lower=False)

    # -- products and the V-cycle ---------------------------------------------------------
    def apply(self, l, x, b=None, mode=0, out=None):
        nx, ny, nz = self.dims[l]
        y = np.empty(self.ndof[l]) if out is None else out
        lib().stencil_apply(nx, ny, nz, _p(self.st[l]), _p(x), _p(b), _p(self.minv[l]), _p(y), mode, self.nt)
        return y

    def vcycle(self, l, b, x0=None):
        """VCycle (I/VCycle.m:23-43) or, with cycle = 1, WCycle
        (I/WCycle.m:23-44: two recursive calls, the second warm-started); from
        a zero iterate unless x0 is given."""
        L, W = lib(), cpu_wok.lib()
        if x0 is None:
            x = np.empty(self.ndof[l])
            if self.nu1 >= 1:
                L.vec_mul(x.size, _p(self.minv[l]), _p(b), _p(x), self.nt)
            else:
                x[:] = 0.0
            first = 1
        else:
            x, first = x0, 0
        for _ in range(first, self.nu1):
            x = self.apply(l, x, b, 2)
        r = self.apply(l, x, b, 1)
        cx, cy, cz = self.dims[l + 1]
        rH = np.empty(self.ndof[l + 1])
        W.restrict_full(cx, cy, cz, _p(r), _p(rH), _p(self.fm[l + 1]), self.nt)
        if l + 1 == self.ng - 1:
            eH = sla.cho_solve(self.chol, rH)
        else:
            eH = self.vcycle(l + 1, rH)
            if self.cycle == 1:
                eH = self.vcycle(l + 1, rH, eH)
        W.prolong_full(cx, cy, cz, _p(np.ascontiguousarray(eH)), _p(x), _p(self.fm[l]), 1, self.nt)
        for _ in range(self.nu2):
            x = self.apply(l, x, b, 2)
        return x

    def solve_iter(self, x, f, tol, maxiter):
        """SolveMG (I/SolveMG.m:26-53) as a generator: yields (it, nr) after
        every PCG iteration; the final iterate is left in ``self.x``."""
        L = lib()
        n, nt = x.size, self.nt
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        r = self.apply(0, x, f, 1) if np.any(x) else f.copy()
        nf = np.sqrt(L.vec_dot(n, _p(f), _p(f), nt))
        nr = np.sqrt(L.vec_dot(n, _p(r), _p(r), nt)) / nf
        it, gamma2 = 1, None
        d = np.zeros(n)
        q = np.empty(n)
        self.x, self.it, self.nr = x, it, nr
        while nr > tol and it <= maxiter:
            s = self.vcycle(0, r)
            rho = L.vec_dot(n, _p(r), _p(s), nt)
            L.vec_axpby(n, 1.0, _p(s), 0.0 if it == 1 else rho / gamma2, _p(d), nt)
            self.apply(0, d, out=q)
            alpha = rho / L.vec_dot(n, _p(d), _p(q), nt)
            L.vec_axpby(n, alpha, _p(d), 1.0, _p(x), nt)
            L.vec_axpby(n, -alpha, _p(q), 1.0, _p(r), nt)
            gamma2 = rho
            nr = np.sqrt(L.vec_dot(n, _p(r), _p(r), nt)) / nf
            it += 1
            self.x, self.it, self.nr = x, it, nr
            yield it, nr

    def solve(self, x, f, tol, maxiter):
        for _ in self.solve_iter(x, f, tol, maxiter):
            pass
        return self.x, self.it, self.nr

    # -- Grad (sensitivities + transposed filter) and ApplyFilter ----------------------------
    def filter(self, x, trans=False):
        if not self.opfilter:
            return np.array(x, dtype=np.float64, copy=True)
        y = np.empty(self.wsum.size)
        lib().filter_taps_apply(*self.dd, self.tw.size, _p(self.off), _p(self.tw), None, _p(self.wsum),
                                _p(np.ascontiguousarray(x, dtype=np.float64)), _p(y), 1 if trans else 0, self.nt)
        return y

    def grad(self, u_full):
        nx, ny, nz = self.dims[0]
        g0 = np.zeros(self.w.size)
        cpu_wok.lib().grad_full(nx, ny, nz, self.n, _p(self.ks), _p(np.ascontiguousarray(u_full)), _p(self.dens),
                                None, self.p, self.emin, 1.0, _p(g0), self.nt)
        return self.filter(g0, trans=True), g0
