"""Python binding of the tosp C ABI (``include/tosp.h``).

The functions keep the names and argument meaning of the reference MATLAB
functions they replace (``SetupGMG``/``SetupGMGWOK``, ``SolveMG``,
``KelemProd``, ``Grad``, ``ApplyFilter``, ``ElemStiffMatrixGQMR``) so host
code reads like the reference's ``StrSLP``; the heavy MATLAB arguments
(``A, P, M, R, perm, kv, W``) live inside a :class:`Solver` handle.

Indices crossing the ABI are 1-based like MATLAB; the Python layer takes the
0-based arrays of :mod:`tosp.problems` and converts.  The CUDA library must be
built (``python topopt-slp-3d_b200/build.py``); without it the first call
into the library raises ``ImportError`` - there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from . import problems  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtosp.so")

TOSP_OK = 0
TOSP_NOT_CONVERGED = 1
TOSP_ERR_BREAKDOWN = -4
PREC_FP64 = 0
PREC_MIXED = 1
STATUS = {0: "OK", 1: "NOT_CONVERGED", -1: "BAD_ARG", -2: "CUDA_ERROR", -3: "OOM", -4: "BREAKDOWN",
          -5: "UNSUPPORTED", -6: "STATE", -7: "CANCELLED", -8: "TIMEOUT"}


class TospError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tosp error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class _Problem(C.Structure):
    _fields_ = [("nelx", C.c_int32), ("nely", C.c_int32), ("nelz", C.c_int32),
                ("el", C.c_double), ("eh", C.c_double), ("ew", C.c_double),
                ("E", C.c_double), ("nu", C.c_double), ("p", C.c_double), ("emin", C.c_double),
                ("mr_n", C.c_int32), ("opfilter", C.c_int32), ("rmin", C.c_double),
                ("freedofs", C.POINTER(C.c_int64)), ("nfree", C.c_int64),
                ("fixed_dens", C.POINTER(C.c_int64)), ("nfixed_dens", C.c_int64),
                ("free_dens_g", C.POINTER(C.c_int64)), ("nfree_dens_g", C.c_int64)]


class MgParams(C.Structure):
    """The ``mg.*`` struct of the reference (I/TopOpt3D.m:171-190)."""
    _fields_ = [("ngrids", C.c_int32), ("cycle", C.c_int32), ("smoother", C.c_int32), ("omega", C.c_double),
                ("smoothiter1", C.c_int32), ("smoothiter2", C.c_int32), ("tolMG", C.c_double),
                ("maxiterMG", C.c_int32), ("nmaxchol", C.c_int32), ("flexible", C.c_int32),
                ("maxstall", C.c_int32), ("warp_stencil_max", C.c_int32), ("small_cycle_max", C.c_int32),
                ("cg_product", C.c_int32), ("replace_drop", C.c_double),
                ("opchol", C.c_int32), ("opcond", C.c_int32), ("tolPCG", C.c_double), ("maxiterPCG", C.c_int32)]


class RequestStats(C.Structure):
    _fields_ = [("it", C.c_int32), ("relres", C.c_double), ("ms_latency", C.c_double), ("ms_queue", C.c_double),
                ("ms_run", C.c_double), ("precision", C.c_int32)]


class SolveStats(C.Structure):
    _fields_ = [("it", C.c_int32), ("relres", C.c_double), ("ms_setup", C.c_double), ("ms_solve", C.c_double),
                ("replacements", C.c_int32)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"tosp CUDA library not built: {LIB_PATH} missing "
                          "(run python topopt-slp-3d_b200/build.py)")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    d = C.c_void_p   # double* (host or device address)
    sig = {
        "tosp_version": (C.c_char_p, []),
        "tosp_default_mg_params": (None, [P(MgParams)]),
        "tosp_create": (C.c_int, [P(_Problem), P(MgParams), C.c_int32, P(C.c_void_p)]),
        "tosp_destroy": (C.c_int, [C.c_void_p]),
        "tosp_last_error": (C.c_char_p, [C.c_void_p]),
        "tosp_info": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int64), P(C.c_int64)]),
        "tosp_set_freedofs": (C.c_int, [C.c_void_p, P(C.c_int64), C.c_int64]),
        "tosp_setup_gmg": (C.c_int, [C.c_void_p, d, C.c_int64]),
        "tosp_kelem_prod": (C.c_int, [C.c_void_p, d, d, C.c_int64]),
        "tosp_kelem_prod_mixed": (C.c_int, [C.c_void_p, d, d, C.c_int64]),
        "tosp_kelem_prod_cg32": (C.c_int, [C.c_void_p, d, d, C.c_int64]),
        "tosp_mg_cycle": (C.c_int, [C.c_void_p, d, d, C.c_int64]),
        "tosp_solve_mg": (C.c_int, [C.c_void_p, d, d, C.c_int64, P(C.c_int32), P(C.c_double)]),
        "tosp_grad": (C.c_int, [C.c_void_p, d, C.c_int64, d, d, C.c_int64]),
        "tosp_apply_filter": (C.c_int, [C.c_void_p, d, d, C.c_int64, C.c_int32]),
        "tosp_filter_weights": (C.c_int, [C.c_void_p, d, C.c_int64]),
        "tosp_compliance": (C.c_int, [C.c_void_p, d, d, C.c_int64, P(C.c_double)]),
        "tosp_last_stats": (C.c_int, [C.c_void_p, P(SolveStats)]),
        "tosp_elem_stiff_mr": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, d]),
        "tosp_kernel_launches": (C.c_int64, []),
        "tosp_time_operator": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, P(C.c_double)]),
        "tosp_kelem_prod_noalloc": (C.c_int, [C.c_void_p, d, d, C.c_int64]),
        "tosp_inject_wait_fault": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "tosp_small_cycle_blocks": (C.c_int, [C.c_void_p, P(C.c_int32)]),
        "tosp_server_create": (C.c_int, [C.c_int32, C.c_int64, P(C.c_void_p)]),
        "tosp_server_prepare": (C.c_int, [C.c_void_p, P(_Problem), P(MgParams), C.c_int32, C.c_int32]),
        "tosp_server_submit": (C.c_int, [C.c_void_p, P(_Problem), P(MgParams), C.c_int32, d, C.c_int64, d, C.c_int64,
                                         P(C.c_int64)]),
        "tosp_server_poll": (C.c_int, [C.c_void_p, C.c_int64, P(C.c_int32)]),
        "tosp_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_double]),
        "tosp_server_result": (C.c_int, [C.c_void_p, C.c_int64, d, C.c_int64, d, C.c_int64, P(RequestStats)]),
        "tosp_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
        "tosp_server_release": (C.c_int, [C.c_void_p, C.c_int64]),
        "tosp_server_info": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_int32), P(C.c_int64), P(C.c_int64)]),
        "tosp_server_destroy": (C.c_int, [C.c_void_p]),
        "tosp_server_counters": (C.c_int, [C.c_void_p, P(C.c_int64), P(C.c_int64), P(C.c_int64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _LazyLib:
    """The ctypes library, mapped on first use: importing ``tosp`` for its
    problem builders or workloads loads no native code.  The first call raises
    ImportError when the library is not built (there is no CPU fallback)."""

    _lib = None

    def loaded(self):
        if _LazyLib._lib is None:
            _LazyLib._lib = _load()
        return _LazyLib._lib

    def __getattr__(self, name):
        return getattr(self.loaded(), name)


_lib = _LazyLib()


def exported_symbols():
    """Names of the entry points bound from the library."""
    return [n for n in dir(_lib.loaded()) if n.startswith("tosp_")]


def kernel_launches():
    """Kernel launches issued by the library since load (all handles)."""
    return int(_lib.tosp_kernel_launches())


def version():
    return _lib.tosp_version().decode()


def _ptr(a):
    """Address of a float64 NumPy array (host) or a CUDA tensor (device)."""
    if isinstance(a, np.ndarray):
        assert a.dtype == np.float64 and a.flags.c_contiguous
        return a.ctypes.data
    if hasattr(a, "data_ptr"):   # torch.Tensor on the GPU (device pointer path)
        return a.data_ptr()
    raise TypeError("expected a float64 numpy array or a CUDA tensor")


def _i64(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(C.POINTER(C.c_int64))


def default_mg(**kw):
    mg = MgParams()
    _lib.tosp_default_mg_params(C.byref(mg))
    for k, v in kw.items():
        setattr(mg, k, v)
    return mg


def ElemStiffMatrixGQMR(el, eh, ew, nu, n):
    """``kv`` of I/ElemStiffMatrixGQMR.m (576 x n^3, column s = k{s}(:))."""
    kv = np.zeros((n ** 3, 576))
    rc = _lib.tosp_elem_stiff_mr(el, eh, ew, nu, n, kv.ctypes.data)
    if rc:
        raise TospError(rc, "tosp_elem_stiff_mr")
    return kv.T.copy()


class Solver:
    """A solve handle: problem, multigrid hierarchy and device state.

    ``pb`` is a :class:`tosp.problems.Problem` (0-based arrays).  ``mr_n`` is
    the multiresolution factor (density sub-elements per direction; design
    mesh = density mesh).  ``fixed_dens`` (0-based, density mesh) defaults
    to the problem's ``fixed_dens`` when ``mr_n == 1``.
    """

    def __init__(self, pb, mg=None, precision=PREC_FP64, mr_n=1, p=3.0, emin=1e-9, opfilter=1, rmin=1.5,
                 fixed_dens=None, free_dens_g=None):
        self.pb = pb
        self.mr_n = mr_n
        self.mg = mg if mg is not None else default_mg()
        fd1, fdp = _i64(np.asarray(pb.freedofs) + 1)
        if fixed_dens is None and mr_n == 1 and pb.fixed_dens is not None:
            fixed_dens = pb.fixed_dens
        self._keep = [fd1]
        prob = _Problem(pb.nelx, pb.nely, pb.nelz, pb.el, pb.eh, pb.ew, pb.E, pb.nu, p, emin, mr_n, opfilter, rmin,
                        fdp, fd1.size, None, 0, None, 0)
        if fixed_dens is not None and len(fixed_dens):
            fx1, fxp = _i64(np.asarray(fixed_dens) + 1)
            self._keep.append(fx1)
            prob.fixed_dens, prob.nfixed_dens = fxp, fx1.size
        if free_dens_g is not None:
            fg1, fgp = _i64(np.asarray(free_dens_g) + 1)
            self._keep.append(fg1)
            prob.free_dens_g, prob.nfree_dens_g = fgp, fg1.size
        h = C.c_void_p()
        rc = _lib.tosp_create(C.byref(prob), C.byref(self.mg), precision, C.byref(h))
        if rc != TOSP_OK:
            raise TospError(rc, _lib.tosp_last_error(None).decode())
        self.h = h
        self.nfree = int(np.asarray(pb.freedofs).size)
        self.ndens = pb.nelem * mr_n ** 3
        self.nfull = 3 * pb.nnodes

    def close(self):
        if getattr(self, "h", None):
            _lib.tosp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, allow=(TOSP_OK,)):
        if rc not in allow:
            raise TospError(rc, _lib.tosp_last_error(self.h).decode())
        return rc

    def info(self):
        ng, nc, nb = C.c_int32(), C.c_int64(), C.c_int64()
        self._check(_lib.tosp_info(self.h, C.byref(ng), C.byref(nc), C.byref(nb)))
        return {"ngrids": ng.value, "ncoarse": nc.value, "device_bytes": nb.value}

    def stats(self):
        st = SolveStats()
        self._check(_lib.tosp_last_stats(self.h, C.byref(st)))
        return {"it": st.it, "relres": st.relres, "ms_setup": st.ms_setup, "ms_solve": st.ms_solve,
                "replacements": st.replacements}

    # -- reference entry points ------------------------------------------------
    def SetupGMG(self, xfil):
        """Densities -> K(rho) and the multigrid hierarchy (GlobalStiffMatrix +
        SetupGMG / SetupGMGWOK)."""
        n = self.ndens
        if isinstance(xfil, np.ndarray):
            xfil = np.ascontiguousarray(xfil, dtype=np.float64)
            assert xfil.size == n
        self._check(_lib.tosp_setup_gmg(self.h, _ptr(xfil), n))

    def KelemProd(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._check(_lib.tosp_kelem_prod(self.h, _ptr(x), _ptr(y), x.size))
        return y

    def KelemProdMixed(self, x):
        """K(rho) x by the mixed V-cycle's finest operator (FP32 vectors, BF16
        SIMP factors; tensor-core sub-cell products when n * nely is even)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._check(_lib.tosp_kelem_prod_mixed(self.h, _ptr(x), _ptr(y), x.size))
        return y

    def KelemProdCG32(self, x):
        """K(rho) x by the CG's product of ``mg.cg_product = 1`` (tensor cores,
        FP32 SIMP factors and vectors)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._check(_lib.tosp_kelem_prod_cg32(self.h, _ptr(x), _ptr(y), x.size))
        return y

    def MGCycle(self, r):
        """One VCycle/WCycle/FMVCycle application s = M^{-1} r (free dofs)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        s = np.empty_like(r)
        self._check(_lib.tosp_mg_cycle(self.h, _ptr(r), _ptr(s), r.size))
        return s

    def SolveMG(self, x, f):
        """``[x, it] = SolveMG(x, f, ...)``: returns (x, it, relres, status)."""
        x = np.array(x, dtype=np.float64, copy=True)
        f = np.ascontiguousarray(f, dtype=np.float64)
        it, rr = C.c_int32(), C.c_double()
        rc = self._check(_lib.tosp_solve_mg(self.h, _ptr(x), _ptr(f), x.size, C.byref(it), C.byref(rr)),
                         allow=(TOSP_OK, TOSP_NOT_CONVERGED))
        return x, it.value, rr.value, rc

    def Grad(self, u_full, return_unfiltered=False):
        u = np.ascontiguousarray(u_full, dtype=np.float64)
        g = np.empty(self.ndens)
        g0 = np.empty(self.ndens) if return_unfiltered else None
        self._check(_lib.tosp_grad(self.h, _ptr(u), u.size, _ptr(g), _ptr(g0) if g0 is not None else None,
                                   self.ndens))
        return (g, g0) if return_unfiltered else g

    def ApplyFilter(self, x, trans=False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._check(_lib.tosp_apply_filter(self.h, _ptr(x), _ptr(y), x.size, 1 if trans else 0))
        return y

    def FilterWeights(self):
        w = np.empty(self.ndens)
        self._check(_lib.tosp_filter_weights(self.h, _ptr(w), self.ndens))
        return w

    def Compliance(self, f, u):
        f = np.ascontiguousarray(f, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        F = C.c_double()
        self._check(_lib.tosp_compliance(self.h, _ptr(f), _ptr(u), f.size, C.byref(F)))
        return F.value

    def time_operator(self, precision=PREC_FP64, reps=10):
        """Mean device time (ms) of one finest-level operator kernel launch."""
        ms = C.c_double()
        self._check(_lib.tosp_time_operator(self.h, precision, reps, C.byref(ms)))
        return ms.value

    def SetFreedofs(self, freedofs):
        fd1, fdp = _i64(np.asarray(freedofs) + 1)
        self._check(_lib.tosp_set_freedofs(self.h, fdp, fd1.size))
        self.nfree = fd1.size


class FallbackSolver:
    """The mixed-precision solve path with an FP64 fallback, for designs whose
    contrast the FP32 V-cycle cannot resolve.

    Same entry points as :class:`Solver`.  A mixed ``SolveMG`` that stalls
    (relative residual not halved in ``maxstall`` iterations), runs out of
    iterations or breaks down is finished by an FP64 solve (second handle, same
    problem and multigrid parameters) started from the mixed iterate; the
    returned iteration count is the sum of both.  After ``sticky`` fallbacks
    the FP64 path serves every later solve (an SLP design only gets crisper),
    so ``SetupGMG`` then builds only the FP64 hierarchy.  ``Grad``,
    ``ApplyFilter`` and ``Compliance`` are FP64 in both handles and run on the
    one holding the current densities.
    """

    def __init__(self, pb, mg=None, mr_n=1, p=3.0, emin=1e-9, opfilter=1, rmin=1.5, maxstall=100, sticky=1,
                 **kw):
        mg = mg if mg is not None else default_mg()
        mgm = MgParams.from_buffer_copy(mg)
        mgm.maxstall = maxstall
        mgm.flexible = 1
        mg64 = MgParams.from_buffer_copy(mg)
        mg64.maxstall = 0
        mg64.flexible = 0
        mg64.cg_product = 0      # the FP64 handle's CG product is FP64
        self._args = dict(mr_n=mr_n, p=p, emin=emin, opfilter=opfilter, rmin=rmin, **kw)
        self.pb, self._mg64, self.sticky = pb, mg64, sticky
        self.mixed = Solver(pb, mgm, precision=PREC_MIXED, **self._args)
        self.fp64 = None
        self.fallbacks = 0
        self.use_fp64 = False
        self._x = None           # densities of the last SetupGMG
        self._fp64_ready = False

    def _fp64(self):
        if self.fp64 is None:
            self.fp64 = Solver(self.pb, self._mg64, precision=PREC_FP64, **self._args)
        if not self._fp64_ready:
            self.fp64.SetupGMG(self._x)
            self._fp64_ready = True
        return self.fp64

    def _active(self):
        return self._fp64() if self.use_fp64 else self.mixed

    def close(self):
        self.mixed.close()
        if self.fp64 is not None:
            self.fp64.close()

    def SetupGMG(self, xfil):
        self._x = np.array(xfil, dtype=np.float64, copy=True)
        self._fp64_ready = False
        self._active().SetupGMG(self._x)

    def SolveMG(self, x, f):
        it0 = 0
        if not self.use_fp64:
            try:
                u, it, rr, rc = self.mixed.SolveMG(x, f)
            except TospError as e:
                if e.code != TOSP_ERR_BREAKDOWN:
                    raise
                u, it, rc = np.array(x, dtype=np.float64, copy=True), 0, e.code
            if rc == TOSP_OK:
                return u, it, rr, rc
            self.fallbacks += 1
            x, it0 = u, it
            if self.fallbacks >= self.sticky:
                self.use_fp64 = True
        u, it, rr, rc = self._fp64().SolveMG(x, f)
        return u, it0 + it, rr, rc

    def Grad(self, u_full, return_unfiltered=False):
        return self._active().Grad(u_full, return_unfiltered=return_unfiltered)

    def ApplyFilter(self, x, trans=False):
        return self.mixed.ApplyFilter(x, trans=trans)

    def Compliance(self, f, u):
        return self.mixed.Compliance(f, u)


def _problem_struct(pb, mr_n, p, emin, opfilter, rmin, fixed_dens=None, free_dens_g=None):
    """tosp_problem for `pb` plus the arrays it points to (keep them alive)."""
    keep = []
    fd1, fdp = _i64(np.asarray(pb.freedofs) + 1)
    keep.append(fd1)
    prob = _Problem(pb.nelx, pb.nely, pb.nelz, pb.el, pb.eh, pb.ew, pb.E, pb.nu, p, emin, mr_n, opfilter, rmin,
                    fdp, fd1.size, None, 0, None, 0)
    if fixed_dens is not None and len(fixed_dens):
        fx1, fxp = _i64(np.asarray(fixed_dens) + 1)
        keep.append(fx1)
        prob.fixed_dens, prob.nfixed_dens = fxp, fx1.size
    if free_dens_g is not None:
        fg1, fgp = _i64(np.asarray(free_dens_g) + 1)
        keep.append(fg1)
        prob.free_dens_g, prob.nfree_dens_g = fgp, fg1.size
    return prob, keep


class Server:
    """The serving loop of tosp.h: admission by slots and HBM budget,
    concurrent requests on their own streams, handles cached per shape."""

    def __init__(self, max_slots=4, hbm_budget_bytes=64 << 30):
        h = C.c_void_p()
        rc = _lib.tosp_server_create(max_slots, int(hbm_budget_bytes), C.byref(h))
        if rc != TOSP_OK:
            raise TospError(rc, "tosp_server_create")
        self.h = h
        self.meta = {}

    def submit(self, pb, xfil, f=None, mg=None, precision=PREC_MIXED, mr_n=1, p=3.0, emin=1e-9, opfilter=1,
               rmin=1.5):
        mg = mg if mg is not None else default_mg()
        prob, keep = _problem_struct(pb, mr_n, p, emin, opfilter, rmin)
        xfil = np.ascontiguousarray(xfil, dtype=np.float64)
        f = np.ascontiguousarray(pb.f if f is None else f, dtype=np.float64)
        rid = C.c_int64()
        rc = _lib.tosp_server_submit(self.h, C.byref(prob), C.byref(mg), precision, xfil.ctypes.data, xfil.size,
                                     f.ctypes.data, f.size, C.byref(rid))
        if rc != TOSP_OK:
            raise TospError(rc, "tosp_server_submit")
        self.meta[rid.value] = (f.size, xfil.size)
        return rid.value

    def prepare(self, pb, count=1, mg=None, precision=PREC_MIXED, mr_n=1, p=3.0, emin=1e-9, opfilter=1, rmin=1.5):
        """Create `count` idle handles for the problem's shape ahead of its
        requests."""
        mg = mg if mg is not None else default_mg()
        prob, keep = _problem_struct(pb, mr_n, p, emin, opfilter, rmin)
        rc = _lib.tosp_server_prepare(self.h, C.byref(prob), C.byref(mg), precision, count)
        if rc != TOSP_OK:
            raise TospError(rc, "tosp_server_prepare")

    def state(self, rid):
        st = C.c_int32()
        rc = _lib.tosp_server_poll(self.h, rid, C.byref(st))
        if rc != TOSP_OK:
            raise TospError(rc, "tosp_server_poll")
        return st.value

    def wait(self, rid, timeout=600.0):
        rc = _lib.tosp_server_wait(self.h, rid, timeout)
        if rc != TOSP_OK:
            raise TospError(rc, "tosp_server_wait")

    def result(self, rid, release=True):
        nfree, ndens = self.meta[rid]
        u = np.empty(nfree)
        g = np.empty(ndens)
        st = RequestStats()
        rc = _lib.tosp_server_result(self.h, rid, u.ctypes.data, nfree, g.ctypes.data, ndens, C.byref(st))
        if rc < 0:
            raise TospError(rc, "request failed")
        if release:
            _lib.tosp_server_release(self.h, rid)
            self.meta.pop(rid, None)
        return u, g, {"it": st.it, "relres": st.relres, "ms_latency": st.ms_latency, "ms_queue": st.ms_queue,
                      "ms_run": st.ms_run, "precision": st.precision, "status": rc}

    def cancel(self, rid):
        return _lib.tosp_server_cancel(self.h, rid)

    def info(self):
        a, q, b, c = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        _lib.tosp_server_info(self.h, C.byref(a), C.byref(q), C.byref(b), C.byref(c))
        return {"active": a.value, "queued": q.value, "used_bytes": b.value, "cached_handles": c.value}

    def counters(self):
        t, b, m = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.tosp_server_counters(self.h, C.byref(t), C.byref(b), C.byref(m))
        return {"ticks": t.value, "batched_iterations": b.value, "max_batch": m.value}

    def close(self):
        if getattr(self, "h", None):
            _lib.tosp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
