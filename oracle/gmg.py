"""Oracle (test infrastructure only): geometric multigrid and MG-PCG.

Restates
  * ``I/Prolongation.m:15-55``        -> :func:`prolongation`
  * ``I/SetupGMG.m:16-77``            -> :func:`setup_gmg`
  * ``I/StartStrSLP.m:107-133``       -> :func:`gmg_levels`
  * ``I/Smooth.m:14-23``              -> :func:`smooth`
  * ``I/VCycle.m:23-43``, ``I/WCycle.m:23-44``, ``I/FMVCycle.m:22-39``
  * ``I/SolveMG.m:26-53``             -> :func:`solve_mg`

Substitution: MATLAB's ``amd`` + sparse ``chol`` of the coarsest matrix
(I/SetupGMG.m:51-59) is replaced by a dense LAPACK Cholesky
(``scipy.linalg.cho_factor``); the coarse solve ``R\\(R'\\rH(perm))`` is equal
up to rounding.
"""
import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp


def prolongation(nxf, nyf, nzf, nxc, nyc, nzc, freedofsf):
    """Trilinear P between vertex-nested grids (I/Prolongation.m:15-55).

    Returns ``(P, freedofsc)``: P restricted to rows ``freedofsf`` and columns
    ``freedofsc`` (0-based); a coarse dof is free when the fine dof at the same
    position is free (:38-46, :54).
    """
    w = np.array([1.0, 0.5, 0.25, 0.125])
    zc, xc, yc = np.meshgrid(np.arange(nzc), np.arange(nxc), np.arange(nyc), indexing="ij")
    zc, xc, yc = zc.ravel(), xc.ravel(), yc.ravel()
    col = (zc * nxc + xc) * nyc + yc
    rows, cols, vals = [], [], []
    for dz in (-1, 0, 1):
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                z, x, y = 2 * zc + dz, 2 * xc + dx, 2 * yc + dy
                ok = (z >= 0) & (z < nzf) & (x >= 0) & (x < nxf) & (y >= 0) & (y < nyf)
                row = (z * nxf + x) * nyf + y
                val = w[dx * dx + dy * dy + dz * dz]
                for comp in range(3):
                    rows.append(3 * row[ok] + comp)
                    cols.append(3 * col[ok] + comp)
                    vals.append(np.full(ok.sum(), val))
    nf, nc = 3 * nxf * nyf * nzf, 3 * nxc * nyc * nzc
    P = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nf, nc)).tocsr()
    # coincident fine dof of every coarse dof
    aux = (3 * (((2 * zc) * nxf + 2 * xc) * nyf + 2 * yc)[:, None] + np.arange(3)[None, :]).ravel()
    freemask_f = np.zeros(nf, dtype=bool)
    freemask_f[freedofsf] = True
    freedofsc = np.nonzero(freemask_f[aux])[0]
    return P[freedofsf][:, freedofsc].tocsr(), freedofsc


def gmg_levels(nelx, nely, nelz, ngrids, nmaxchol=60000, opchol=0):
    """Level-count rules of I/StartStrSLP.m:107-133.

    Returns ``(ngrids, opchol)`` or raises when geometric MG is impossible
    (the reference then falls back to AMG, which is out of scope).
    """
    def divisible(k):
        m = 2 ** (k - 1)
        return nelx % m == 0 and nely % m == 0 and nelz % m == 0
    ng = ngrids
    while not divisible(ng):
        ng -= 1
    if ng < 2:
        raise ValueError("geometric multigrid impossible for this mesh")
    if opchol == 0:
        while ((nelx / 2 ** (ng - 1) + 1) * (nely / 2 ** (ng - 1) + 1) * (nelz / 2 ** (ng - 1) + 1) * 3
               > nmaxchol and opchol == 0):
            m = 2 ** ng
            if nelx % m == 0 and nely % m == 0 and nelz % m == 0:
                ng += 1
            else:
                opchol = 1
    return ng, opchol


class Hierarchy:
    """The cell arrays ``A, P, M`` and the coarse factor of I/SetupGMG.m."""

    def __init__(self, A, P, Mdiag, chol, freedofs, omega, pcg=None):
        self.A, self.P, self.Mdiag, self.chol = A, P, Mdiag, chol
        self.freedofs, self.omega = freedofs, omega
        self.pcg = pcg   # (tolPCG, maxiterPCG) with opchol = 1, else None


def setup_gmg(K, nelx, nely, nelz, freedofs, ngrids, omega, opchol=0, tolPCG=1e-8, maxiterPCG=10000):
    """I/SetupGMG.m:16-77 with ``smoother = 0`` (Jacobi).

    ``M{i} = (1/omega) diag(A{i})`` is kept as its diagonal.  ``opchol = 1``
    solves the coarsest grid by PCG with the diagonal preconditioner
    (I/SetupGMG.m:52-57 with ``opcond = 0``, I/VCycle.m:28-35) instead of the
    Cholesky factor.
    """
    nel = [(nelx // 2 ** i, nely // 2 ** i, nelz // 2 ** i) for i in range(ngrids)]
    fd = [np.asarray(freedofs)]
    P = []
    for i in range(ngrids - 1):
        (ex, ey, ez), (cx, cy, cz) = nel[i], nel[i + 1]
        Pi, fdc = prolongation(ex + 1, ey + 1, ez + 1, cx + 1, cy + 1, cz + 1, fd[i])
        P.append(Pi)
        fd.append(fdc)
    A = [K.tocsr()]
    for i in range(1, ngrids):
        A.append((P[i - 1].T @ A[i - 1] @ P[i - 1]).tocsr())
    Mdiag = [A[i].diagonal() / omega for i in range(ngrids - 1)]
    if opchol == 1:
        return Hierarchy(A, P, Mdiag, None, fd, omega, pcg=(tolPCG, maxiterPCG))
    chol = sla.cho_factor(A[-1].toarray(), lower=False)
    return Hierarchy(A, P, Mdiag, chol, fd, omega)


def smooth(A, Mdiag, b, x0, niter):
    """Damped Jacobi ``x = x + M\\(b - A*x)`` (I/Smooth.m:14-18)."""
    x = x0.copy()
    for _ in range(niter):
        x = x + (b - A @ x) / Mdiag
    return x


def pcg_diag(A, b, tol, maxit):
    """MATLAB's ``pcg(A, b, tol, maxit, diag(diag(A)))`` from a zero iterate:
    preconditioned CG, stopped once ||r|| <= tol ||b|| or after maxit
    iterations (the last iterate is returned)."""
    d = A.diagonal()
    x = np.zeros(b.size)
    nb = np.linalg.norm(b)
    if nb == 0.0:
        return x
    r = b.copy()
    p = r / d
    rho = r @ p
    for _ in range(maxit):
        q = A @ p
        alpha = rho / (p @ q)
        x = x + alpha * p
        r = r - alpha * q
        if np.linalg.norm(r) <= tol * nb:
            break
        z = r / d
        rho_new = r @ z
        p = z + (rho_new / rho) * p
        rho = rho_new
    return x


def coarse_solve(H, rH):
    """``R\\(R'\\rH(perm))`` of I/VCycle.m:40 (dense Cholesky substitute), or
    with ``opchol = 1`` the coarsest PCG of I/VCycle.m:28-35."""
    if H.pcg is not None:
        return pcg_diag(H.A[-1], rH, H.pcg[0], H.pcg[1])
    return sla.cho_solve(H.chol, rH)


def vcycle(H, b, x0, nu1, nu2, nv=0):
    """I/VCycle.m:23-43 (0-based level ``nv``)."""
    ngrids = len(H.A)
    x = smooth(H.A[nv], H.Mdiag[nv], b, x0, nu1)
    rh = b - H.A[nv] @ x
    rH = H.P[nv].T @ rh
    if nv == ngrids - 2:
        eH = coarse_solve(H, rH)
    else:
        eH = vcycle(H, rH, np.zeros(rH.size), nu1, nu2, nv + 1)
    x = x + H.P[nv] @ eH
    return smooth(H.A[nv], H.Mdiag[nv], b, x, nu2)


def wcycle(H, b, x0, nu1, nu2, nv=0):
    """I/WCycle.m:23-44: two recursive calls, the second warm-started (:39-40)."""
    ngrids = len(H.A)
    x = smooth(H.A[nv], H.Mdiag[nv], b, x0, nu1)
    rh = b - H.A[nv] @ x
    rH = H.P[nv].T @ rh
    if nv == ngrids - 2:
        eH = coarse_solve(H, rH)
    else:
        eH = wcycle(H, rH, np.zeros(rH.size), nu1, nu2, nv + 1)
        eH = wcycle(H, rH, eH, nu1, nu2, nv + 1)
    x = x + H.P[nv] @ eH
    return smooth(H.A[nv], H.Mdiag[nv], b, x, nu2)


def fmvcycle(H, b, nu1, nu2, nv=0):
    """I/FMVCycle.m:22-39."""
    ngrids = len(H.A)
    rH = H.P[nv].T @ b
    if nv == ngrids - 2:
        x = coarse_solve(H, rH)
    else:
        x = fmvcycle(H, rH, nu1, nu2, nv + 1)
    x = H.P[nv] @ x
    return vcycle(H, b, x, nu1, nu2, nv)


def precondition(H, r, cycle, nu1, nu2):
    """One preconditioner application as dispatched in I/SolveMG.m:31-37."""
    if cycle == 0:
        return vcycle(H, r, np.zeros(r.size), nu1, nu2)
    if cycle == 1:
        return wcycle(H, r, np.zeros(r.size), nu1, nu2)
    if cycle == 2:
        return fmvcycle(H, r, nu1, nu2)
    raise ValueError("cycle must be 0, 1 or 2")


def solve_mg(H, x, f, cycle, nu1, nu2, tol, maxiter, apply_A=None, history=None):
    """MG-preconditioned CG of I/SolveMG.m:26-53.

    Returns ``(x, it)`` with the reference's counter convention (``it`` starts
    at 1 and is incremented once per iteration).  ``apply_A`` replaces the
    fine-level product (``KelemProd`` of I/WOK/SolveMGWOK.m:30,49).
    """
    Av = apply_A if apply_A is not None else (lambda v: H.A[0] @ v)
    x = x.copy()
    r = f - Av(x)
    nf = np.linalg.norm(f)
    nr = np.linalg.norm(r) / nf
    it = 1
    d = None
    gamma2 = None
    while nr > tol and it <= maxiter:
        s = precondition(H, r, cycle, nu1, nu2)
        rho = r @ s
        if it == 1:
            d = s
        else:
            d = (rho / gamma2) * d + s
        q = Av(d)
        alpha = rho / (d @ q)
        x = x + alpha * d
        r = r - alpha * q
        gamma2 = rho
        nr = np.linalg.norm(r) / nf
        it += 1
        if history is not None:
            history.append(nr)
    return x, it
