"""Sequential linear programming driver (host) on top of the GPU solve path.

Restates the trust-region SLP loop of ``I/StrSLP.m:46-560`` (``I/`` =
``Implementation/``) for the configuration the solve path serves
(matrix-free geometric MG, ``mr.n = mr.d``, ``elem.fix = 0``): per step it
solves the LP subproblem on the host, filters the new design, rebuilds K(rho)
and the hierarchy, solves K u = f with the previous u as warm start
(``pcgp.opu0``), and on acceptance recomputes the sensitivities.  The final
optional rounding is ``GradProj`` (``I/GradProj.m``).

The solve path is any object with ``ApplyFilter(x, trans)``, ``SetupGMG(xfil)``,
``SolveMG(x0, f) -> (u, it, relres, status)`` and ``Grad(u_full)`` -
:class:`tosp.Solver` on the GPU.

LP solvers: ``"highs"`` - ``scipy.optimize.linprog(method="highs-ds")``, the
dual simplex like the reference's ``linprog`` (``I/StrSLP.m:239-245,267-290``);
``"knapsack"`` - the exact solution of this LP (one inequality with positive
coefficients plus bounds) by sorting the cost/coefficient ratios, O(N log N).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class SlpParams:
    """``slp.*`` of I/TopOpt3D.m:61-72."""
    tolS: float = 1e-4
    tolG: float = 1e-3
    tolF: float = 5e-2
    maxcount: int = 3
    maxiter: int = 500
    delta0: float = 0.1
    eta: float = 0.1
    rho: float = 0.5
    alphaR: float = 0.25
    alphaA: float = 2.0
    lp: str = "highs"


@dataclass
class PrjParams:
    """``prj.*`` of I/TopOpt3D.m:73-92 used by GradProj."""
    op: bool = False
    nearlim: bool = True
    maxang: float = 89.9
    gthresh: float = 1e-4
    ut: float = 0.95
    lt: float = 0.05
    vumin: float = 0.7
    vlmax: float = 0.3
    heavi: bool = True
    eta: float = 0.25
    beta: float = 1.0
    dbeta: float = 2.0
    betamax: float = 1000.0


@dataclass
class SlpResult:
    xstar: np.ndarray
    x: np.ndarray
    u: np.ndarray
    F: float
    iters: int
    rejected: int
    opstop: int
    pcgit: list = field(default_factory=list)
    history: list = field(default_factory=list)
    pcgstatus: list = field(default_factory=list)   # SolveMG status of every solve (0: converged)


def _threshold_ratio(ratio, red, excess):
    """Smallest candidate ratio r with sum(red[ratio <= r]) >= excess, by a
    weighted quickselect (linear time; no full sort).  A sample first brackets
    the answer so that the selection runs on a small subset."""
    r, w = ratio, red
    offset = 0.0
    if r.size > 200000:
        rng = np.random.default_rng(12345)
        smp = rng.choice(r.size, 20000, replace=False)
        sr, sw = r[smp], w[smp]
        o = np.argsort(sr)
        cw = np.cumsum(sw[o]) * (float(w.sum()) / float(sw.sum()))
        j = int(np.searchsorted(cw, excess))
        lo_b = sr[o[max(j - 400, 0)]] if j - 400 >= 0 else -np.inf
        hi_b = sr[o[min(j + 400, o.size - 1)]] if j + 400 < o.size else np.inf
        s_below = float(np.sum(w, where=r < lo_b))
        mid = (r >= lo_b) & (r <= hi_b)
        s_mid = float(np.sum(w, where=mid))
        if s_below < excess <= s_below + s_mid:
            r, w, offset = r[mid], w[mid], s_below
    while True:
        if r.size == 0:                 # round-off in the running sums
            return float(ratio.max())
        pivot = np.partition(r, r.size // 2)[r.size // 2]
        lt = r < pivot
        s_lt = float(w[lt].sum())
        if offset + s_lt >= excess and s_lt > 0.0:
            r, w = r[lt], w[lt]
            continue
        eq = r == pivot
        s_eq = float(w[eq].sum())
        if offset + s_lt + s_eq >= excess:
            return pivot
        offset += s_lt + s_eq
        gt = ~(lt | eq)
        r, w = r[gt], w[gt]


def lp_knapsack(g, a, c, lo, hi, rtol=1e-9):
    """min g's  s.t.  a's <= c, lo <= s <= hi  with a > 0.

    Returns (s, fval, lam, ok): start from the unconstrained minimiser
    (hi where g < 0, lo elsewhere); if a's > c, lower the variables that cost
    least per unit of constraint (smallest |g|/a among g < 0) until a's = c.
    Candidates whose ratios differ by at most rtol (relative, chained) form one
    group that moves by a common fraction, so the step does not depend on
    round-off between mirror-symmetric elements.  lam is the multiplier of the
    inequality (>= 0, MATLAB's lambda.ineqlin).

    The threshold ratio is found by weighted selection; only the candidates in
    a narrow window around it are sorted to form the groups.
    """
    s = np.where(g < 0, hi, lo).astype(np.float64)
    excess = a @ s - c
    if excess <= 0:
        return s, float(g @ s), 0.0, True
    candm = (g < 0) & (hi > lo)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(candm, -g / a, np.inf)       # cost per unit of constraint
    red = np.where(candm, a * (hi - lo), 0.0)          # reduction if moved fully to lo
    if not candm.any() or float(red.sum()) < excess:
        return None, None, None, False                # infeasible within the box
    cand = np.nonzero(candm)[0]
    rstar = _threshold_ratio(ratio[cand], red[cand], excess)
    width = 1e-3
    while True:
        lo_r, hi_r = rstar * (1 - width), rstar * (1 + width)
        w_idx = np.nonzero((ratio >= lo_r) & (ratio <= hi_r))[0]
        w_idx = w_idx[np.argsort(ratio[w_idx], kind="stable")]
        wr = ratio[w_idx]
        # groups chain by gaps <= rtol; a chain reaching the window edge could
        # continue outside it, so widen the window then
        gaps_ok = wr[1:] - wr[:-1] > rtol * np.abs(wr[1:])
        edge_lo = wr[0] - lo_r <= rtol * abs(wr[0])
        edge_hi = hi_r - wr[-1] <= rtol * abs(hi_r)
        if not (edge_lo or edge_hi) or width >= 1.0:
            break
        width = min(1.0, width * 10)
    below = ratio < lo_r
    offset = float(np.sum(red, where=below))
    newgrp = np.ones(wr.size, dtype=bool)
    newgrp[1:] = gaps_ok
    gid = np.cumsum(newgrp) - 1
    gred = np.bincount(gid, weights=red[w_idx])
    gcum = offset + np.cumsum(gred)
    k = min(int(np.searchsorted(gcum, excess)), gred.size - 1)
    grp_sel = gid == k
    gmin = wr[grp_sel][0]
    done = ratio < gmin                               # every earlier group moves fully to lo
    s = np.where(done, lo, s)
    prev = gcum[k - 1] if k > 0 else offset
    frac = (excess - prev) / gred[k]
    grp = w_idx[grp_sel]
    s[grp] = hi[grp] - frac * (hi[grp] - lo[grp])
    lam = float(np.mean(wr[grp_sel]))
    return s, float(g @ s), lam, True


def lp_highs(g, a, c, lo, hi):
    from scipy.optimize import linprog
    res = linprog(g, A_ub=a[None, :], b_ub=[c], bounds=np.stack([lo, hi], axis=1), method="highs-ds")
    if res.status != 0:
        return None, None, None, False, 0
    lam = float(-res.ineqlin.marginals[0]) if res.ineqlin is not None else 0.0
    return res.x, float(res.fun), lam, True, int(res.nit)


def _heav_root(eta, beta, x, velem, s):
    """Volume of the projected densities minus s (I/HeavRoot.m)."""
    c = np.tanh(beta * eta)
    d = 1.0 / (c + np.tanh(beta * (1.0 - eta)))
    return float(velem @ ((c + np.tanh(beta * (x - eta))) * d)) - s


def heaviside_proj(x, prj, velem, scur, sdes, betaupd):
    """Volume-preserving smooth Heaviside projection (I/HeavisideProj.m:1-40).

    Optionally raises beta (times dbeta, capped at betamax); finds eta in
    [0, 1] with the projected volume equal to sdes (moving the target towards
    scur in 20 steps while f(0) f(1) > 0); returns (xstar, prj) with prj's eta
    and beta updated.  MATLAB's fzero is replaced by Brent's method on [0, 1].
    """
    from scipy.optimize import brentq
    x = np.asarray(x, dtype=np.float64)
    if betaupd:
        prj.beta = min(prj.beta * prj.dbeta, prj.betamax)
    s = sdes
    f0 = _heav_root(0.0, prj.beta, x, velem, s)
    f1 = _heav_root(1.0, prj.beta, x, velem, s)
    i = 0
    while f0 * f1 > 0 and i < 20:
        i += 1
        s = scur * (i / 20.0) + sdes * (1 - i / 20.0)
        f0 = _heav_root(0.0, prj.beta, x, velem, s)
        f1 = _heav_root(1.0, prj.beta, x, velem, s)
    if f0 == 0.0:
        prj.eta = 0.0
    elif f1 == 0.0:
        prj.eta = 1.0
    else:
        prj.eta = brentq(lambda e: _heav_root(e, prj.beta, x, velem, s), 0.0, 1.0, xtol=1e-14, rtol=1e-15)
    c = np.tanh(prj.beta * prj.eta)
    cd = 1.0 / (c + np.tanh(prj.beta * (1.0 - prj.eta)))
    return (c + np.tanh(prj.beta * (x - prj.eta))) * cd, prj


def snap(v, scale=1.0):
    """``v`` rounded to multiples of 2^-30 * scale, scale raised to a power of
    two: values that agree up to the rounding of two solve paths (a GPU and a
    CPU one, or two runs with different atomic orders) become exactly equal,
    and ties then break by element index in the stable sorts."""
    q = 2.0 ** (np.ceil(np.log2(scale)) - 30) if scale > 0 else 2.0 ** -30
    return np.round(np.asarray(v, dtype=np.float64) / q) * q


def grad_proj(x, g, prj, Vmax, velem):
    """Rounding of the densities to 0/1 along -grad(Lag) (I/GradProj.m:1-124).

    Tie rule (not in the reference, which runs one solve path): x and g are
    snapped to 2^-30 of their scale first (:func:`snap`), so designs
    thresholded from the GPU path and from the CPU oracle are identical
    whenever the two inputs agree to rounding."""
    x = snap(x)
    g = np.asarray(g, dtype=np.float64)
    g = -snap(g, float(np.abs(g).max()))
    gnorm = np.linalg.norm(g)
    coslim = np.cos(np.deg2rad(prj.maxang))
    gt = prj.gthresh * np.abs(g).max()
    volfrac = (velem @ x) / velem.sum()
    xtop = np.nonzero(x >= prj.ut)[0]
    ntop = xtop.size
    done = int(np.round(Vmax / velem[0]))
    nup = done - ntop
    xnew = np.zeros(x.size)
    if nup <= 0:
        su = np.argsort(-x[xtop], kind="stable")
        xnew[xtop[su[:done]]] = 1.0
        return xnew
    xnew[xtop] = 1.0
    xvar = np.nonzero((x > prj.lt) & (x < prj.ut))[0]
    nvar = xvar.size
    if nvar == 0:
        return xnew
    dvol = min(nvar, nup, int(np.round(volfrac * x.size)) - ntop)

    def cos_of(xn):
        d = xn - x
        nd = np.linalg.norm(d)
        return (d @ g) / (gnorm * nd) if nd > 0 else -1.0

    if prj.nearlim:
        ivol = np.argsort(-x[xvar], kind="stable")
        xnew[xvar[ivol[:max(dvol, 0)]]] = 1.0
        cosang = cos_of(xnew)
    else:
        cosang = -1.0
    if cosang < coslim:
        gv = g[xvar].copy()
        iup = np.nonzero(gv > 0.0)[0]
        iup2 = np.nonzero((gv == 0.0) & (x[xvar] >= prj.vumin))[0]
        g[xvar[iup2]] = 1e16
        gv = g[xvar]
        iup = np.concatenate([iup, iup2])
        niup = iup.size
        idown = np.nonzero(gv < -gt)[0]
        nidown = idown.size
        alphau = (1 - x[xvar[iup]]) / gv[iup]
        alphad = -x[xvar[idown]] / gv[idown]
        su = np.argsort(alphau, kind="stable")
        sd = np.argsort(alphad, kind="stable")
        alphau, alphad = alphau[su], alphad[sd]
        xup = x[xvar[iup[su]]]
        xdown = x[xvar[idown[sd]]]
        ku = np.nonzero(xup < prj.vumin)[0]
        kup = niup if ku.size == 0 else int(ku[0])
        kd = np.nonzero(xdown > prj.vlmax)[0]
        kdown = nidown if kd.size == 0 else int(kd[0])
        if niup == 0:
            if nidown == 0:
                return xnew
            alpha = alphad[:kdown]
        else:
            imax = min(dvol, kup)
            if nidown == 0:
                alpha = alphau[:imax]
            elif imax == 0:
                alpha = alphad[:kdown]
            else:
                i2 = np.nonzero(alphad > alphau[imax - 1])[0]
                imax2 = kdown if i2.size == 0 else min(kdown, int(i2[0]))
                alpha = np.sort(np.concatenate([alphau[:imax], alphad[:imax2]]))
        pos = alpha.size - 1
        while pos >= 0 and cosang < coslim:
            xnew[xvar] = np.maximum(0.0, np.minimum(1.0, x[xvar] + alpha[pos] * g[xvar]))
            cosang = cos_of(xnew)
            pos -= 1
        if cosang < coslim:
            xnew[xvar] = x[xvar]
    return xnew


def str_slp(solver, pb, volfrac, x0, slp=None, prj=None, fixed=None, on_iter=None):
    """Trust-region SLP of I/StrSLP.m with ``volineq = true`` and MG solves.

    ``solver``: the solve path (see the module docstring); ``pb`` the problem
    (free dofs and loads); ``x0`` the initial design variables on the
    density (= design) mesh; ``fixed``: 0-based fixed design variables.
    """
    slp = slp or SlpParams()
    prj = prj or PrjParams()
    x = np.asarray(x0, dtype=np.float64).copy()
    nelem = x.size
    V = pb.l * pb.h * pb.w
    velem = np.full(nelem, V / nelem)
    Vmax = volfrac * V
    fixed = np.zeros(0, dtype=np.int64) if fixed is None else np.asarray(fixed, dtype=np.int64)
    free = np.setdiff1d(np.arange(nelem), fixed)
    theta1 = theta2 = thetaMax = 1.0
    countS = countG = countF = 0
    it_acc = itrej = 0
    delta = slp.delta0
    res = SlpResult(None, None, None, 0.0, 0, 0, 2)

    xfil = solver.ApplyFilter(x)
    solver.SetupGMG(xfil)
    u, pit, _, pst = solver.SolveMG(np.zeros(pb.f.size), pb.f)
    res.pcgit.append(pit)
    res.pcgstatus.append(pst)
    Fold = float(pb.f @ u)
    F = Fold
    ufull = np.zeros(3 * pb.nnodes)
    ufull[pb.freedofs] = u
    Fgrad = solver.Grad(ufull)
    A = solver.ApplyFilter(velem, trans=True) / Vmax          # I/StrSLP.m:222-228
    b = (velem @ xfil - Vmax) / Vmax
    sL = np.maximum(-delta, -x)
    sU = np.minimum(delta, 1 - x)
    sL[fixed] = 0.0
    sU[fixed] = 0.0
    lam = 0.0
    gp = np.minimum(1, np.maximum(0.0, x[free] - Fgrad[free])) - x[free]
    gpnorm = np.abs(gp).max() if gp.size else 0.0
    if gpnorm < 1e-12 and b < 1e-12 and (x - 1.0).max() < 1e-12 and x.min() > -1e-12:
        countG = countF = slp.maxcount

    while (countG < slp.maxcount or countF < slp.maxcount) and countS < slp.maxcount and it_acc < slp.maxiter:
        if slp.lp == "knapsack":
            s, fval, lam_new, ok = lp_knapsack(Fgrad, A, -b, sL, sU)
            nit = 1
        else:
            s, fval, lam_new, ok, nit = lp_highs(Fgrad, A, -b, sL, sU)
        if not ok:
            # infeasible step box: minimise the infeasibility (I/StrSLP.m:272-286)
            from scipy.optimize import linprog
            A2 = np.concatenate([A, [-1.0, 1.0]])
            c2 = np.concatenate([np.zeros(nelem), [1.0, 1.0]])
            lo2 = np.concatenate([np.maximum(-0.8 * delta, -x), [0.0, 0.0]])
            hi2 = np.concatenate([np.minimum(0.8 * delta, 1 - x), [np.inf, np.inf]])
            lo2[fixed] = 0.0
            hi2[fixed] = 0.0
            r2 = linprog(c2, A_ub=A2[None, :], b_ub=[-b], bounds=np.stack([lo2, hi2], axis=1), method="highs-ds")
            s = r2.x[:nelem]
            fval = float(Fgrad @ s)
            lam_new = float(-r2.ineqlin.marginals[0])
        elif nit == 0:
            s = np.zeros(nelem)
        lam = lam_new
        snorm = np.abs(s).max()
        xold, bold, deltaold = x, b, delta
        x = x + s
        xfil = solver.ApplyFilter(x)
        b = (velem @ xfil - Vmax) / Vmax
        solver.SetupGMG(xfil)
        u, pit, _, pst = solver.SolveMG(u, pb.f)              # warm start, pcgp.opu0
        res.pcgit.append(pit)
        res.pcgstatus.append(pst)
        F = float(pb.f @ u)
        predopt = -fval
        predfsb = abs(bold) - abs(A @ s + bold)
        aredopt = Fold - F
        aredfsb = abs(bold) - abs(b)
        thetaMin = min(theta1, theta2)
        thetaLarge = (1 + 1e6 / ((it_acc + 1) ** 1.1)) * thetaMin
        thetaSup = 1.0 if predopt > 0.5 * predfsb else (0.5 * predfsb) / (predfsb - predopt)
        theta = min(thetaLarge, thetaSup, thetaMax)
        theta2, theta1 = theta1, theta
        pred = theta * predopt + (1 - theta) * predfsb
        ared = theta * aredopt + (1 - theta) * aredfsb
        if ared < slp.eta * pred:                               # rejected
            itrej += 1
            delta = max(slp.alphaR * snorm, 0.1 * deltaold)
            thetaMax = theta
            x, b, F = xold, bold, Fold
        else:                                                   # accepted
            if ared >= slp.rho * pred:
                delta = min(slp.alphaA * deltaold, 1.0)
            delta = max(delta, 0.0001)
            thetaMax = 1.0
            Fold = F
            ufull = np.zeros(3 * pb.nnodes)
            ufull[pb.freedofs] = u
            Fgrad = solver.Grad(ufull)
            Lgrad = Fgrad[free] + lam * A[free]
            gp = np.minimum(1, np.maximum(0.0, x[free] - Lgrad)) - x[free]
            gpnorm = np.abs(gp).max() if gp.size else 0.0
            it_acc += 1
            countG = countG + 1 if gpnorm <= slp.tolG else 0
            countF = countF + 1 if ared <= slp.tolF else 0
        countS = countS + 1 if snorm <= slp.tolS else 0
        sL = np.maximum(-delta, -x)
        sU = np.minimum(delta, 1 - x)
        sL[fixed] = 0.0
        sU[fixed] = 0.0
        res.history.append({"it": it_acc, "F": F, "ared": ared, "pred": pred, "snorm": snorm, "delta": deltaold,
                            "gpnorm": gpnorm, "pcgit": pit})
        if on_iter:
            on_iter(res.history[-1])

    if countG >= slp.maxcount and countF >= slp.maxcount:
        res.opstop = 0
    elif countS >= slp.maxcount:
        res.opstop = 1
    else:
        res.opstop = 2
    if prj.op:
        # rounding to 0/1 (I/StrSLP.m:566-592): optional volume-preserving
        # Heaviside projection, sensitivities at the projected densities, GradProj
        if prj.heavi:
            vcur = float(velem @ xfil)
            xfil, prj = heaviside_proj(xfil, prj, velem, vcur, vcur, False)
            solver.SetupGMG(xfil)
            ufull = np.zeros(3 * pb.nnodes)
            ufull[pb.freedofs] = u
            Fgrad = solver.Grad(ufull)
            A = velem / Vmax
        res.xstar = grad_proj(xfil, Fgrad + lam * A, prj, Vmax, velem)
    else:
        res.xstar = xfil
    res.x, res.u, res.F, res.iters, res.rejected = x, u, F, it_acc, itrej
    return res


def density_mesh_problem(pb, n):
    """The problem on the density mesh (n times finer), built from the same
    support/load rows (the ``strT`` of I/ExtraResults.m for CorrectFunctionValue)."""
    from . import problems
    if pb.supp is None or pb.loads is None:
        raise ValueError("the problem needs its support/load rows to be rebuilt on the density mesh")
    return problems.build(pb.nelx * n, pb.nely * n, pb.nelz * n, pb.supp, pb.loads, el=pb.el / n, eh=pb.eh / n,
                          ew=pb.ew / n, E=pb.E, nu=pb.nu)


def correct_function_value(pb, n, xstar, mg=None, precision=0, p=3.0, emin=1e-9):
    """``Ftrue`` of I/CorrectFunctionValue.m:1-58: the compliance of the
    multiresolution design re-solved with one displacement element per density
    element (no multiresolution), on the GPU solve path."""
    from . import Solver, default_mg
    strT = density_mesh_problem(pb, n)
    s = Solver(strT, mg if mg is not None else default_mg(), precision=precision, mr_n=1, p=p, emin=emin,
               opfilter=0, rmin=1.0)
    s.SetupGMG(np.asarray(xstar, dtype=np.float64))
    u, it, rr, rc = s.SolveMG(np.zeros(strT.f.size), strT.f)
    F = float(strT.f @ u)
    s.close()
    return F, it, rr
