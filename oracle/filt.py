"""Oracle (test infrastructure only): density filter and sensitivities.

Restates
  * ``I/ElemNeighborhood.m:93-181`` -> :func:`elem_neighborhood`
  * ``I/ApplyFilter.m:74-81``       -> :func:`apply_filter`
  * ``I/Grad.m:18-62``              -> :func:`grad`
"""
import math

import numpy as np
import scipy.sparse as sp

from .fem import dof_table, density_table


def filter_offsets(rmin, el, eh, ew, opfilter):
    """Neighbour offsets and weights inside the filter radius.

    I/ElemNeighborhood.m:93-122: per z-offset ``relx = floor(sqrt(rmin^2-dz^2)/el)``,
    per (z, x)-offset ``rely = floor(sqrt(rmin^2-dz^2-dx^2)/eh)``; Gaussian weight
    ``exp(-d^2/(2 (rmin/3)^2)) / (2 pi rmin/3)`` (opfilter 1) or hat
    ``(rmin-d)/rmin`` (opfilter 2).  Returns a list of (dx, dy, dz, weight)
    covering all signs; the zero offset carries ``beta`` (or 1).
    """
    frz = math.floor(rmin / ew)
    rmin2 = rmin ** 2
    if opfilter == 1:
        alpha = 1 / (2 * ((rmin / 3) ** 2))
        beta = 1 / (2 * math.pi * (rmin / 3))
    out = []
    for kz in range(frz + 1):
        dz2 = (kz * ew) ** 2
        dxm = math.floor(math.sqrt(rmin2 - dz2) / el)
        for ix in range(dxm + 1):
            dx2 = (ix * el) ** 2
            dym = math.floor(math.sqrt(rmin2 - dz2 - dx2) / eh)
            for jy in range(dym + 1):
                if opfilter == 1:
                    wt = math.exp(-(dz2 + dx2 + (jy * eh) ** 2) * alpha) * beta
                else:
                    wt = (rmin - math.sqrt(dz2 + dx2 + (jy * eh) ** 2)) / rmin
                if kz == 0 and ix == 0 and jy == 0:
                    wt = beta if opfilter == 1 else 1.0   # :143-147
                for sz in ((1, -1) if kz else (1,)):
                    for sx in ((1, -1) if ix else (1,)):
                        for sy in ((1, -1) if jy else (1,)):
                            out.append((sx * ix, sy * jy, sz * kz, wt))
    return out


def elem_neighborhood(nelx, nely, nelz, el, eh, ew, rmin, opfilter, fixed=None):
    """Filter matrix W and row sums w (I/ElemNeighborhood.m:93-181).

    ``fixed``: 0-based indices of elements with fixed densities; their rows
    and columns are decoupled with a unit diagonal (:173-179).
    """
    nel = nelx * nely * nelz
    ez, ex, ey = np.meshgrid(np.arange(nelz), np.arange(nelx), np.arange(nely), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    e1 = np.arange(nel)
    rows, cols, vals = [], [], []
    for dx, dy, dz, wt in filter_offsets(rmin, el, eh, ew, opfilter):
        x2, y2, z2 = ex + dx, ey + dy, ez + dz
        ok = (x2 >= 0) & (x2 < nelx) & (y2 >= 0) & (y2 < nely) & (z2 >= 0) & (z2 < nelz)
        rows.append(e1[ok])
        cols.append((z2[ok] * nelx + x2[ok]) * nely + y2[ok])
        vals.append(np.full(ok.sum(), wt))
    W = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nel, nel)).tocsr()
    if fixed is not None and len(fixed):
        keep = np.ones(nel)
        keep[fixed] = 0.0
        Dk = sp.diags(keep)
        W = Dk @ W @ Dk
        W = W + sp.diags(1.0 - keep)
        W = W.tocsr()
    w = np.asarray(W.sum(axis=1)).ravel()
    return W, w


def apply_filter(x, W, w, opfilter, trans):
    """I/ApplyFilter.m:74-81."""
    if opfilter == 0:
        return x.copy()
    if trans:
        return W.T @ (x / w)
    return (W @ x) / w


def grad(nelx, nely, nelz, ks, u_full, dens, p, emin, W, w, opfilter, free_elems=None, E=1.0):
    """Compliance sensitivities, then the transposed filter (I/Grad.m:18-62).

    ``u_full``: displacement on all 3*nnodes dofs; ``dens``: filtered
    densities on the density mesh; ``free_elems``: 0-based displacement
    elements of ``str.freeDensG`` (None = all).  Uses ``mr.interp = false``
    (I/Grad.m:45-49).
    """
    n = round(len(ks) ** (1 / 3))
    dofs = dof_table(nelx, nely, nelz)
    didx = density_table(nelx, nely, nelz, n)
    if free_elems is not None:
        dofs, didx = dofs[free_elems], didx[free_elems]
    ue = u_full[dofs]
    g0 = np.zeros(dens.size)
    for s in range(len(ks)):
        q = np.einsum("ei,ij,ej->e", ue, ks[s], ue)
        xs = dens[didx[:, s]]
        g0[didx[:, s]] = -p * np.power(xs, p - 1) * (E - emin) * q
    return apply_filter(g0, W, w, opfilter, True), g0
