"""Oracle (test infrastructure only): element matrices, numbering and the
multiresolution stiffness operator.

Restates, for trilinear (hex8, ``elem.deg = 1``, Lagrange) elements:
  * ``I/ElemStiffMatrixGQMR.m:10-240``  -> :func:`elem_stiff_gqmr`
  * ``I/DegreesOfFreedom.m:19-54``      -> :func:`dof_table`
  * ``I/StartMR.m:58-83`` and ``I/GlobalStiffMatrix.m:33-47`` -> :func:`density_table`
  * ``I/GlobalStiffMatrix.m:16-65``     -> :func:`global_stiff_matrix`
  * ``I/WOK/KelemProd.m:14-185``        -> :func:`kelem_prod`
"""
import numpy as np
import scipy.sparse as sp

# Local node order of a hex8 element (I/DegreesOfFreedom.m:24-38 after sort,
# I/ElemStiffMatrixGQMR.m:77-82): y fastest, then x, then z.
LOCAL_NODES = np.array([(0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 0),
                        (0, 0, 1), (0, 1, 1), (1, 0, 1), (1, 1, 1)])  # (dx, dy, dz)


def constitutive(nu, E=1.0):
    """Isotropic D matrix, I/ElemStiffMatrixGQMR.m:27-29 (E = 1 at :13)."""
    v = nu
    D = np.zeros((6, 6))
    D[:3, :3] = v
    np.fill_diagonal(D[:3, :3], 1 - v)
    D[3, 3] = D[4, 4] = D[5, 5] = (1 - 2 * v) / 2
    return (E / ((1 + v) * (1 - 2 * v))) * D


def elem_stiff_gqmr(el, eh, ew, nu, n):
    """Stiffness integrands of the n^3 density sub-cubes of one element.

    I/ElemStiffMatrixGQMR.m:10-240 (deg = 1, 2-point Gauss per sub-cube,
    ``k2 = ct*(a*b*c)*k2; k2 = (k2+k2')/2`` at :233-234).
    Returns ``k`` of shape (n^3, 24, 24); sub-cube order is y fastest, then x,
    then z (loop ``elz, elx, ely`` at :54-56).
    """
    a, b, c = el / 2.0, eh / 2.0, ew / 2.0
    D = constitutive(nu)
    centers = np.array([-1.0 + (2 * i + 1) / n for i in range(n)])  # :32
    gp = np.array([-1.0 / np.sqrt(3.0), 1.0 / np.sqrt(3.0)])         # :38-40
    gw = np.array([1.0, 1.0])
    ks = np.zeros((n ** 3, 24, 24))
    ind = 0
    for elz in range(n):
        for elx in range(n):
            for ely in range(n):
                k2 = np.zeros((24, 24))
                minx, maxx = centers[elx] - 1.0 / n, centers[elx] + 1.0 / n
                miny, maxy = centers[ely] - 1.0 / n, centers[ely] + 1.0 / n
                minz, maxz = centers[elz] - 1.0 / n, centers[elz] + 1.0 / n
                ct = ((maxx - minx) / 2) * ((maxy - miny) / 2) * ((maxz - minz) / 2)
                for g3 in range(2):
                    for g1 in range(2):
                        for g2 in range(2):
                            x1 = ((maxx - minx) / 2) * gp[g1] + (maxx + minx) / 2
                            x2 = ((maxy - miny) / 2) * gp[g2] + (maxy + miny) / 2
                            x3 = ((maxz - minz) / 2) * gp[g3] + (maxz + minz) / 2
                            sx = 2 * LOCAL_NODES[:, 0] - 1
                            sy = 2 * LOCAL_NODES[:, 1] - 1
                            sz = 2 * LOCAL_NODES[:, 2] - 1
                            dxp = (1 / (8 * a)) * sx * (1 + sy * x2) * (1 + sz * x3)
                            dyp = (1 / (8 * b)) * sy * (1 + sx * x1) * (1 + sz * x3)
                            dzp = (1 / (8 * c)) * sz * (1 + sx * x1) * (1 + sy * x2)
                            B = np.zeros((6, 24))   # :218-227
                            B[0, 0::3] = dxp
                            B[1, 1::3] = dyp
                            B[2, 2::3] = dzp
                            B[3, 0::3] = dyp
                            B[3, 1::3] = dxp
                            B[4, 1::3] = dzp
                            B[4, 2::3] = dyp
                            B[5, 0::3] = dzp
                            B[5, 2::3] = dxp
                            k2 += (gw[g1] * gw[g2] * gw[g3]) * (B.T @ D @ B)
                k2 = ct * (a * b * c) * k2
                ks[ind] = (k2 + k2.T) / 2
                ind += 1
    return ks


def kv_matrix(ks):
    """``kv`` layout of the reference: column s is ``k{s}(:)`` (column-major)."""
    return np.stack([k.flatten(order="F") for k in ks], axis=1)


def node_index(x, y, z, nx, ny):
    """0-based node number: y fastest, then x, then z (I/EnterData.m:130)."""
    return (z * nx + x) * ny + y


def dof_table(nelx, nely, nelz):
    """Global 0-based dofs of every element, shape (nelem, 24).

    I/DegreesOfFreedom.m:19-54: elements walk y fastest, then x, then z; local
    dof = 3*local_node + component.
    """
    nx, ny = nelx + 1, nely + 1
    ez, ex, ey = np.meshgrid(np.arange(nelz), np.arange(nelx), np.arange(nely), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    nodes = np.stack([node_index(ex + dx, ey + dy, ez + dz, nx, ny) for dx, dy, dz in LOCAL_NODES], axis=1)
    dofs = (3 * nodes[:, :, None] + np.arange(3)[None, None, :]).reshape(-1, 24)
    return dofs


def density_table(nelx, nely, nelz, n):
    """0-based density-mesh indices of the n^3 sub-elements of every element.

    I/StartMR.m:58-83 (``fde``) and the sorted index vector ``v`` of
    I/GlobalStiffMatrix.m:33-47: sub-element order y fastest, then x, then z.
    Shape (nelem, n^3).
    """
    nely_d, nelx_d = nely * n, nelx * n
    ez, ex, ey = np.meshgrid(np.arange(nelz), np.arange(nelx), np.arange(nely), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    cols = []
    for sz in range(n):
        for sx in range(n):
            for sy in range(n):
                cols.append((ez * n + sz) * nelx_d * nely_d + (ex * n + sx) * nely_d + (ey * n + sy))
    return np.stack(cols, axis=1)


def simp(x, p, emin, E=1.0):
    """SIMP Young's factor emin + (E-emin) x^p (I/GlobalStiffMatrix.m:17,49)."""
    return emin + (E - emin) * np.power(x, p)


def element_matrices(ks, wsub):
    """K_e = sum_s w_{e,s} KE_s for every element (I/WOK/KelemProd.m:74)."""
    return np.einsum("es,sij->eij", wsub, ks)


def global_stiff_matrix(nelx, nely, nelz, ks, dens, p, emin, freedofs, E=1.0):
    """Assembled K(rho) restricted to the free dofs (I/GlobalStiffMatrix.m:16-65).

    ``dens``: filtered densities on the density mesh (n = 1: one per element).
    ``freedofs``: 0-based free dof indices.
    """
    n = round(len(ks) ** (1 / 3))
    dofs = dof_table(nelx, nely, nelz)
    didx = density_table(nelx, nely, nelz, n)
    w = simp(dens[didx], p, emin, E)
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    iK = np.repeat(dofs, 24, axis=1).ravel()
    jK = np.tile(dofs, (1, 24)).ravel()
    rows, cols, vals = [], [], []
    chunk = 20000
    for s in range(0, dofs.shape[0], chunk):
        Ke = element_matrices(ks, w[s:s + chunk])
        vals.append(Ke.reshape(-1))
    sK = np.concatenate(vals)
    K = sp.coo_matrix((sK, (iK, jK)), shape=(ndof, ndof)).tocsr()
    K.sum_duplicates()
    return K[freedofs][:, freedofs].tocsr()


def kelem_prod(nelx, nely, nelz, ks, dens, p, emin, freedofs, x, E=1.0):
    """Matrix-free y = K(rho) x on free dofs (I/WOK/KelemProd.m:14-100,185).

    Zero-extends x over the fixed dofs (:14-16), accumulates
    ``y(dofs) += (sum_s w_s KE_s) xc(dofs)`` per element and restricts (:185).
    """
    n = round(len(ks) ** (1 / 3))
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    xc = np.zeros(ndof)
    xc[freedofs] = x
    y = kelem_prod_full(nelx, nely, nelz, ks, simp(dens, p, emin, E), xc, n)
    return y[freedofs]


def kelem_prod_full(nelx, nely, nelz, ks, wdens, xc, n):
    """Element loop of I/WOK/KelemProd.m:57-100 on a full-length vector."""
    dofs = dof_table(nelx, nely, nelz)
    didx = density_table(nelx, nely, nelz, n)
    ue = xc[dofs]
    ye = np.zeros_like(ue)
    W = wdens[didx]
    for s in range(len(ks)):
        ye += W[:, s:s + 1] * (ue @ ks[s].T)
    return np.bincount(dofs.ravel(), weights=ye.ravel(), minlength=xc.size)
