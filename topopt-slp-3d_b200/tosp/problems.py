"""Problem definitions: the reference's ``str`` struct and its builders.

Host-side logic mirroring the problem input of TopOpt-SLP-3D:
  * supports -> ``freedofs`` (I/EnterData.m:122-156),
  * loads    -> ``f`` restricted to the free dofs (I/EnterData.m:159-797),
  * void/solid regions -> ``fixedDens`` (I/EnterData.m:800-905, I/StartMR.m:86-152),
  * loading the saved fixtures ``I/Tests/*.mat``.
(``I/`` abbreviates the reference's ``Implementation/`` folder.)

Axes follow the reference: y is the vertical (height) axis, z the width.
Node numbering is y fastest, then x, then z; all indices here are 0-based.
"""
import math
from dataclasses import dataclass, field

import numpy as np


def _layer(c, h):
    """Node layer (0-based) nearest to coordinate c (I/EnterData.m:122-127)."""
    r = c - math.floor(c / h) * h          # MATLAB mod for non-negative c
    return int(math.floor(c / h) + (1 if r > h / 2 else 0))


def _line_weights(c0, cf, h):
    """1-D nodal weights of a load distributed over [c0, cf].

    I/EnterData.m:203-349: one node gets ``cf-c0`` when both ends round to the
    same layer; otherwise the first node gets ``(n0-1/2)h - c0``, interior
    nodes ``h`` and the last ``cf - (nf-3/2)h`` (1-based layers n0, nf).  Area
    loads use the product of two such lists (I/EnterData.m:350-782).
    """
    n0, nf = _layer(c0, h), _layer(cf, h)
    if n0 == nf:
        return [n0], [cf - c0]
    n01, nf1 = n0 + 1, nf + 1                 # 1-based layers of the reference
    nodes = list(range(n0, nf + 1))
    wts = [(n01 - 0.5) * h - c0] + [h] * (nf - n0 - 1) + [cf - (nf1 - 1.5) * h]
    return nodes, wts


@dataclass
class Problem:
    """The fields of the reference's ``str`` struct used on the solve path."""
    nelx: int
    nely: int
    nelz: int
    el: float = 1.0
    eh: float = 1.0
    ew: float = 1.0
    E: float = 1.0
    nu: float = 0.3
    freedofs: np.ndarray = None          # 0-based, sorted
    f: np.ndarray = None                 # loads on the free dofs
    fixed_dens: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    fixed_dens_val: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fix: np.ndarray = None               # rows [ex0 exf ey0 eyf ez0 ezf solid], 1-based layers
    supp: np.ndarray = None
    loads: np.ndarray = None
    name: str = ""

    @property
    def nx(self):
        return self.nelx + 1

    @property
    def ny(self):
        return self.nely + 1

    @property
    def nz(self):
        return self.nelz + 1

    @property
    def nnodes(self):
        return self.nx * self.ny * self.nz

    @property
    def nelem(self):
        return self.nelx * self.nely * self.nelz

    @property
    def l(self):
        return self.nelx * self.el

    @property
    def h(self):
        return self.nely * self.eh

    @property
    def w(self):
        return self.nelz * self.ew

    def f_full(self):
        """Load vector over all 3*nnodes dofs."""
        out = np.zeros(3 * self.nnodes)
        out[self.freedofs] = self.f
        return out


def supports_to_freedofs(pb, supp):
    """``str.freedofs`` from support rows ``[x0 xf y0 yf z0 zf ix iy iz]``.

    I/EnterData.m:122-156: every node in the rounded layer box loses the
    components whose flag is set.
    """
    fixed = np.zeros(3 * pb.nnodes, dtype=bool)
    for row in np.atleast_2d(supp):
        x0, xf, y0, yf, z0, zf, ix, iy, iz = [float(v) for v in row]
        nxs = range(_layer(x0, pb.el), _layer(xf, pb.el) + 1)
        nys = range(_layer(y0, pb.eh), _layer(yf, pb.eh) + 1)
        nzs = range(_layer(z0, pb.ew), _layer(zf, pb.ew) + 1)
        for kz in nzs:
            for kx in nxs:
                for ky in nys:
                    node = (kz * pb.nx + kx) * pb.ny + ky
                    for comp, flag in enumerate((ix, iy, iz)):
                        if flag != 0:
                            fixed[3 * node + comp] = True
    return np.nonzero(~fixed)[0].astype(np.int64)


def loads_to_f(pb, loads, freedofs):
    """``str.f`` (restricted to the free dofs) from load rows
    ``[x0 xf y0 yf z0 zf Fx Fy Fz]`` (I/EnterData.m:159-797).

    A coordinate range with ``c0 != cf`` is a distributed direction; the nodal
    weights are products of :func:`_line_weights` lists.
    """
    f = np.zeros(3 * pb.nnodes)
    for row in np.atleast_2d(loads):
        x0, xf, y0, yf, z0, zf, Fx, Fy, Fz = [float(v) for v in row]
        lx = _line_weights(x0, xf, pb.el) if xf != x0 else ([_layer(x0, pb.el)], [1.0])
        ly = _line_weights(y0, yf, pb.eh) if yf != y0 else ([_layer(y0, pb.eh)], [1.0])
        lz = _line_weights(z0, zf, pb.ew) if zf != z0 else ([_layer(z0, pb.ew)], [1.0])
        for kz, wz in zip(*lz):
            for kx, wx in zip(*lx):
                for ky, wy in zip(*ly):
                    node = (kz * pb.nx + kx) * pb.ny + ky
                    # at most two factors differ from 1, so this product is
                    # bit-identical to the reference's ``d*(edge term)*F``
                    wgt = wx * wy * wz
                    f[3 * node + 0] += wgt * Fx
                    f[3 * node + 1] += wgt * Fy
                    f[3 * node + 2] += wgt * Fz
    return f[freedofs]


def fixed_from_rows(nelx, nely, nelz, fix, mult=1):
    """Fixed elements and values from ``str.fix`` rows on a mesh refined by
    ``mult`` (I/StartMR.m:86-112; ``mult = 1`` is the displacement mesh)."""
    fixd = np.zeros(nelx * nely * nelz * mult ** 3, dtype=bool)
    val = np.zeros(fixd.size)
    nx_, ny_ = nelx * mult, nely * mult
    for row in np.atleast_2d(fix):
        ex0, exf, ey0, eyf, ez0, ezf, solid = [int(v) for v in row]
        xs = np.arange((ex0 - 1) * mult, exf * mult)
        ys = np.arange((ey0 - 1) * mult, eyf * mult)
        zs = np.arange((ez0 - 1) * mult, ezf * mult)
        Z, X, Y = np.meshgrid(zs, xs, ys, indexing="ij")
        idx = ((Z * nx_ + X) * ny_ + Y).ravel()
        fixd[idx] = True
        if solid == 1:
            val[idx] = 1.0
    fixed = np.nonzero(fixd)[0].astype(np.int64)
    return fixed, val[fixed]


def build(nelx, nely, nelz, supp, loads, fix=None, el=1.0, eh=1.0, ew=1.0, E=1.0, nu=0.3, name=""):
    """Build a :class:`Problem` from support/load/region rows like EnterData."""
    pb = Problem(nelx, nely, nelz, el, eh, ew, E, nu, name=name)
    pb.supp = np.atleast_2d(np.asarray(supp, dtype=float))
    pb.loads = np.atleast_2d(np.asarray(loads, dtype=float))
    pb.freedofs = supports_to_freedofs(pb, pb.supp)
    pb.f = loads_to_f(pb, pb.loads, pb.freedofs)
    if fix is not None and len(fix):
        pb.fix = np.atleast_2d(np.asarray(fix, dtype=np.int64))
        pb.fixed_dens, pb.fixed_dens_val = fixed_from_rows(nelx, nely, nelz, pb.fix)
    return pb


def load_mat(path):
    """Load a saved reference problem (``I/Tests/*.mat``, a struct ``str``).

    ``freedofs`` is stored 1-based as uint16/int32/double and ``f`` as
    int16/double; both are cast (0-based int64 and float64).
    """
    import scipy.io as sio
    s = sio.loadmat(path, squeeze_me=True, struct_as_record=False)["str"]
    pb = Problem(int(s.nelx), int(s.nely), int(s.nelz), float(s.el), float(s.eh), float(s.ew),
                 float(s.E), float(s.nu), name=str(path))
    pb.freedofs = np.asarray(s.freedofs, dtype=np.int64).ravel() - 1
    pb.f = np.asarray(s.f, dtype=np.float64).ravel()
    names = s._fieldnames
    if "supp" in names:
        pb.supp = np.atleast_2d(np.asarray(s.supp, dtype=float))
    if "loads" in names:
        pb.loads = np.atleast_2d(np.asarray(s.loads, dtype=float))
    if "fix" in names:
        pb.fix = np.atleast_2d(np.asarray(s.fix, dtype=np.int64))
    if "fixedDens" in names and np.size(s.fixedDens):
        pb.fixed_dens = np.asarray(s.fixedDens, dtype=np.int64).ravel() - 1
        pb.fixed_dens_val = np.asarray(s.fixedDensVal, dtype=np.float64).ravel()
    return pb


# ---------------------------------------------------------------------------
# Synthetic workloads.  Sizes are given in the reference's axes
# (nelx = length, nely = height, nelz = width).
# ---------------------------------------------------------------------------

def cantilever(nelx, nely, nelz):
    """Cantilever: the x = 0 face fully fixed; a unit downward (-y) load spread
    along the bottom edge at x = L (line load along z at y = 0, total -1)."""
    pb = Problem(nelx, nely, nelz)
    supp = [[0, 0, 0, pb.h, 0, pb.w, 1, 1, 1]]
    loads = [[pb.l, pb.l, 0, 0, 0, pb.w, 0, -1.0 / pb.w, 0]]
    return build(nelx, nely, nelz, supp, loads, name=f"cantilever{nelx}x{nely}x{nelz}")


def bridge(nelx, nely, nelz):
    """Bridge: pinned at both bottom corner lines (x = 0 and x = L, y = 0,
    all z; all components fixed), uniform downward traction on the top face
    (area load on the xz plane at y = h, total -1)."""
    pb = Problem(nelx, nely, nelz)
    supp = [[0, 0, 0, 0, 0, pb.w, 1, 1, 1],
            [pb.l, pb.l, 0, 0, 0, pb.w, 1, 1, 1]]
    loads = [[0, pb.l, pb.h, pb.h, 0, pb.w, 0, -1.0 / (pb.l * pb.w), 0]]
    return build(nelx, nely, nelz, supp, loads, name=f"bridge{nelx}x{nely}x{nelz}")


def torsion(nelx, nely, nelz):
    """Torsion: the x = 0 face fixed; a tangential couple on the x = L face
    made of four edge-midpoint loads (like the reference's ``bt*`` fixtures)."""
    pb = Problem(nelx, nely, nelz)
    L, H, W = pb.l, pb.h, pb.w
    supp = [[0, 0, 0, H, 0, W, 1, 1, 1]]
    loads = [[L, L, H / 2, H / 2, 0, 0, 0, 1, 0],
             [L, L, H / 2, H / 2, W, W, 0, -1, 0],
             [L, L, H, H, W / 2, W / 2, 0, 0, -1],
             [L, L, 0, 0, W / 2, W / 2, 0, 0, 1]]
    return build(nelx, nely, nelz, supp, loads, name=f"torsion{nelx}x{nely}x{nelz}")
