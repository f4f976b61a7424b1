"""Generate tests/golden/solutions.npz: small golden solutions of the solve
path from the NumPy/SciPy oracle (oracle/: assembled K, SetupGMG, SolveMG,
Grad), for the GPU parity tests and as a pin of the oracle itself.

    python tests/golden/make_solutions.py

Cases (reference axes: nelx length, nely height, nelz width):
  * ``cb48x16x16``: the reference's own problem file
    Implementation/Tests/cb48x16x16.mat (supports, point load, freedofs and f
    as stored in tests/golden/fixtures.npz), densities 0.3, MR factor 1;
  * ``config0_24x12x12``: the 48x24x24 cantilever workload at half size
    (x = 0 face fixed, unit load along the bottom edge at x = L), densities
    0.3, MR factor 1, filter radius 1.5, V-cycle with omega 0.6;
  * ``config1_16x8x8_mr2``: the multiresolution workload at reduced size,
    MR factor 2, i.i.d. U[0.001, 1] densities (seed 0) through the radius-2
    density filter (rmin 1.0), V-cycle with omega 0.5.
Every case: 3 grids, 1+1 Jacobi sweeps, PCG from zero to 1e-8 with the
reference's beta, then Grad with the transposed filter.  Stored per case:
the inputs that are not rebuilt from code (densities), the reference's `it`,
u on the free dofs, the compliance F = f'u and the filtered sensitivities.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "topopt-slp-3d_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import fem, filt, gmg  # noqa: E402
from tosp import problems as P  # noqa: E402

CASES = {
    "cb48x16x16": dict(n=1, omega=0.6, rmin=1.5, density="const0.3"),
    "config0_24x12x12": dict(n=1, omega=0.6, rmin=1.5, density="const0.3"),
    "config1_16x8x8_mr2": dict(n=2, omega=0.5, rmin=1.0, density="uniform_filtered"),
}
NGRIDS, TOL, P_SIMP, EMIN = 3, 1e-8, 3.0, 1e-9


def fixture_problem(name):
    g = np.load(os.path.join(HERE, "fixtures.npz"))
    nelx, nely, nelz = [int(v) for v in g[name + "/dims"]]
    el, eh, ew, E, nu = g[name + "/sizes"]
    return P.build(nelx, nely, nelz, g[name + "/supp"], g[name + "/loads"], el=el, eh=eh, ew=ew, E=E, nu=nu)


def case_problem(name):
    if name == "cb48x16x16":
        return fixture_problem(name)
    if name == "config0_24x12x12":
        return P.cantilever(24, 12, 12)
    return P.cantilever(16, 8, 8)


def solve_case(name, spec):
    pb = case_problem(name)
    n = spec["n"]
    nd = pb.nelem * n ** 3
    W, w = filt.elem_neighborhood(pb.nelx * n, pb.nely * n, pb.nelz * n, pb.el / n, pb.eh / n, pb.ew / n,
                                  spec["rmin"], 1)
    if spec["density"] == "const0.3":
        dens = np.full(nd, 0.3)
    else:
        dens = filt.apply_filter(np.random.default_rng(0).uniform(0.001, 1.0, nd), W, w, 1, False)
    ks = fem.elem_stiff_gqmr(pb.el, pb.eh, pb.ew, pb.nu, n)
    K = fem.global_stiff_matrix(pb.nelx, pb.nely, pb.nelz, ks, dens, P_SIMP, EMIN, pb.freedofs)
    H = gmg.setup_gmg(K, pb.nelx, pb.nely, pb.nelz, pb.freedofs, NGRIDS, spec["omega"])
    u, it = gmg.solve_mg(H, np.zeros(pb.f.size), pb.f, 0, 1, 1, TOL, 1000)
    ufull = np.zeros(3 * pb.nnodes)
    ufull[pb.freedofs] = u
    g, _ = filt.grad(pb.nelx, pb.nely, pb.nelz, ks, ufull, dens, P_SIMP, EMIN, W, w, 1)
    return {"dens": dens, "it": np.array([it]), "u": u, "F": np.array([pb.f @ u]), "g": g,
            "relres": np.array([np.linalg.norm(pb.f - K @ u) / np.linalg.norm(pb.f)])}


def main():
    out = {}
    for name, spec in CASES.items():
        r = solve_case(name, spec)
        for k, v in r.items():
            if k == "dens" and spec["density"] == "const0.3":
                continue
            out[name + "/" + k] = v
        print(name, "it", int(r["it"][0]), "F", float(r["F"][0]), "relres", float(r["relres"][0]))
    np.savez_compressed(os.path.join(HERE, "solutions.npz"), **out)


if __name__ == "__main__":
    main()
