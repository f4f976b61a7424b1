"""Synthetic density fields and the benchmark workloads.

The reference publishes no benchmark data; these seeded generators stand in
for its problems with the sizes and value ranges of the configurations:
  * ``uniform_filtered``: i.i.d. U[0.001, 1] densities on the density mesh,
    then the radius-2 density filter (multiresolution cantilever, 96x48x48).
  * ``grf_heaviside``: a Gaussian random field (white noise smoothed by a
    Gaussian kernel of standard deviation 8 density cells, periodic FFT),
    mapped to [0, 1] through the normal CDF, projected with the smooth
    Heaviside of the reference (I/HeavisideProj.m, beta = 4, eta = 0.5) and
    scaled into [0.001, 1] (192x96x96 mixed-precision workload).
Arrays are in the reference's density order (y fastest, then x, then z).
"""
import math

import numpy as np

from . import problems


def heaviside(x, beta, eta):
    """Smooth Heaviside projection (tanh form) with H(0) = 0, H(1) = 1."""
    num = np.tanh(beta * eta) + np.tanh(beta * (x - eta))
    return num / (math.tanh(beta * eta) + math.tanh(beta * (1.0 - eta)))


def grf_heaviside(nelx_d, nely_d, nelz_d, seed=1, sigma=8.0, beta=4.0, eta=0.5, lo=0.001):
    from scipy.special import ndtr
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((nelz_d, nelx_d, nely_d))
    F = np.fft.rfftn(noise)
    kz = np.fft.fftfreq(nelz_d)[:, None, None]
    kx = np.fft.fftfreq(nelx_d)[None, :, None]
    ky = np.fft.rfftfreq(nely_d)[None, None, :]
    F *= np.exp(-2.0 * (math.pi * sigma) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    field = np.fft.irfftn(F, s=noise.shape)
    field = (field - field.mean()) / field.std()
    v = heaviside(ndtr(field), beta, eta)
    return (lo + (1.0 - lo) * v).ravel()


def uniform_raw(nelem_d, seed=0, lo=0.001):
    return np.random.default_rng(seed).uniform(lo, 1.0, nelem_d)


# Workloads in the reference's axes: nelx (length) x nely (height) x nelz (width).
# Jacobi relaxation of the reference's default parameter set (mg.omega,
# I/TopOpt3D.m:174); the 48x24x24 case states its own 0.6.  With 0.6 the
# damped-Jacobi sweep is not convergent on strongly heterogeneous SIMP
# stiffness (max eigenvalue of D^-1 K about 4.4 for i.i.d. densities against
# 3.1 for a uniform one), so the V-cycle is indefinite on some modes.
REF_OMEGA = 0.5

WORKLOADS = {
    "cantilever192x96x96_mr2": dict(dims=(192, 96, 96), n=2, density="grf", ngrids=5, rmin=1.0, omega=REF_OMEGA,
                                    pcg_iterations_fp64=110),
    "cantilever96x48x48_mr2": dict(dims=(96, 48, 48), n=2, density="uniform_filtered", ngrids=4, rmin=1.0,
                                   omega=REF_OMEGA),
    "cantilever48x24x24": dict(dims=(48, 24, 24), n=1, density="const0.3", ngrids=3, rmin=1.5, omega=0.6),
    # smaller cases of the same kernels (profiler captures)
    "cantilever128x64x64_mr2": dict(dims=(128, 64, 64), n=2, density="grf", ngrids=4, rmin=1.0, omega=REF_OMEGA),
    "cantilever128x64x64": dict(dims=(128, 64, 64), n=1, density="grf", ngrids=4, rmin=1.5, omega=REF_OMEGA),
    # the 160 x 40 x 80 bridge of the MR-3 SLP loop (reference axes: height 80)
    "bridge160x80x40_mr3": dict(dims=(160, 80, 40), n=3, density="grf", ngrids=4, rmin=2.5 / 3, omega=REF_OMEGA,
                                problem="bridge"),
}


def build_workload(name, filter_fn=None):
    """Return (problem, n, xfil, spec).  ``filter_fn(x)`` applies the density
    filter for the uniform workload (the GPU filter of a solver handle)."""
    spec = WORKLOADS[name]
    nelx, nely, nelz = spec["dims"]
    n = spec["n"]
    pb = getattr(problems, spec.get("problem", "cantilever"))(nelx, nely, nelz)
    nd = pb.nelem * n ** 3
    if spec["density"] == "grf":
        xfil = grf_heaviside(nelx * n, nely * n, nelz * n, seed=1)
    elif spec["density"] == "uniform_filtered":
        raw = uniform_raw(nd, seed=0)
        xfil = filter_fn(raw) if filter_fn is not None else raw
    else:
        xfil = np.full(nd, 0.3)
    return pb, n, xfil, spec


# ---------------------------------------------------------------------------
# Serving stream: seed-7 requests with Poisson arrivals.
# ---------------------------------------------------------------------------
SERVING_NX = (32, 64, 96, 128)
SERVING_BC = ("cantilever", "bridge", "torsion")


def serving_levels(nx):
    """Grids for an nx x nx/2 x nx/2 mesh: coarsest grid of 8 (or 12) x 4 x 4
    elements, within the reference's level rule."""
    ng = 1
    while nx // (2 ** ng) >= 8 and (nx // 2) % (2 ** ng) == 0:
        ng += 1
    return ng


def serving_requests(count=512, seed=7, pool=3):
    """Request descriptors: (nx, n, bc, field index, eta).  Density fields are
    drawn from a small pool of seeded Gaussian random fields per shape (each
    request shifts the Heaviside threshold), so generating the stream stays
    cheap."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx = int(rng.choice(SERVING_NX))
        n = int(rng.choice((1, 2)))
        bc = str(rng.choice(SERVING_BC))
        out.append((nx, n, bc, int(rng.integers(pool)), float(rng.uniform(0.4, 0.6))))
    return out


def serving_problem(nx, bc):
    builder = {"cantilever": problems.cantilever, "bridge": problems.bridge, "torsion": problems.torsion}[bc]
    return builder(nx, nx // 2, nx // 2)


class FieldPool:
    """Seeded GRF fields per (nx, n, index), generated on first use."""

    def __init__(self, seed=7):
        self.seed = seed
        self.cache = {}

    def field(self, nx, n, idx, eta):
        key = (nx, n, idx)
        if key not in self.cache:
            from scipy.special import ndtr
            rng = np.random.default_rng((self.seed, nx, n, idx))
            shape = (nx // 2 * n, nx * n, nx // 2 * n)     # (z, x, y) of the density mesh
            noise = rng.standard_normal(shape)
            F = np.fft.rfftn(noise)
            kz = np.fft.fftfreq(shape[0])[:, None, None]
            kx = np.fft.fftfreq(shape[1])[None, :, None]
            ky = np.fft.rfftfreq(shape[2])[None, None, :]
            F *= np.exp(-2.0 * (math.pi * 4.0 * n) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
            fld = np.fft.irfftn(F, s=shape, axes=(0, 1, 2))
            self.cache[key] = ndtr((fld - fld.mean()) / fld.std()).ravel()
        return 0.001 + 0.999 * heaviside(self.cache[key], 4.0, eta)
