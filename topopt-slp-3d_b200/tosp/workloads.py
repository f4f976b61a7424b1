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
WORKLOADS = {
    "cantilever192x96x96_mr2": dict(dims=(192, 96, 96), n=2, density="grf", ngrids=5, rmin=1.0),
    "cantilever96x48x48_mr2": dict(dims=(96, 48, 48), n=2, density="uniform_filtered", ngrids=4, rmin=1.0),
    "cantilever48x24x24": dict(dims=(48, 24, 24), n=1, density="const0.3", ngrids=3, rmin=1.5),
}


def build_workload(name, filter_fn=None):
    """Return (problem, n, xfil, spec).  ``filter_fn(x)`` applies the density
    filter for the uniform workload (the GPU filter of a solver handle)."""
    spec = WORKLOADS[name]
    nelx, nely, nelz = spec["dims"]
    n = spec["n"]
    pb = problems.cantilever(nelx, nely, nelz)
    nd = pb.nelem * n ** 3
    if spec["density"] == "grf":
        xfil = grf_heaviside(nelx * n, nely * n, nelz * n, seed=1)
    elif spec["density"] == "uniform_filtered":
        raw = uniform_raw(nd, seed=0)
        xfil = filter_fn(raw) if filter_fn is not None else raw
    else:
        xfil = np.full(nd, 0.3)
    return pb, n, xfil, spec
