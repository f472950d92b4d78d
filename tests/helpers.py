"""Shared helpers of the test-suite: seeded inputs and comparisons."""
import itertools
import json
import os
from math import comb

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def combos(n, k):
    """Lexicographic k-combinations of range(n) (component order of SimiLie's antisymmetric index)."""
    return list(itertools.combinations(range(n), k))


def comp_index(n, dims):
    return combos(n, len(dims)).index(tuple(sorted(dims)))


def kat_field(N, ndim, k):
    """Fixture of tests/exterior/derivative.cpp:15-100: component c holds c+1
    everywhere except c+2 at node (1,...,1).  Shape (N,)*ndim + (C(ndim,k),)."""
    nc = comb(ndim, k)
    a = np.zeros((N,) * ndim + (nc,))
    for c in range(nc):
        a[..., c] = c + 1.0
        a[(1,) * ndim + (c,)] = c + 2.0
    return a


def stretched_coords(n, ratio=1.01, h0=None, start=0.0):
    """Geometric node coordinates with spacing ratio `ratio`."""
    if h0 is None:
        h0 = 1.0 / n
    h = h0 * ratio ** np.arange(n - 1)
    return start + np.concatenate([[0.0], np.cumsum(h)])


def rel_err(got, ref):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.max(np.abs(ref))
    if scale == 0:
        return float(np.max(np.abs(got)))
    return float(np.max(np.abs(got - ref)) / scale)


def random_form(rng, shape, ncomp):
    return rng.standard_normal(tuple(shape) + (ncomp,))


def sinusoid_field(n_pts, seed, modes=8, kmax=16, noise=1e-3):
    """Input of the 512^2 scalar Laplacian workload: sum of `modes` products of
    sines with integer wavenumbers 1..kmax, amplitudes U[-1,1], phases U[0,1),
    plus U[-noise, noise] noise."""
    rng = np.random.default_rng(seed)
    x = np.arange(n_pts) / n_pts
    X, Y = np.meshgrid(x, x, indexing="ij")
    f = np.zeros((n_pts, n_pts))
    for _ in range(modes):
        kx, ky = rng.integers(1, kmax + 1, size=2)
        a = rng.uniform(-1, 1)
        px, py = rng.uniform(0, 1, size=2)
        f += a * np.sin(2 * np.pi * (kx * X + px)) * np.sin(2 * np.pi * (ky * Y + py))
    f += rng.uniform(-noise, noise, size=f.shape)
    return f


def gaussian_random_field(n_pts, seed, ncomp=2, power=-2.0, dtype=np.float64):
    """Components drawn as independent Gaussian random fields with power
    spectrum |k|^power (k = 0 removed), normalised to unit RMS."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(n_pts) * n_pts
    ky = np.fft.rfftfreq(n_pts) * n_pts
    K2 = kx[:, None] ** 2 + ky[None, :] ** 2
    amp = np.zeros_like(K2)
    nz = K2 > 0
    amp[nz] = K2[nz] ** (power / 4.0)  # |k|^(power/2) in amplitude
    out = np.empty((n_pts, n_pts, ncomp), dtype=dtype)
    for c in range(ncomp):
        noise = rng.standard_normal((n_pts, n_pts // 2 + 1)) + 1j * rng.standard_normal((n_pts, n_pts // 2 + 1))
        f = np.fft.irfft2(noise * amp, s=(n_pts, n_pts))
        f /= np.sqrt(np.mean(f ** 2))
        out[..., c] = f
    return out
