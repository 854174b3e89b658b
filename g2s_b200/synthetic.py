"""Seeded synthetic training images for the QuickSampling workloads.

No public dataset is involved: every workload of this package runs on
synthetic, seeded inputs whose shapes, sizes and value distributions follow
the benchmark descriptions (continuous Gaussian random fields with an
exponential covariance, binary sinuous-channel images, bivariate
field + indicator).  Arrays are returned in the G2S grid convention
(numpy shape ``(…, ny, nx)`` i.e. x is the fastest axis, float32).
"""
from __future__ import annotations

import numpy as np


def grf(shape, ranges, seed: int) -> np.ndarray:
    """Gaussian random field with exponential covariance.

    Seeded N(0,1) white noise is filtered in Fourier space by the square root
    of the spectrum of C(h) = exp(-|h / range|) (anisotropic ranges per axis,
    given in numpy axis order), then standardised to mean 0 and variance 1.
    The field is generated on a periodic grid twice the size of the output
    and cropped, so the result shows no wrap-around seam.
    """
    shape = tuple(int(s) for s in shape)
    ranges = tuple(float(r) for r in ranges)
    assert len(shape) == len(ranges)
    big = tuple(2 * s for s in shape)
    axes = [np.minimum(np.arange(b), b - np.arange(b)).astype(np.float64) / r for b, r in zip(big, ranges)]
    grids = np.meshgrid(*axes, indexing="ij")
    h = np.sqrt(sum(g * g for g in grids))
    cov = np.exp(-h)
    spec = np.fft.rfftn(cov).real
    spec = np.sqrt(np.maximum(spec, 0.0))
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(big)
    field = np.fft.irfftn(np.fft.rfftn(noise) * spec, s=big, axes=tuple(range(len(big))))
    field = field[tuple(slice(0, s) for s in shape)]
    field = (field - field.mean()) / field.std()
    return field.astype(np.float32)


def channels2d(shape=(250, 250), n_channels: int = 20, seed: int = 1, target=(0.25, 0.30)) -> np.ndarray:
    """Binary sinuous-channel image: background 0, channels 1.

    Each channel centre line is y = a*sin(2*pi*x/lam + phi) + y0 with
    lam ~ U[60,180], a ~ U[5,25], width ~ U[4,9] px, y0 ~ U[0,ny),
    phi ~ U[0,2*pi).  The widths are scaled by a common factor (bisection)
    so that the facies-1 proportion lands inside ``target``.
    """
    ny, nx = shape
    rng = np.random.default_rng(seed)
    lam = rng.uniform(60, 180, n_channels)
    amp = rng.uniform(5, 25, n_channels)
    width = rng.uniform(4, 9, n_channels)
    y0 = rng.uniform(0, ny, n_channels)
    phi = rng.uniform(0, 2 * np.pi, n_channels)
    x = np.arange(nx, dtype=np.float64)[None, :]
    y = np.arange(ny, dtype=np.float64)[:, None]

    def render(scale):
        img = np.zeros(shape, dtype=bool)
        for i in range(n_channels):
            centre = amp[i] * np.sin(2 * np.pi * x / lam[i] + phi[i]) + y0[i]
            img |= np.abs(y - centre) < 0.5 * width[i] * scale
        return img

    lo, hi = 0.05, 4.0
    mid = 1.0
    img = render(mid)
    frac = img.mean()
    goal = 0.5 * (target[0] + target[1])
    for _ in range(40):
        if target[0] <= frac <= target[1]:
            break
        if frac < goal:
            lo = mid
        else:
            hi = mid
        mid = 0.5 * (lo + hi)
        img = render(mid)
        frac = img.mean()
    return img.astype(np.float32)


def tubes3d(shape=(256, 256, 256), seed: int = 1, target: float = 0.20) -> np.ndarray:
    """Binary 3-D sinusoid tubes (facies 1 about ``target`` of the volume).

    Tubes run along x; the centre line is (y, z) = (ay*sin(2*pi*x/lam+phi) + y0,
    az*cos(2*pi*x/lam+phi) + z0).  Radii are scaled by bisection towards the
    target proportion.
    """
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    n = max(4, int(round(nx * ny / 1500)))
    lam = rng.uniform(60, 180, n)
    ay = rng.uniform(5, 25, n)
    az = rng.uniform(1, 6, n)
    rad = rng.uniform(2, 5, n)
    y0 = rng.uniform(0, ny, n)
    z0 = rng.uniform(0, nz, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    x = np.arange(nx, dtype=np.float64)
    yy = np.arange(ny, dtype=np.float64)[:, None]
    zz = np.arange(nz, dtype=np.float64)[:, None, None]

    def render(scale):
        # each tube is rendered only over the (z, y) window its centre line
        # and radius can reach (outside it d2 >= r^2 everywhere)
        img = np.zeros(shape, dtype=bool)
        for i in range(n):
            r = rad[i] * scale
            cy = ay[i] * np.sin(2 * np.pi * x / lam[i] + phi[i]) + y0[i]
            cz = az[i] * np.cos(2 * np.pi * x / lam[i] + phi[i]) + z0[i]
            ya, yb = max(0, int(np.floor(cy.min() - r))), min(ny, int(np.ceil(cy.max() + r)) + 1)
            za, zb = max(0, int(np.floor(cz.min() - r))), min(nz, int(np.ceil(cz.max() + r)) + 1)
            if ya >= yb or za >= zb:
                continue
            d2 = (yy[None, ya:yb, :] - cy[None, None, :]) ** 2 + (zz[za:zb] - cz[None, None, :]) ** 2
            img[za:zb, ya:yb, :] |= d2 < r ** 2
        return img

    lo, hi, mid = 0.05, 6.0, 1.0
    img = render(mid)
    for _ in range(30):
        frac = img.mean()
        if abs(frac - target) < 0.01:
            break
        if frac < target:
            lo = mid
        else:
            hi = mid
        mid = 0.5 * (lo + hi)
        img = render(mid)
    return img.astype(np.float32)


def bivariate(field: np.ndarray, quantile: float = 0.7) -> np.ndarray:
    """Stack a continuous field with its indicator at ``quantile``:
    returns shape field.shape + (2,) (variables interleaved, G2S layout)."""
    thr = np.quantile(field, quantile)
    ind = (field > thr).astype(np.float32)
    return np.stack([field.astype(np.float32), ind], axis=-1)
