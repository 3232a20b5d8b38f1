"""Seeded synthetic DEMs for benchmarks and tests.

The reference's examples run on a private raster and on an absent Perlin-noise
package, so the workloads here use a generator of our own, fixed as follows:

1. white noise N(0, 1) of shape (ny, nx) from ``numpy.random.default_rng(seed)``;
2. rFFT2, amplitude multiplied by k^-2 with k = sqrt(kx^2 + ky^2) in cycles/cell
   and the k = 0 term set to 0, inverse rFFT2 (a spectral 1/f^2 surface);
3. min-max rescale to [0, relief] metres;
4. optional tilt ``tilt * dx * row`` (metres; rows count southwards);
5. ``npits`` Gaussian pits: centre uniform over cells, depth U(1, 20) m, radius
   U(3, 30) cells times ``pit_scale``, ``z -= depth * exp(-r^2 / R^2)`` evaluated
   within 4R of the centre;
6. cast to float32.

Everything is computed in float64 and rounded once at the end.
"""
from __future__ import annotations

import numpy as np


def spectral_dem(nx: int, ny: int, seed: int, relief: float = 500.0, dx: float = 1.0,
                 tilt: float = 0.0, npits: int = 0, pit_scale: float | None = None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((ny, nx))
    F = np.fft.rfft2(noise)
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    F = F / (k * k)
    F[0, 0] = 0.0
    z = np.fft.irfft2(F, s=(ny, nx))
    zmin, zmax = z.min(), z.max()
    z = (z - zmin) / (zmax - zmin) * relief
    if tilt:
        z = z + tilt * dx * np.arange(ny, dtype=np.float64)[:, None]
    if npits:
        if pit_scale is None:
            pit_scale = max(nx, ny) / 4096.0
        cx = rng.integers(0, nx, npits)
        cy = rng.integers(0, ny, npits)
        depth = rng.uniform(1.0, 20.0, npits)
        rad = rng.uniform(3.0, 30.0, npits) * pit_scale
        for x0, y0, d, R in zip(cx, cy, depth, rad):
            w = int(np.ceil(4.0 * R))
            xa, xb = max(0, x0 - w), min(nx, x0 + w + 1)
            ya, yb = max(0, y0 - w), min(ny, y0 + w + 1)
            yy, xx = np.mgrid[ya:yb, xa:xb]
            r2 = (xx - x0) ** 2 + (yy - y0) ** 2
            z[ya:yb, xa:xb] -= d * np.exp(-r2 / (R * R))
    return z.astype(np.float32)


def lognormal_weights(n: int, seed: int, sigma: float = 0.5) -> np.ndarray:
    """Per-cell precipitation weights, lognormal(mu=0, sigma) float32."""
    rng = np.random.default_rng(seed)
    return rng.lognormal(0.0, sigma, n).astype(np.float32)


# Named workloads (sizes, relief, pits and boundary modes of the benchmark configs).
def routing_plain_512(seed: int = 1):
    """512 x 512, dx = 30 m, relief 0-500 m + 0.005 m/m tilt, all edges outlets."""
    return dict(z=spectral_dem(512, 512, seed, relief=500.0, dx=30.0, tilt=0.005), nx=512, ny=512,
                dx=30.0, mode="normal")


def routing_lakes(n: int = 4096, seed: int = 2, dx: float = 30.0):
    """n x n, relief 0-1500 m, 2000 pits per 4096^2 (scaled by area), periodic
    east-west with outlets on the north and south rows, carve rerouting."""
    npits = int(round(2000 * (n * n) / (4096.0 * 4096.0)))
    return dict(z=spectral_dem(n, n, seed, relief=1500.0, dx=dx, npits=max(npits, 1)), nx=n, ny=n,
                dx=dx, mode="periodic_EW")


def graphflood_plain(n: int = 2048, seed: int = 3):
    """n x n, dx = 10 m, relief 0-1500 m, pits scaled to the grid, all edges outlets."""
    npits = int(round(2000 * (n * n) / (4096.0 * 4096.0)))
    return dict(z=spectral_dem(n, n, seed, relief=1500.0, dx=10.0, npits=max(npits, 1)), nx=n, ny=n,
                dx=10.0, mode="normal")


def ragged_tiles(ntiles: int = 512, seed: int = 4, side_min: int = 128, side_max: int = 1024,
                 max_pits: int = 200, dx: float = 30.0, relief: float = 500.0):
    """A ragged batch: per tile, nx and ny drawn independently log-uniform in
    [side_min, side_max], its own generator seed, 0..max_pits pits (radii scaled by
    max(nx, ny)/1024) and a boundary mode drawn from {normal, periodic_EW}.
    Returns a list of dicts (z, nx, ny, dx, mode)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(side_min), np.log(side_max)
    tiles = []
    for t in range(ntiles):
        nx = int(round(np.exp(rng.uniform(lo, hi))))
        ny = int(round(np.exp(rng.uniform(lo, hi))))
        npits = int(rng.integers(0, max_pits + 1))
        mode = "periodic_EW" if rng.integers(0, 2) else "normal"
        z = spectral_dem(nx, ny, seed * 100003 + t, relief=relief, dx=dx, npits=npits,
                         pit_scale=max(nx, ny) / 1024.0)
        tiles.append(dict(z=z, nx=nx, ny=ny, dx=dx, mode=mode))
    return tiles
