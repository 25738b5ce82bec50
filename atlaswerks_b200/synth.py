"""Seeded synthetic inputs for the registration workloads.

The reference's own tests use synthetic bullseye volumes
(Testing/TestUtils.cxx:17-113); its benchmarks name no public dataset. The
workloads here are Gaussian-blob volumes warped by a smooth random
displacement, all fixed by a numpy PCG64 seed:

* ``blobs`` — sum of isotropic Gaussian blobs, centres uniform in the
  interior, sigma ~ U(4, 10) voxels, amplitude ~ U(0.3, 1), clipped to [0, 1].
* ``smooth_displacement`` — white noise per component, Gaussian-filtered with
  sigma 8 voxels (periodic, in Fourier space), scaled so max |u| = umax.
* ``warp`` — target(x) = source(x + u(x)), trilinear, zero outside.
* ``bullseye`` — nested spheres of alternating intensity, restating
  TestUtils::GenBullseye (Testing/TestUtils.cxx:17-23).

Arrays are float32 [nz, ny, nx] (x fastest); vector fields [3, nz, ny, nx].
"""
from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np

Shape = Tuple[int, int, int]


def rng_for(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def blobs(shape: Shape, n_blobs: int, rng: np.random.Generator,
          sigma_range=(4.0, 10.0), amp_range=(0.3, 1.0)) -> np.ndarray:
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    img = np.zeros(shape, np.float64)
    smax = sigma_range[1]
    for _ in range(n_blobs):
        c = [rng.uniform(min(smax, n / 2 - 1), max(n - smax, n / 2 + 1)) for n in (nx, ny, nz)]
        s = rng.uniform(*sigma_range)
        a = rng.uniform(*amp_range)
        img += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
    return np.clip(img, 0.0, 1.0).astype(np.float32)


def smooth_displacement(shape: Shape, umax: float, rng: np.random.Generator,
                        sigma: float = 8.0) -> np.ndarray:
    nz, ny, nx = shape
    noise = rng.standard_normal((3,) + shape)
    kz = np.fft.fftfreq(nz)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    kx = np.fft.rfftfreq(nx)[None, None, :]
    g = np.exp(-2.0 * (np.pi * sigma) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    u = np.stack([np.fft.irfftn(np.fft.rfftn(noise[c]) * g, s=shape, axes=(0, 1, 2))
                  for c in range(3)])
    mag = np.sqrt((u ** 2).sum(0)).max()
    u *= umax / mag
    return u.astype(np.float32)


def trilinear(img: np.ndarray, px: np.ndarray, py: np.ndarray, pz: np.ndarray) -> np.ndarray:
    """Trilinear sample of img at float positions, zero outside (per corner)."""
    nz, ny, nx = img.shape
    fx, fy, fz = np.floor(px), np.floor(py), np.floor(pz)
    t, u, v = px - fx, py - fy, pz - fz
    fx, fy, fz = fx.astype(np.int64), fy.astype(np.int64), fz.astype(np.int64)
    out = np.zeros(px.shape, np.float64)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                cx, cy, cz = fx + dx, fy + dy, fz + dz
                ok = (cx >= 0) & (cx < nx) & (cy >= 0) & (cy < ny) & (cz >= 0) & (cz < nz)
                w = (t if dx else 1 - t) * (u if dy else 1 - u) * (v if dz else 1 - v)
                val = np.zeros(px.shape, np.float64)
                val[ok] = img[cz[ok], cy[ok], cx[ok]]
                out += w * val
    return out


def warp(img: np.ndarray, u: np.ndarray) -> np.ndarray:
    nz, ny, nx = img.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return trilinear(img.astype(np.float64), x + u[0], y + u[1], z + u[2]).astype(np.float32)


def greedy_pair(shape: Shape, seed: int, n_blobs: int = 8, umax: float = 3.0,
                noise_sd: float = 0.0, sigma_range=(4.0, 10.0),
                smooth_sigma: float = 8.0) -> Tuple[np.ndarray, np.ndarray]:
    """(I0 source, I1 target) for pair registration: I1 = I0 warped by a
    smooth random displacement, plus optional Gaussian noise on both.
    sigma_range / smooth_sigma shrink the blobs and the displacement
    correlation length for grids much smaller than 64^3."""
    rng = rng_for(seed)
    src = blobs(shape, n_blobs, rng, sigma_range)
    u = smooth_displacement(shape, umax, rng, smooth_sigma)
    tgt = warp(src, u)
    if noise_sd > 0:
        src = (src + rng.normal(0.0, noise_sd, shape)).astype(np.float32)
        tgt = (tgt + rng.normal(0.0, noise_sd, shape)).astype(np.float32)
    return src, tgt


def bullseye(shape: Shape, radii: Sequence[float], center=None) -> np.ndarray:
    """Nested spheres: intensity alternates 1, 0, 1, ... from the outermost
    radius inwards (TestUtils::GenBullseye, Testing/TestUtils.cxx:17-23)."""
    nz, ny, nx = shape
    if center is None:
        center = ((nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2)
    img = np.zeros(shape, np.float32)
    val = 1.0
    for rad in sorted(radii, reverse=True):
        img[r <= rad] = val
        val = 1.0 - val
    return img


def atlas_subjects(n_subjects: int, seed: int, sizes=(96, 112, 128, 144, 160),
                   n_blobs: int = 24, umax: float = 5.0, grids=None):
    """Uneven-grid atlas inputs: a common blob template, sampled on each
    subject's grid (normalised coordinates), warped by its own smooth
    displacement and scaled by U(0.9, 1.1). Each axis is drawn from `sizes`
    unless `grids` gives every subject's (nx, ny, nz)."""
    rng = rng_for(seed)
    # template blob parameters in normalised [0,1]^3 coordinates
    params = [(rng.uniform(0.15, 0.85, 3), rng.uniform(0.03, 0.07), rng.uniform(0.3, 1.0))
              for _ in range(n_blobs)]
    subjects = []
    for k in range(n_subjects):
        nx, ny, nz = (int(rng.choice(sizes)) for _ in range(3))
        if grids is not None:
            nx, ny, nz = grids[k]
        z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny,
                              (np.arange(nx) + 0.5) / nx, indexing="ij")
        img = np.zeros((nz, ny, nx), np.float64)
        for c, s, a in params:
            img += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
        img = np.clip(img, 0, 1).astype(np.float32)
        u = smooth_displacement((nz, ny, nx), umax, rng)
        img = warp(img, u) * np.float32(rng.uniform(0.9, 1.1))
        subjects.append(img.astype(np.float32))
    return subjects
