"""Seeded synthetic 8-bit sRGB images for the analysis-stage workloads.

No public image set is available offline, so every workload uses images drawn
from one generator with the statistics the workloads call for:

* a sum of 1/f^alpha colour noise, alpha uniform in [1.5, 2.5] (alpha is the
  exponent of the power spectrum, so amplitudes fall as f^(-alpha/2));
* linear gradients and Gaussian blobs;
* 0-40 random filled polygons with hard edges;
* a per-image saturation uniform in [0, 1];
* optional per-pixel Gaussian sensor noise, sigma uniform in [0.5, 3] DN;
* quantisation to uint8.

The same seed always gives the same image (numpy's PCG64 generator).
"""

from __future__ import annotations

import numpy as np

__all__ = ["generate_srgb8", "workload_seed"]


def workload_seed(config_id: int, image_index: int = 0) -> int:
    """Seed convention: config_id * 10**6 + image_index."""
    return int(config_id) * 1_000_000 + int(image_index)


def _colour_noise(rng: np.random.Generator, height: int, width: int) -> np.ndarray:
    """Three independent 1/f^alpha noise planes, each scaled to [0, 1]."""
    alpha = rng.uniform(1.5, 2.5)
    fy = np.fft.fftfreq(height).astype(np.float32)[:, None]
    fx = np.fft.rfftfreq(width).astype(np.float32)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    amplitude = f ** (-alpha / 2.0)
    amplitude[0, 0] = 0.0
    planes = []
    for _ in range(3):
        spectrum = (rng.standard_normal(amplitude.shape, dtype=np.float32)
                    + 1j * rng.standard_normal(amplitude.shape, dtype=np.float32))
        plane = np.fft.irfft2(spectrum * amplitude, s=(height, width)).astype(np.float32)
        lo, hi = np.percentile(plane[:: max(1, height // 256), :: max(1, width // 256)], [1, 99])
        plane = (plane - lo) / max(hi - lo, 1e-6)
        planes.append(np.clip(plane, 0.0, 1.0))
    return np.stack(planes, axis=-1)


def _fill_polygon(image: np.ndarray, vertices: np.ndarray, colour: np.ndarray) -> None:
    """Even-odd scanline fill at pixel centres, vectorised over rows."""
    height, width, _ = image.shape
    y0 = max(int(np.floor(vertices[:, 1].min())), 0)
    y1 = min(int(np.ceil(vertices[:, 1].max())), height - 1)
    if y1 < y0:
        return
    ys = np.arange(y0, y1 + 1, dtype=np.float64) + 0.5
    a = vertices
    b = np.roll(vertices, -1, axis=0)
    ay, by = a[:, 1][None, :], b[:, 1][None, :]
    ax, bx = a[:, 0][None, :], b[:, 0][None, :]
    yy = ys[:, None]
    crosses = ((ay <= yy) & (by > yy)) | ((by <= yy) & (ay > yy))
    with np.errstate(divide="ignore", invalid="ignore"):
        xs = ax + (yy - ay) * (bx - ax) / (by - ay)
    xs = np.where(crosses, xs, np.inf)
    xs.sort(axis=1)
    rows = y1 - y0 + 1
    diff = np.zeros((rows, width + 1), dtype=np.int32)
    for k in range(0, xs.shape[1] - 1, 2):
        start, end = xs[:, k], xs[:, k + 1]
        valid = np.isfinite(start) & np.isfinite(end)
        if not valid.any():
            continue
        s = np.clip(np.ceil(start[valid] - 0.5), 0, width).astype(np.int64)
        e = np.clip(np.ceil(end[valid] - 0.5), 0, width).astype(np.int64)
        r = np.nonzero(valid)[0]
        np.add.at(diff, (r, s), 1)
        np.add.at(diff, (r, e), -1)
    mask = np.cumsum(diff[:, :width], axis=1) > 0
    region = image[y0:y1 + 1]
    region[mask] = colour


def generate_srgb8(width: int, height: int, seed: int, sensor_noise: bool = False) -> np.ndarray:
    """Returns a (height, width, 3) uint8 sRGB image."""
    rng = np.random.default_rng(seed)
    image = _colour_noise(rng, height, width)

    # Linear gradients.
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float32)
    for _ in range(int(rng.integers(1, 4))):
        angle = rng.uniform(0, 2 * np.pi)
        t = (np.cos(angle) * xx / width + np.sin(angle) * yy / height)
        t = (t - t.min()) / max(float(t.max() - t.min()), 1e-6)
        c0 = rng.uniform(0, 1, 3).astype(np.float32)
        c1 = rng.uniform(0, 1, 3).astype(np.float32)
        weight = rng.uniform(0.2, 0.6)
        gradient = c0[None, None, :] + t[..., None] * (c1 - c0)[None, None, :]
        image = (1 - weight) * image + weight * gradient

    # Gaussian blobs.
    for _ in range(int(rng.integers(0, 12))):
        cx, cy = rng.uniform(0, width), rng.uniform(0, height)
        sigma = rng.uniform(0.02, 0.2) * min(width, height)
        x0, x1 = int(max(cx - 3 * sigma, 0)), int(min(cx + 3 * sigma, width))
        y0, y1 = int(max(cy - 3 * sigma, 0)), int(min(cy + 3 * sigma, height))
        if x1 <= x0 or y1 <= y0:
            continue
        gx = np.exp(-0.5 * ((np.arange(x0, x1) - cx) / sigma) ** 2).astype(np.float32)
        gy = np.exp(-0.5 * ((np.arange(y0, y1) - cy) / sigma) ** 2).astype(np.float32)
        g = (gy[:, None] * gx[None, :])[..., None] * rng.uniform(0.3, 0.9)
        colour = rng.uniform(0, 1, 3).astype(np.float32)
        image[y0:y1, x0:x1] = (1 - g) * image[y0:y1, x0:x1] + g * colour

    # Hard-edged polygons.
    for _ in range(int(rng.integers(0, 41))):
        n = int(rng.integers(3, 9))
        cx, cy = rng.uniform(0, width), rng.uniform(0, height)
        radius = rng.uniform(0.02, 0.25) * min(width, height)
        angles = np.sort(rng.uniform(0, 2 * np.pi, n))
        radii = radius * rng.uniform(0.4, 1.0, n)
        vertices = np.stack([cx + radii * np.cos(angles), cy + radii * np.sin(angles)], axis=1)
        _fill_polygon(image, vertices, rng.uniform(0, 1, 3).astype(np.float32))

    # Per-image saturation.
    saturation = rng.uniform(0.0, 1.0)
    luma = image @ np.array([0.2126, 0.7152, 0.0722], dtype=np.float32)
    image = luma[..., None] + saturation * (image - luma[..., None])

    image = np.clip(image, 0.0, 1.0) * 255.0
    if sensor_noise:
        sigma = rng.uniform(0.5, 3.0)
        image = image + rng.standard_normal(image.shape, dtype=np.float32) * sigma
    return np.clip(np.rint(image), 0, 255).astype(np.uint8)
