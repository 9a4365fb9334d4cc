"""Seeded ray batches for parity tests (rays are {origin, end point})."""
import numpy as np


def random_rays(rng, n, lo, hi):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    return np.concatenate([o, o + d], 1).astype(np.float32)


def aimed_rays(rng, faces, n, spread=1.0):
    """Rays from random points toward vertices, edge midpoints and centres of
    random faces: the places where shared edges produce equal distances and
    the lowest-index rule decides."""
    f = faces.reshape(-1, 3, 3).astype(np.float64)
    idx = rng.integers(0, len(f), n)
    kind = rng.integers(0, 3, n)
    vert = f[idx, rng.integers(0, 3, n)]
    mid = 0.5 * (f[idx, rng.integers(0, 3, n)] + f[idx, (rng.integers(0, 3, n))])
    cen = f[idx].mean(1)
    target = np.where(kind[:, None] == 0, vert, np.where(kind[:, None] == 1, mid, cen))
    c = f.reshape(-1, 3).mean(0)
    o = c + rng.normal(size=(n, 3)) * spread
    return np.concatenate([o, target], 1).astype(np.float32)


def grazing_rays(rng, faces, n, eps=1e-3):
    """Rays nearly parallel to the plane of random faces."""
    f = faces.reshape(-1, 3, 3).astype(np.float64)
    idx = rng.integers(0, len(f), n)
    p = f[idx]
    u = p[:, 1] - p[:, 0]
    v = p[:, 2] - p[:, 0]
    nrm = np.cross(u, v)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    a, b = rng.random((2, n))
    inside = p[:, 0] + a[:, None] * 0.5 * u + b[:, None] * 0.5 * v
    d = u / np.linalg.norm(u, axis=1, keepdims=True) + eps * rng.normal(size=(n, 1)) * nrm
    o = inside - d * rng.uniform(0.5, 2.0, (n, 1)) + nrm * eps * rng.normal(size=(n, 1))
    return np.concatenate([o, o + d], 1).astype(np.float32)


def scene_box(faces):
    p = faces.reshape(-1, 3)
    return p.min(0), p.max(0)


def mixed_rays(rng, faces, n):
    lo, hi = scene_box(faces)
    pad = 0.25 * (hi - lo).max()
    k = n // 3
    return np.concatenate([random_rays(rng, k, lo - pad, hi + pad), aimed_rays(rng, faces, k),
                           grazing_rays(rng, faces, n - 2 * k)])
