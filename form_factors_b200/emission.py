"""Per-face ray budgeting of the reference, in float32 exactly as it rounds.

* weights: two per face (front, rear), both the face area
  (cpuFactorsCalculator/cpu_system.cpp:121-129)
* total weight: sequential float sum of 2*area (cpu_system.cpp:126)
* rays per side: max(1, (int)(n_rays * (w / total))) when w > 0
  (emission/malley_emission.cpp:50-60)
"""
import numpy as np


def face_areas(faces):
    """math::triangle_area (math/triangle.cpp:86-92): sqrtf(dot(n, n)) / 2 in float32."""
    f = np.ascontiguousarray(faces, np.float32).reshape(-1, 3, 3)
    u = f[:, 1] - f[:, 0]
    v = f[:, 2] - f[:, 0]
    n = np.stack([u[:, 1] * v[:, 2] - u[:, 2] * v[:, 1],
                  u[:, 2] * v[:, 0] - u[:, 0] * v[:, 2],
                  u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]], 1)
    dd = (n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]
    return np.sqrt(dd).astype(np.float32) / np.float32(2)


def two_sided_weights(faces, total_start=0.0):
    """(weights2, total): front and rear weight = area; total accumulates
    2*area face by face in float32 from total_start."""
    a = face_areas(faces)
    w = np.repeat(a, 2).astype(np.float32)
    steps = np.concatenate([[np.float32(total_start)], (np.float32(2) * a).astype(np.float32)])
    total = np.cumsum(steps, dtype=np.float32)[-1]
    return w, np.float32(total)


def emitted(n_rays, weights, total):
    """Vector form of malley_emission::emitted_front/rear."""
    w = np.asarray(weights, np.float32)
    k = (np.float32(n_rays) * (w / np.float32(total))).astype(np.float32)
    with np.errstate(invalid="ignore"):
        k = np.trunc(k)
    k = np.where(np.isfinite(k), k, 0).astype(np.int64)
    out = np.where(w > 0, np.maximum(1, k), 0)
    return out.astype(np.int32)


def ray_counts(n_rays, weights2, total):
    """(front, rear) int32 ray counts per face from interleaved weights."""
    w = np.asarray(weights2, np.float32).reshape(-1, 2)
    return emitted(n_rays, w[:, 0], total), emitted(n_rays, w[:, 1], total)


def front_only(n_faces, rays_per_face):
    """Front-only emission with a fixed count per face (one-sided semantics)."""
    return (np.full(n_faces, rays_per_face, np.int32), np.zeros(n_faces, np.int32))
