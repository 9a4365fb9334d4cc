"""Seeded synthetic scenes for the form-factor workloads.

Faces are float32 arrays of shape (n, 9): three vertices per triangle, the
36-byte ``math::triangle_t`` layout of the reference (math/types.h:51-54).
Meshes are int32 arrays of shape (m, 3): ``{first_idx, n_faces, padding}``
(form_factors/system.h:33-39).

Workloads:
* ``parallel_plates``      two coaxial unit squares (plate grid layout of
                           subject/objects.cpp:52-77), normals facing each other
* ``perpendicular_plates`` two unit squares sharing an edge
* ``icosphere``            subdivided icosahedron, inward or outward normals
* ``enclosure``            icosphere (subdivision 5, 20 480 triangles, inward)
                           holding two perpendicular 1x1 plates of 20x20 cells
* ``clutter``              random equilateral triangles in a unit-cube enclosure
* ``unit_box``             the 12-triangle closed box of test/form_factors.cpp:150-186
"""
import math

import numpy as np


def plate_grid(width=1.0, height=1.0, cells_x=10, cells_y=10):
    """Two triangles per cell, normals +z: (A, B, D) and (C, D, B), cells in
    the order of subject/objects.cpp:52-77 (i outer, j inner), float32 steps."""
    sx, sy = np.float32(width / cells_x), np.float32(height / cells_y)
    i, j = np.meshgrid(np.arange(cells_x), np.arange(cells_y), indexing="ij")
    x = (sx * i.astype(np.float32)).ravel()
    y = (sy * j.astype(np.float32)).ravel()
    z = np.zeros_like(x)
    A = np.stack([x, y, z], 1)
    B = np.stack([x + sx, y, z], 1)
    C = np.stack([x + sx, y + sy, z], 1)
    D = np.stack([x, y + sy, z], 1)
    out = np.empty((cells_x * cells_y * 2, 9), np.float32)
    out[0::2] = np.concatenate([A, B, D], 1)
    out[1::2] = np.concatenate([C, D, B], 1)
    return out


def flip(faces):
    """Reverse the winding (swap vertices 1 and 2), flipping the normal."""
    f = faces.reshape(-1, 3, 3).copy()
    f[:, [1, 2]] = f[:, [2, 1]]
    return f.reshape(-1, 9)


def transform(faces, rot=None, shift=(0, 0, 0)):
    p = faces.reshape(-1, 3).astype(np.float64)
    if rot is not None:
        p = p @ np.asarray(rot, np.float64).T
    p = p + np.asarray(shift, np.float64)
    return p.astype(np.float32).reshape(-1, 9)


def parallel_plates(cells=10, distance=1.0):
    """Bottom plate at z=0 facing +z, top plate at z=distance facing -z."""
    bottom = plate_grid(1, 1, cells, cells)
    top = transform(flip(bottom), shift=(0, 0, distance))
    return np.concatenate([bottom, top])


def perpendicular_plates(cells=10):
    """Floor z=0 facing +z over [0,1]^2 and wall x=0 facing +x over y,z in [0,1]."""
    floor = plate_grid(1, 1, cells, cells)
    # map (x, y, 0) -> (0, y, x): normal +z -> +x after the winding flip
    rot = np.array([[0, 0, 0], [0, 1, 0], [1, 0, 0]], np.float64)
    wall = flip(transform(floor, rot=rot))
    return np.concatenate([floor, wall])


def per_face_meshes(n):
    m = np.zeros((n, 3), np.int32)
    m[:, 0] = np.arange(n)
    m[:, 1] = 1
    return m


def icosphere(subdivisions=5, radius=1.0, inward=True, center=(0, 0, 0)):
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius + np.asarray(center, np.float64)
    F = np.array(faces)
    tri = V[F].reshape(-1, 9).astype(np.float32)  # outward winding
    return flip(tri) if inward else tri


def enclosure(subdivisions=5, plate_cells=20):
    """Closed enclosure: inward icosphere of radius 1 around two perpendicular
    1x1 plates (plate_cells x plate_cells cells each) that share an edge."""
    sphere = icosphere(subdivisions, 1.0, inward=True)
    plates = transform(perpendicular_plates(plate_cells), shift=(-0.5, -0.5, -0.5))
    return np.concatenate([sphere, plates])


def random_rotations(rng, n):
    """Uniform rotations on SO(3) from uniform unit quaternions (Shoemake)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], 1)
    x, y, z, w = q.T
    R = np.empty((n, 3, 3))
    R[:, 0] = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], 1)
    R[:, 1] = np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], 1)
    R[:, 2] = np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1)
    return R


def unit_cube_enclosure(cells=13):
    """Unit cube [0,1]^3 of 6*cells^2*2 triangles with inward normals."""
    base = plate_grid(1, 1, cells, cells)  # z=0 plane
    ryz = np.array([[0, 0, 1], [0, 1, 0], [1, 0, 0]], np.float64)  # (x,y,z)->(z,y,x): x=0 plane
    rxz = np.array([[1, 0, 0], [0, 0, 1], [0, 1, 0]], np.float64)  # (x,y,z)->(x,z,y): y=0 plane
    sides = [base, transform(base, shift=(0, 0, 1)),
             transform(base, rot=ryz), transform(base, rot=ryz, shift=(1, 0, 0)),
             transform(base, rot=rxz), transform(base, rot=rxz, shift=(0, 1, 0))]
    return _orient_inward(np.concatenate(sides), center=(0.5, 0.5, 0.5))


def _orient_inward(faces, center):
    f = faces.reshape(-1, 3, 3).astype(np.float64)
    n = np.cross(f[:, 1] - f[:, 0], f[:, 2] - f[:, 0])
    c = f.mean(1)
    outward = np.einsum("ij,ij->i", n, c - np.asarray(center)) > 0
    out = faces.copy()
    out[outward] = flip(faces[outward])
    return out


def clutter(n_tris=2000, edge=0.05, seed=1, enclosure_cells=13):
    """n_tris random equilateral triangles (centres uniform in the unit cube,
    uniform orientation) inside a unit-cube enclosure with inward normals
    (enclosure_cells = 0: no enclosure)."""
    rng = np.random.default_rng(seed)
    r = edge / math.sqrt(3.0)
    ang = np.array([0, 2 * math.pi / 3, 4 * math.pi / 3])
    local = np.stack([r * np.cos(ang), r * np.sin(ang), np.zeros(3)], 1)  # (3, 3)
    R = random_rotations(rng, n_tris)
    centers = rng.random((n_tris, 3))
    # keep whole triangles inside the box
    centers = r + centers * (1 - 2 * r)
    pts = np.einsum("nij,kj->nki", R, local) + centers[:, None, :]
    tris = pts.reshape(-1, 9).astype(np.float32)
    if enclosure_cells <= 0:
        return tris
    return np.concatenate([tris, unit_cube_enclosure(enclosure_cells)])


def unit_box():
    """The closed unit box of test/form_factors.cpp:150-186 (one mesh)."""
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
                 np.float32)
    idx = {0: (0, 1, 2), 1: (0, 3, 2), 8: (0, 1, 5), 9: (0, 4, 5), 4: (0, 3, 7), 5: (0, 4, 7), 6: (1, 2, 6),
           7: (1, 5, 6), 2: (3, 2, 6), 3: (3, 7, 6), 10: (4, 5, 6), 11: (4, 7, 6)}
    out = np.zeros((12, 9), np.float32)
    for k, (a, b, c) in idx.items():
        out[k] = np.concatenate([v[a], v[b], v[c]])
    return out


def uv_sphere(n_lat, n_lon, radius=1.0, inward=True, center=(0, 0, 0)):
    """Latitude/longitude sphere of 2 * n_lon * (n_lat - 1) triangles (one
    triangle per polar quad, two elsewhere), no degenerate faces."""
    th = np.linspace(0, np.pi, n_lat + 1)
    ph = np.linspace(0, 2 * np.pi, n_lon + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    V = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1) * radius + np.asarray(center)
    tris = []
    j = np.arange(n_lon)
    tris.append(np.stack([V[0, j], V[1, j + 1], V[1, j]], 1))               # north cap
    for i in range(1, n_lat - 1):
        tris.append(np.stack([V[i, j], V[i, j + 1], V[i + 1, j + 1]], 1))
        tris.append(np.stack([V[i, j], V[i + 1, j + 1], V[i + 1, j]], 1))
    tris.append(np.stack([V[n_lat - 1, j], V[n_lat - 1, j + 1], V[n_lat, j]], 1))  # south cap
    out = np.concatenate(tris).reshape(-1, 9).astype(np.float32)
    out = _orient_inward(out, center)
    return out if inward else flip(out)


def family_scene(family, n_target, rng):
    """A scene of about n_target triangles of one family: 'plates' (two
    parallel plate grids at distance 1), 'sphere' (inward UV sphere) or
    'clutter' (random equilateral triangles in a unit-cube enclosure)."""
    n_target = max(int(n_target), 24)
    if family == "plates":
        k = max(1, int(round(np.sqrt(n_target / 4.0))))
        return parallel_plates(k, 1.0)
    if family == "sphere":
        n_lon = max(4, int(round(np.sqrt(n_target))))
        n_lat = max(3, int(round(n_target / (2.0 * n_lon))) + 1)
        return uv_sphere(n_lat, n_lon, 1.0, inward=True)
    k = max(1, int(round(np.sqrt(n_target / 48.0))))  # enclosure: a quarter of the faces
    n_c = max(1, n_target - 12 * k * k)
    return clutter(n_c, 0.05, seed=int(rng.integers(1 << 31)), enclosure_cells=k)


def batch_workload(n_scenes=256, n_min=200, n_max=20000, rays_min=1000, rays_max=10000, seed=4):
    """Batched workload: triangle counts log-uniform in [n_min, n_max], the
    three families in turn, rays per face uniform in [rays_min, rays_max].
    Returns (list of faces arrays, rays per face per scene)."""
    rng = np.random.default_rng(seed)
    fams = ("plates", "sphere", "clutter")
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_scenes))
    rays = rng.integers(rays_min, rays_max + 1, n_scenes)
    out = [family_scene(fams[i % 3], sizes[i], rng) for i in range(n_scenes)]
    return out, rays.astype(np.int64)


def areas(faces):
    f = faces.reshape(-1, 3, 3).astype(np.float32)
    u = f[:, 1] - f[:, 0]
    v = f[:, 2] - f[:, 0]
    n = np.cross(u, v)
    return np.sqrt((n * n).sum(1)) / 2
