"""Generates the golden fixtures in this directory from the reference's own
CPU code (oracle/_ref/libffref.so, built from the reference sources by
oracle/Makefile target `ref`).  Run from the repository root:

    python tests/golden/make_golden.py

Fixtures (compressed .npz, all seeded):
  intersect.npz   random rays x triangles -> math::triangle_intersect codes and points
  rotate.npz      random (subject, target) -> math::rotate_towards matrices
  emitted.npz     (n_rays, weight, total) -> malley_emission::emitted_front
  ray_kat.npz     the scenes and rays of the reference's ray-caster tests
                  (test/ray_casting.cpp:46-322) -> naive_cpu and zgrid_cpu hits/points
  cast_plates.npz two 10x10-cell parallel plates, 20 000 rays of the reference's
                  malley_cpu emission -> naive_cpu and zgrid_cpu hits/points
  cast_mixed.npz  a clutter scene and mixed (random / aimed / grazing) rays ->
                  naive_cpu hits/points
  ff_ref.npz      the reference form-factor calculator (cpu_form_factors +
                  malley_cpu + naive_cpu, 40 000 rays) on the test scenes of
                  test/form_factors.cpp:78-186
  csv_ref.npz     a 24 x 24 float matrix of edge values (signed zeros,
                  infinities, NaNs, extremes, subnormals, ties at the seventh
                  digit, count / outgoing ratios, random magnitudes) and the
                  bytes csv_export::export_csv writes for it

  obj_ref.npz     a generated OBJ scene (mixed number and face styles, objects,
                  a material library) and what obj_import::scene returns for it

`python tests/golden/make_golden.py csv` (or `obj`) writes that fixture only.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from form_factors_b200 import scenes  # noqa: E402
from oracle_lib import Reference  # noqa: E402
import rays as R  # noqa: E402


def tri(a, b, c):
    return np.array(a + b + c, np.float32)


def ray_to_triangle(origin, t):
    """math::ray_to_triangle: from origin towards the centre, end at half way."""
    t = np.asarray(t, np.float32).reshape(3, 3)
    center = (t[0] + t[1] + t[2]) / np.float32(3)
    o = np.asarray(origin, np.float32)
    return np.concatenate([o, o + (center - o) / np.float32(2)]).astype(np.float32)


def kat_scenes():
    floor1 = tri([0, 0, 0], [1, 0, 0], [0, 1, 0])
    floor2 = tri([1, 0, 0], [0, 1, 0], [1, 1, 0])
    stack = tri([0, 0, -1], [1, 0, -1], [0, 1, -1])
    floor = np.stack([floor1, floor2])
    stacked = np.stack([floor1, stack])
    large = np.stack([floor1 + np.tile(np.float32([0, 0, 0.1 * i]), 3) for i in range(-500, 500)]).astype(np.float32)

    def center(t):
        return t.reshape(3, 3).mean(0).astype(np.float32)

    out = {}
    # ProcessAllRays / JustWorks: floor scene, rays from +-1 above the centres
    c0, c1 = center(floor[0]), center(floor[1])
    out["floor"] = (floor, np.stack([ray_to_triangle(c0 + np.float32([0, 0, 1]), floor[0]),
                                     ray_to_triangle(c1 + np.float32([0, 0, -1]), floor[1])]))
    # HandleRayIntersectingTriangle, FindNearestTriangle, SkipTriangleNearButInOppositeDirection,
    # IntersectTriganglesNotPlanes: stacked scene
    s0, s1 = center(stacked[0]), center(stacked[1])
    r_intersect = np.concatenate([s0 + np.float32([0, 0, .5]), s0 - np.float32([0, 0, .5])]).astype(np.float32)
    out["stack"] = (stacked, np.stack([r_intersect,
                                       ray_to_triangle(s0 + np.float32([0, 0, 1]), stacked[0]),
                                       ray_to_triangle(s1 + np.float32([0, 0, .9]), stacked[1]),
                                       ray_to_triangle(s1 + np.float32([2, 2, 2]), stacked[1])]))
    # ProcessLargeScene: 1000 stacked floors, ray from the side
    l0 = center(large[0])
    out["large"] = (large, np.stack([ray_to_triangle(l0 + np.float32([2, 2, -2]), large[0])]))
    return out


def csv_matrix(rng):
    """24 x 24 float32 matrix exercising every branch of "%g" formatting."""
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 3.4028235e38, -3.4028235e38,
                        1.17549435e-38, 1e-45, -1e-45, 1e-40, 0.5, 1.0, 100000.0, 999999.0, 999999.5, 1e6,
                        0.0001, 9.99999e-05, 1e-05, 123456.7, 0.1, 1.0 / 3.0], np.float32)
    ties = np.ldexp(np.float32(1.0), np.arange(-149, 128, 3)).astype(np.float32)  # 93 powers of two
    out = rng.integers(1, 5000, 150)
    ratios = (rng.integers(0, 5000, 150) % (out + 1)).astype(np.float32) * (np.float32(1.0) / out.astype(np.float32))
    mags = (rng.standard_normal(309) * np.float32(10.0) ** rng.integers(-40, 38, 309)).astype(np.float32)
    v = np.concatenate([special, ties, ratios.astype(np.float32), mags])[:576]
    return v.reshape(24, 24).astype(np.float32)


def csv_fixture(ref, rng):
    import tempfile
    ff = csv_matrix(rng)
    with tempfile.TemporaryDirectory() as d:
        text = ref.csv_text(ff, d)
    np.savez_compressed(os.path.join(HERE, "csv_ref.npz"), ff=ff, text=np.frombuffer(text, np.uint8))


def obj_fixture(ref):
    import tempfile
    import obj_text as O
    faces = scenes.clutter(60, 0.1, seed=12, enclosure_cells=2)
    meshes = [(0, 20), (20, 30), (50, len(faces) - 50)]
    rng = np.random.default_rng(77)
    mtl = O.mtl_text(["alpha", "beta"], rng).encode()
    obj = O.obj_text(faces, meshes, ["alpha", "beta"], mtllib="golden.mtl", seed=78)
    with tempfile.TemporaryDirectory() as d:
        open(os.path.join(d, "golden.mtl"), "wb").write(mtl)
        path = os.path.join(d, "golden.obj")
        open(path, "wb").write(obj)
        rc, f, m, mats = ref.obj_scene(path)
    assert rc == 0, rc
    np.savez_compressed(os.path.join(HERE, "obj_ref.npz"), obj=np.frombuffer(obj, np.uint8),
                        mtl=np.frombuffer(mtl, np.uint8), faces=f, meshes=m, materials=mats)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "obj":
        obj_fixture(Reference())
        print("obj_ref.npz written to", HERE)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "csv":
        csv_fixture(Reference(), np.random.default_rng(20261204))
        print("csv_ref.npz written to", HERE)
        return
    if not Reference.available():
        sys.exit("oracle/_ref/libffref.so is missing: make -C oracle ref")
    ref = Reference()
    rng = np.random.default_rng(20261203)

    # --- intersect
    n = 4000
    tris = rng.normal(size=(n, 9)).astype(np.float32)
    rays = rng.normal(size=(n, 6)).astype(np.float32)
    # aim half of the rays at their triangle so that hits are frequent
    tgt = tris.reshape(n, 3, 3).mean(1)
    rays[::2, 3:] = tgt[::2] + (rays[::2, 3:] - tgt[::2]) * np.float32(1e-3)
    codes = np.zeros(n, np.int32)
    pts = np.zeros((n, 3), np.float32)
    for i in range(n):
        c, p = ref.triangle_intersect(rays[i], tris[i])
        codes[i], pts[i] = c, p
    np.savez_compressed(os.path.join(HERE, "intersect.npz"), tris=tris, rays=rays, codes=codes, points=pts)

    # --- rotate
    m = 2000
    subj = rng.normal(size=(m, 3)).astype(np.float32)
    subj[::2] = np.float32([0, 0, 1])
    to = (rng.normal(size=(m, 3)) * rng.choice([1e-3, 1.0, 10.0], (m, 1))).astype(np.float32)
    to[5] = [0, 0, -1]
    to[7] = [0, 0, -3]
    to[9] = [0, 0, 1]
    mats = np.stack([ref.rotate_towards(subj[i], to[i]) for i in range(m)])
    np.savez_compressed(os.path.join(HERE, "rotate.npz"), subject=subj, to=to, mats=mats)

    # --- emitted
    args = [(40000, 0.5, 4.0), (40000, 0.5, 20.0), (40000000, 0.005, 4.0), (1000, 1e-9, 1.0), (123, 0.3, 0.7),
            (22080000, 6.1e-4, 29.126305), (7, 0.0, 1.0), (10, -1.0, 1.0), (1000, 1.0, 1.0)]
    em = np.array([ref.emitted(*a) for a in args], np.int32)
    np.savez_compressed(os.path.join(HERE, "emitted.npz"), args=np.array(args, np.float64), counts=em)

    # --- reference ray-caster known answers
    kat = {}
    for name, (faces, rs) in kat_scenes().items():
        h1, p1, _, _ = ref.cast(Reference.NAIVE_CPU, faces, rs)
        h3, p3, _, _ = ref.cast(Reference.ZGRID_CPU, faces, rs)
        kat[name + "_faces"] = faces
        kat[name + "_rays"] = rs
        kat[name + "_naive_hit"] = h1
        kat[name + "_naive_pts"] = p1
        kat[name + "_zgrid_hit"] = h3
    np.savez_compressed(os.path.join(HERE, "ray_kat.npz"), **kat)

    # --- plates with the reference's own emission
    faces = scenes.parallel_plates(10, 1.0)
    w = np.zeros(2 * len(faces), np.float32)
    w[:] = 1.0
    rays_ref = ref.emit(faces, 20000, w, float(2 * len(faces)))
    h1, p1, _, _ = ref.cast(Reference.NAIVE_CPU, faces, rays_ref)
    h3, p3, _, _ = ref.cast(Reference.ZGRID_CPU, faces, rays_ref)
    np.savez_compressed(os.path.join(HERE, "cast_plates.npz"), faces=faces, rays=rays_ref, naive_hit=h1,
                        naive_pts=p1, zgrid_hit=h3, zgrid_pts=p3)

    # --- clutter with mixed rays
    faces = scenes.clutter(200, 0.08, seed=11, enclosure_cells=4)
    rs = R.mixed_rays(np.random.default_rng(5), faces, 6000)
    h1, p1, _, _ = ref.cast(Reference.NAIVE_CPU, faces, rs)
    np.savez_compressed(os.path.join(HERE, "cast_mixed.npz"), faces=faces, rays=rs, naive_hit=h1, naive_pts=p1)

    # --- reference form factors on the test scenes (two-sided, mesh matrices)
    ff = {}
    sq = lambda off: [tri([0, 0, 0], [1, 0, 0], [0, 1, 0]) + np.tile(np.float32(off), 3),
                      tri([1, 0, 0], [1, 1, 0], [0, 1, 0]) + np.tile(np.float32(off), 3)]
    for d in (0.5, 1.0, 2.0):
        faces = np.stack(sq([0, 0, 0]) + sq([0, 0, d])).astype(np.float32)
        meshes = np.array([[0, 2, 0], [2, 2, 0]], np.int32)
        rc, mat = ref.form_factors(faces, meshes, 40000, caster=Reference.NAIVE_CPU)
        assert rc == 0
        ff["parallel_%g_faces" % d] = faces
        ff["parallel_%g_ff" % d] = mat
    wall = [tri([0, 0, 0], [0, 1, 0], [0, 0, 1]), tri([0, 1, 0], [0, 0, 1], [0, 1, 1])]
    faces = np.stack(sq([0, 0, 0]) + wall).astype(np.float32)
    rc, mat = ref.form_factors(faces, np.array([[0, 2, 0], [2, 2, 0]], np.int32), 40000,
                               caster=Reference.NAIVE_CPU)
    ff["perpendicular_faces"] = faces
    ff["perpendicular_ff"] = mat
    faces = scenes.unit_box()
    rc, mat = ref.form_factors(faces, np.array([[0, 12, 0]], np.int32), 40000, caster=Reference.NAIVE_CPU)
    ff["box_faces"] = faces
    ff["box_ff"] = mat
    np.savez_compressed(os.path.join(HERE, "ff_ref.npz"), **ff)
    csv_fixture(ref, np.random.default_rng(20261204))
    obj_fixture(ref)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
