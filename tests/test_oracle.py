"""CPU tests: the oracle against the reference's golden vectors and the live
reference build, the host-side ray budgeting, the scenes, and the C ABI
library's exports.  No GPU needed."""
import os

import numpy as np
import pytest

from form_factors_b200 import emission, native, scenes
import rays as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


# --------------------------------------------------------------------------
# the oracle against the committed golden vectors (made from the reference)
# --------------------------------------------------------------------------
def test_intersect_matches_golden(oracle):
    g = golden("intersect.npz")
    hits = 0
    for ray, tri, code, pt in zip(g["rays"], g["tris"], g["codes"], g["points"]):
        c, p = oracle.triangle_intersect(ray, tri)
        assert c == code
        if c == 0:
            hits += 1
            assert np.array_equal(bits(p), bits(pt))
    assert hits > 100


def test_rotate_towards_matches_golden(oracle):
    g = golden("rotate.npz")
    for s, t, m in zip(g["subject"], g["to"], g["mats"]):
        assert np.array_equal(bits(oracle.rotate_towards(s, t)), bits(m))


def test_emitted_matches_golden(oracle):
    g = golden("emitted.npz")
    for (n, w, t), k in zip(g["args"], g["counts"]):
        assert oracle.emitted(int(n), np.float32(w), np.float32(t)) == k
        assert emission.emitted(int(n), [np.float32(w)], np.float32(t))[0] == k


@pytest.mark.parametrize("name", ["floor", "stack", "large"])
def test_ray_caster_known_answers(oracle, name):
    """The reference's ray-caster tests (test/ray_casting.cpp:154-322): hit
    points are the triangle centres, the nearest of a stack wins, a face
    behind the origin is skipped."""
    g = golden("ray_kat.npz")
    faces, rays = g[name + "_faces"], g[name + "_rays"]
    hit, pts = oracle.cast_naive(faces, rays)
    assert np.array_equal(hit, g[name + "_naive_hit"])
    assert np.array_equal(hit, g[name + "_zgrid_hit"])
    assert np.array_equal(bits(pts), bits(g[name + "_naive_pts"]))
    # near_enough(hit_point, centre) of the reference tests (squared distance < 1e-8)
    f = faces.reshape(-1, 3, 3)
    for h, p in zip(hit, pts):
        c = f[h].mean(0)
        assert ((p - c) ** 2).sum() < 1e-8


@pytest.mark.parametrize("name", ["cast_plates.npz", "cast_mixed.npz"])
def test_naive_cast_matches_golden(oracle, name):
    g = golden(name)
    hit, pts = oracle.cast_naive(g["faces"], g["rays"])
    assert np.array_equal(hit, g["naive_hit"])
    m = hit >= 0
    assert m.sum() > 100
    assert np.array_equal(bits(pts[m]), bits(g["naive_pts"][m]))
    if "zgrid_hit" in g.files:  # the reference's grid caster agrees with its brute force here
        assert np.array_equal(g["zgrid_hit"], g["naive_hit"])


def test_philox_known_answers(oracle):
    """Published Random123 known-answer vectors for philox4x32-10."""
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, want in kat:
        assert list(oracle.philox(ctr, key)) == want


def test_sincos_turn24_accuracy(oracle):
    ks = np.concatenate([np.arange(0, 1 << 24, 4099), [0, 1, (1 << 21) - 1, 1 << 21, (1 << 22), (1 << 24) - 1]])
    for k in ks:
        s, c = oracle.sincos_turn24(int(k))
        a = 2 * np.pi * k / (1 << 24)
        assert abs(s - np.sin(a)) < 4e-7 and abs(c - np.cos(a)) < 4e-7


def test_emission_is_cosine_weighted(oracle):
    """Mean cos(theta) of Malley directions is 2/3 for any triangle size with
    the normalised normal; the raw normal (reference) is only right for |n| = 1."""
    big = np.array([[0, 0, 0, 3, 0, 0, 0, 0, 3]], np.float32)  # n = (0, -9, 0)
    n = 20000
    for flags, ok in ((0, True), (1, False)):
        rays = oracle.emit(big, [n], [0], seed=3, flags=flags)
        d = rays[:, 3:] - rays[:, :3]
        cos = -d[:, 1] / np.linalg.norm(d, axis=1)
        assert (abs(cos.mean() - 2 / 3) < 0.01) == ok


# --------------------------------------------------------------------------
# the oracle against the live reference build (when present)
# --------------------------------------------------------------------------
def test_intersect_matches_reference_random(oracle, reference):
    rng = np.random.default_rng(1)
    for _ in range(3000):
        tri = rng.normal(size=9).astype(np.float32)
        ray = rng.normal(size=6).astype(np.float32)
        if rng.random() < 0.5:
            ray[3:] = tri.reshape(3, 3).mean(0) + (ray[3:] - tri.reshape(3, 3).mean(0)) * 1e-3
        a, b = oracle.triangle_intersect(ray, tri), reference.triangle_intersect(ray, tri)
        assert a[0] == b[0]
        if a[0] == 0:
            assert np.array_equal(bits(a[1]), bits(b[1]))


def test_naive_matches_oracle_on_mixed_rays(oracle, reference):
    faces = scenes.enclosure(3, 6)
    rays = R.mixed_rays(np.random.default_rng(2), faces, 3000)
    hit, pts = oracle.cast_naive(faces, rays)
    h1, p1, _, _ = reference.cast(reference.NAIVE_CPU, faces, rays)
    assert np.array_equal(hit, h1)
    m = hit >= 0
    assert np.array_equal(bits(pts[m]), bits(p1[m]))


def test_zgrid_matches_oracle_on_emitted_rays(oracle, reference):
    """The reference's zgrid_cpu asserts on rays that start outside its XY
    grid (math/grid.cpp:85-86), so it is compared on emission rays only, whose
    origins lie on the faces."""
    faces = scenes.enclosure(3, 6)
    n = len(faces)
    rays = oracle.emit(faces, np.full(n, 3, np.int32), np.full(n, 2, np.int32), seed=8)
    hit, _ = oracle.cast_naive(faces, rays, want_points=False)
    h3, _, _, _ = reference.cast(reference.ZGRID_CPU, faces, rays, threads=4)
    assert (hit >= 0).mean() > 0.5
    assert np.array_equal(hit, h3)


def test_ray_budget_matches_reference(reference):
    faces = scenes.clutter(50, 0.05, seed=1, enclosure_cells=3)
    w, total = emission.two_sided_weights(faces)
    for n_rays in (1000, 40000, 1234567):
        fr, re = emission.ray_counts(n_rays, w, total)
        for f in range(0, len(faces), 7):
            assert fr[f] == reference.emitted(n_rays, w[2 * f], total)
            assert re[f] == reference.emitted(n_rays, w[2 * f + 1], total)


def test_reference_form_factors_match_golden(reference):
    g = golden("ff_ref.npz")
    faces = g["box_faces"]
    rc, mat = reference.form_factors(faces, np.array([[0, 12, 0]], np.int32), 40000, caster=reference.NAIVE_CPU)
    assert rc == 0 and np.array_equal(mat, g["box_ff"])


# --------------------------------------------------------------------------
# analytic view factors and the reference's recorded results
# --------------------------------------------------------------------------
def test_analytic_view_factors(oracle):
    assert abs(oracle.vf_parallel(1, 1, 1) - 0.199825) < 1e-5
    assert abs(oracle.vf_perpendicular(1, 1, 1) - 0.200044) < 1e-5


def test_reference_matrices_near_half_analytic(oracle):
    """The reference's two-sided F is half the textbook view factor
    (cpu_system.cpp:121-129,193-195; test/form_factors.cpp:195)."""
    g = golden("ff_ref.npz")
    for d in (0.5, 1.0, 2.0):
        ff = g["parallel_%g_ff" % d]
        want = oracle.vf_parallel(1, 1, d) / 2
        assert abs(ff[0, 1] - want) < 0.01 and abs(ff[1, 0] - want) < 0.01
    assert abs(g["perpendicular_ff"][1, 0] - oracle.vf_perpendicular(1, 1, 1) / 2) < 0.01
    assert abs(g["box_ff"][0, 0] - 0.5) < 0.01


# --------------------------------------------------------------------------
# scenes and the library boundary
# --------------------------------------------------------------------------
def test_scenes_shapes_and_orientation():
    enc = scenes.enclosure(5, 20)
    assert enc.shape == (22080, 9)
    s = enc[:20480].reshape(-1, 3, 3).astype(np.float64)
    n = np.cross(s[:, 1] - s[:, 0], s[:, 2] - s[:, 0])
    assert (np.einsum("ij,ij->i", n, s.mean(1)) < 0).all()  # inward
    cl = scenes.clutter(2000, 0.05, seed=1)
    assert cl.shape == (2000 + 2028, 9)
    p = cl.reshape(-1, 3)
    assert p.min() >= -1e-6 and p.max() <= 1 + 1e-6
    pp = scenes.parallel_plates(10, 1.0).reshape(-1, 3, 3)
    nz = np.cross(pp[:, 1] - pp[:, 0], pp[:, 2] - pp[:, 0])[:, 2]
    assert (nz[:200] > 0).all() and (nz[200:] < 0).all()


def test_library_exports_every_declared_symbol():
    from form_factors_b200 import build
    build.build()
    lib = native.load()
    declared = native.declared_symbols()
    assert "ffb_cast" in declared and "ffb_form_factor_counts" in declared
    for name in declared:
        assert hasattr(lib, name), name


def test_context_creation_fails_cleanly_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from form_factors_b200 import build
    build.build()
    with pytest.raises(native.FFBError) as e:
        native.Context(0)
    assert e.value.code == -307
