"""GPU parity of the ray-traced thermal equations.

Bit-exact against the oracle (same Philox rays, brute-force cast):
* disc emission of the distant source (emission/parallel_rays_cpu.cpp:88-106);
* per-(face, side) hit tallies of the parallel rays
  (thermal_equation/parallel_rays_cpu.cpp:110-122);
* the radiance equation's absorbed power per mesh in 64-bit fixed point
  (thermal_equation/radiance_cpu.cpp:142-180).
Against the reference itself (oracle/_ref, the reference's radiance_cpu and
parallel_rays_cpu equations over its naive_cpu caster):
* emission per mesh of the radiance step, float for float;
* absorbed power per mesh within 4 sigma, sigma measured from GPU runs with
  independent rays (the two use different random sources).
"""
import numpy as np
import pytest

from form_factors_b200 import native, scenes

pytestmark = pytest.mark.gpu

BOX_MESHES = [(0, 2, 0), (2, 2, 0), (4, 2, 1), (6, 2, 1), (8, 2, 0), (10, 2, 0)]
BOX_MATERIALS = [(0.9, 0.5, 0.8, 0.3), (0.4, 1.0, 0.6, 0.9)]  # emissivity front/rear, absorbance front/rear
BOX_TEMPS = np.array([300, 350, 400, 310, 320, 330], np.float32)


def _sources():
    return [([0.3, -0.2, -1.0], [0.5, 0.5, 0.5], 3.0, 1.2),   # not normalised, as the reference allows
            ([0.0, 0.0, 1.0], [0.0, 0.0, 0.0], 2.0, 1.0),     # +z: identity rotation
            ([0.0, 0.0, -1.0], [0.1, 0.2, 0.3], 2.5, 0.7),    # -z: the reflection branch
            ([1.0, 2.0, 0.5], [0.4, 0.6, 0.5], 4.0, 2.0)]


@pytest.mark.parametrize("k", range(4))
def test_disc_emission_bit_exact(ctx, oracle, k):
    direction, center, distance, radius = _sources()[k]
    got = ctx.emit_parallel(native.DiscSource.make(direction, center, distance, radius), 5000, seed=17, epoch=2)
    want = oracle.emit_parallel(oracle.disc_source(direction, center, distance, radius), 5000, seed=17, epoch=2)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", ["box", "clutter", "sphere"])
def test_parallel_ray_tallies_bit_exact(ctx, oracle, name):
    faces = {"box": scenes.unit_box(), "clutter": scenes.clutter(300, 0.08, seed=2, enclosure_cells=3),
             "sphere": scenes.icosphere(3, 1.0, inward=False)}[name]
    ctx.scene_set(faces)
    center, r = native.bounding_sphere(faces)
    for k, (direction, _, _, _) in enumerate(_sources()):
        src = (direction, center, 1.1 + 1.1 * r, 1.1 * r)
        want = oracle.parallel_rays(faces, oracle.disc_source(*src), 40000, seed=5, epoch=k)
        for dims, skip in ((None, True), ((7, 9, 5), False)):
            ctx.grid_build(dims=dims, skip_empty=skip)
            got = ctx.parallel_rays(native.DiscSource.make(*src), 40000, seed=5, epoch=k)
            assert np.array_equal(got, want), (name, k, dims)
        assert want.sum() > 1000


def test_radiance_absorption_bit_exact(ctx, oracle):
    faces = scenes.clutter(200, 0.1, seed=4, enclosure_cells=3)
    n = len(faces)
    rng = np.random.default_rng(8)
    front = rng.integers(0, 60, n).astype(np.int32)
    rear = rng.integers(0, 30, n).astype(np.int32)
    pf = (rng.random(n) * 10).astype(np.float32)
    pr = (rng.random(n) * 3).astype(np.float32)
    pr[::7] = 0
    f2m = (np.arange(n) // 13).astype(np.int32)
    n_m = int(f2m.max()) + 1
    ctx.scene_set(faces)
    ctx.grid_build()
    for flags in (0, 1):
        got = ctx.radiance_absorption(front, rear, pf, pr, f2m, n_m, seed=21, epoch=4, flags=flags)
        want = oracle.radiance_absorption(faces, front, rear, pf, pr, f2m, n_m, seed=21, epoch=4, flags=flags)
        assert np.array_equal(got, want)
        assert got.sum() > 0


def test_radiance_step_emission_equals_reference(ctx, reference):
    """The step's emission per mesh equals the reference's, float for float."""
    faces = scenes.unit_box()
    ctx.scene_set(faces)
    ctx.grid_build()
    em, _ = ctx.radiance_step(faces, BOX_MESHES, BOX_MATERIALS, BOX_TEMPS, 100000, seed=3)
    rc, ref_em, _ = reference.radiance(faces, BOX_MESHES, BOX_MATERIALS, BOX_TEMPS, 1000, caster=1)
    assert rc == 0
    assert np.array_equal(em, ref_em)


def test_radiance_step_conserves_energy_in_a_closed_enclosure(ctx):
    """Inward normals and no rear emission: every ray lands inside, so the
    absorbed total equals the emitted one, but for the few rays in 10^4 that
    float rounding lets through the seams where two walls meet (the brute-force
    definition, and the reference's casters, lose them the same way)."""
    faces = scenes.unit_cube_enclosure(3)  # 6 sides of 18 faces
    meshes = [(18 * k, 18, k % 2) for k in range(6)]
    materials = [(0.9, 0.0, 1.0, 1.0), (0.5, 0.0, 1.0, 1.0)]
    ctx.scene_set(faces)
    ctx.grid_build()
    em, ab = ctx.radiance_step(faces, meshes, materials, [300, 320, 340, 360, 380, 400], 200000, seed=3)
    assert 0 <= 1 - float(ab.sum()) / float(em.sum()) < 2e-4


def _gpu_runs(fn, k):
    return np.stack([fn(epoch) for epoch in range(k)])


def test_radiance_step_within_4_sigma_of_reference(ctx, reference):
    faces = scenes.unit_box()
    ctx.scene_set(faces)
    ctx.grid_build()
    n_rays = 200000
    runs = _gpu_runs(lambda e: ctx.radiance_step(faces, BOX_MESHES, BOX_MATERIALS, BOX_TEMPS, n_rays, seed=9,
                                                 epoch=e)[1], 16).astype(np.float64)
    rc, _, ref = reference.radiance(faces, BOX_MESHES, BOX_MATERIALS, BOX_TEMPS, n_rays, caster=1)
    assert rc == 0
    sigma = runs.std(0, ddof=1)
    assert np.all(np.abs(runs.mean(0) - ref) <= 4 * sigma * np.sqrt(1 + 1 / len(runs)) + 1e-3 * np.abs(ref).max())


def test_distant_source_within_4_sigma_of_reference(ctx, reference):
    faces = scenes.clutter(120, 0.15, seed=6, enclosure_cells=0)
    n = len(faces)
    meshes = [(i * 10, 10, i % 2) for i in range(n // 10)]
    ctx.scene_set(faces)
    ctx.grid_build()
    n_rays, power, direction = 200000, 1361.0, [0.3, -0.4, -0.8]
    runs = _gpu_runs(lambda e: ctx.distant_source_step(faces, meshes, BOX_MATERIALS, n_rays, power, direction,
                                                       seed=10, epoch=e), 16).astype(np.float64)
    rc, ref = reference.parallel_rays(faces, meshes, BOX_MATERIALS, n_rays, power, direction, caster=1)
    assert rc == 0
    assert runs.mean(0).sum() > 0
    sigma = runs.std(0, ddof=1)
    assert np.all(np.abs(runs.mean(0) - ref) <= 4 * sigma * np.sqrt(1 + 1 / len(runs)) + 1e-3 * np.abs(ref).max())


def test_thermal_steps_reject_bad_meshes(ctx):
    faces = scenes.unit_box()
    ctx.scene_set(faces)
    ctx.grid_build()
    with pytest.raises(native.FFBError):
        ctx.radiance_step(faces, [(0, 6, 0)], BOX_MATERIALS, [300.0], 1000, seed=1)  # faces 6..11 in no mesh
    with pytest.raises(native.FFBError):
        ctx.distant_source_step(faces, [(0, 12, 5)], BOX_MATERIALS, 1000, 1.0, [0, 0, 1], seed=1)  # no material 5
