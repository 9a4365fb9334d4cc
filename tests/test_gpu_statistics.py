"""Statistical validation of the form factors (the bar for a Monte Carlo
estimate whose random source differs from the reference's mt19937):

* FP64 analytic view factors of parallel and perpendicular unit squares,
  within 4 sigma of the binomial error sqrt(F (1 - F) / n);
* every matrix entry within 4 sigma of the reference's own calculator
  (cpu_form_factors + malley_cpu, two-sided, raw-normal rotation), on the
  reference's test scenes (golden fixtures) and live on a per-face matrix;
* closed enclosures: every ray of an inward emitter hits something.
"""
import os

import numpy as np
import pytest

from form_factors_b200 import emission, scenes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FOUR_SIGMA = 4.0


def within(a, b, n_a, n_b, k=FOUR_SIGMA):
    f = 0.5 * (a + b)
    sigma = np.sqrt(np.maximum(f * (1 - f), 1e-12) * (1.0 / n_a + 1.0 / n_b))
    return np.abs(a - b) <= k * sigma


def test_config1_parallel_plates_analytic(ctx, oracle):
    """Two unit squares at distance 1, 10x10 cells (200 triangles each),
    100 000 front rays per face, grid 16^3: F01 and F10 against the FP64
    analytic 0.19982 within 4 sigma."""
    faces = scenes.parallel_plates(10, 1.0)
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build(dims=(16, 16, 16))
    rows = np.repeat([0, 1], n // 2).astype(np.int32)
    front, rear = emission.front_only(n, 100_000)
    counts = ctx.form_factor_counts(front, rear, seed=1, face_to_row=rows, n_rows=2).astype(np.float64)
    rays = 100_000 * (n // 2)
    want = oracle.vf_parallel(1, 1, 1)
    sigma = np.sqrt(want * (1 - want) / rays)
    for f in (counts[0, 1] / rays, counts[1, 0] / rays):
        assert abs(f - want) <= FOUR_SIGMA * sigma, (f, want, sigma)
    assert counts[0, 0] == 0 and counts[1, 1] == 0


def test_perpendicular_plates_analytic(ctx, oracle):
    faces = scenes.perpendicular_plates(10)
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build()
    rows = np.repeat([0, 1], n // 2).astype(np.int32)
    front, rear = emission.front_only(n, 50_000)
    counts = ctx.form_factor_counts(front, rear, seed=2, face_to_row=rows, n_rows=2).astype(np.float64)
    rays = 50_000 * (n // 2)
    want = oracle.vf_perpendicular(1, 1, 1)
    sigma = np.sqrt(want * (1 - want) / rays)
    assert abs(counts[0, 1] / rays - want) <= FOUR_SIGMA * sigma
    assert abs(counts[1, 0] / rays - want) <= FOUR_SIGMA * sigma


def _reference_budget(ctx, faces, meshes, n_rays, flags, seed):
    """The reference calculator's semantics on the GPU: two-sided area
    weights, its per-face ray budget, mesh rows, row normalisation."""
    n = len(faces)
    w, total = emission.two_sided_weights(faces)
    front, rear = emission.ray_counts(n_rays, w, total)
    rows = np.zeros(n, np.int32)
    for m, (first, cnt, _) in enumerate(meshes):
        rows[first:first + cnt] = m
    ctx.scene_set(faces)
    ctx.grid_build()
    ff = ctx.form_factors(front, rear, seed=seed, flags=flags, face_to_row=rows, n_rows=len(meshes))
    outgoing = np.zeros(len(meshes), np.int64)
    np.add.at(outgoing, rows, front.astype(np.int64) + rear)
    return ff, outgoing


@pytest.mark.parametrize("case", ["parallel_0.5", "parallel_1", "parallel_2", "perpendicular", "box"])
def test_reference_test_scenes_within_4_sigma_of_reference(ctx, oracle, case):
    """The scenes of test/form_factors.cpp, 40 000 rays, against the matrices
    the reference's own calculator produced (tests/golden/ff_ref.npz)."""
    g = np.load(os.path.join(GOLDEN, "ff_ref.npz"))
    faces = g[case + "_faces"]
    ref = g[case + "_ff"].astype(np.float64)
    meshes = [(0, 12, 0)] if case == "box" else [(0, 2, 0), (2, 2, 0)]
    ff, outgoing = _reference_budget(ctx, faces, meshes, 40000, flags=1, seed=3)
    assert np.all(within(ff.astype(np.float64), ref, outgoing[:, None], outgoing[:, None]))
    # the reference test's own tolerance against half the analytic value
    if case.startswith("parallel"):
        d = float(case.split("_")[1])
        half = oracle.vf_parallel(1, 1, d) / 2
        assert abs(ff[0, 1] - half) < 0.01 and abs(ff[1, 0] - half) < 0.01
    elif case == "perpendicular":
        assert abs(ff[1, 0] - oracle.vf_perpendicular(1, 1, 1) / 2) < 0.01
    else:
        assert abs(ff[0, 0] - 0.5) < 0.01


def test_per_face_matrix_within_4_sigma_of_live_reference(ctx, reference):
    """Per-face meshes (the per-face N x N matrix of the benchmarked
    workloads) on a clutter scene: every entry with enough expected hits within 4 sigma of the
    reference calculator run live (oracle/_ref), raw-normal emission as the
    reference's."""
    faces = scenes.clutter(40, 0.15, seed=8, enclosure_cells=2)
    n = len(faces)
    meshes = np.stack([np.arange(n), np.ones(n, int), np.zeros(n, int)], 1).astype(np.int32)
    n_rays = 2_000_000
    ff, outgoing = _reference_budget(ctx, faces, meshes, n_rays, flags=1, seed=5)
    rc, ref = reference.form_factors(faces, meshes, n_rays, caster=reference.ZGRID_CPU)
    assert rc == 0
    ref = ref.astype(np.float64)
    ff = ff.astype(np.float64)
    rays = outgoing[:, None].astype(np.float64)
    enough = (0.5 * (ff + ref) * rays) >= 30
    assert enough.sum() > 100
    ok = within(ff, ref, rays, rays)
    # 4 sigma: about 6e-5 of the entries may fall outside by chance
    assert (~ok & enough).sum() <= max(2, int(1e-3 * enough.sum())), (~ok & enough).sum()
    # rows sum to the fraction of rays that hit, which closes the box for both
    assert np.allclose(ff.sum(1), ref.sum(1), atol=0.02)


def test_enclosure_rows_sum_to_one(ctx):
    """Inward front-only emission in a closed enclosure: every ray hits."""
    faces = scenes.enclosure(3, 5)
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build()
    front, rear = emission.front_only(n, 2000)
    counts = ctx.form_factor_counts(front, rear, seed=9)
    rows = counts.sum(1, dtype=np.int64)
    assert (rows >= 2000 - 2).all() and rows.sum() >= n * 2000 * (1 - 1e-5)


def test_config3_clutter_bit_exact_with_autotuned_grid(ctx, oracle):
    """2000 random equilateral triangles (edge 0.05) in a 2028-triangle unit
    cube, the grid (32^3..128^3) and the kernel's launch shape chosen by the
    autotuner; the counts stay bit-identical to the oracle whatever it
    picks."""
    faces = scenes.clutter(2000, 0.05, seed=1, enclosure_cells=13)
    n = len(faces)
    front, rear = emission.front_only(n, 12)
    ctx.scene_set(faces)
    best = ctx.autotune(front, rear, seed=3, candidates=[dict(dims=(d, d, d)) for d in (32, 64, 96, 128)],
                        sample_every=4, force=True)
    assert best["dims"][0] in (32, 64, 96, 128) and ctx.trace_shape() == best["shape"]
    got = ctx.form_factor_counts(front, rear, seed=3)
    oracle.set_threads(0)
    want = oracle.form_factor_counts(faces, front, rear, seed=3)
    ctx.set_trace_shape(0)
    assert np.array_equal(got, want)
