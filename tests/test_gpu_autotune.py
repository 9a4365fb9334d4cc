"""The autotuner (ffb_autotune, ffb_batch_autotune) and the fused kernel's
launch shapes: every shape gives the same counts bit for bit, the tuner's
choice is applied and cached, and counts after tuning equal the oracle's.
Reference tuning for comparison: math/grid.cpp:376-386 (grid side only) with
a fixed 128-thread block (cuda_ray_caster/system.cu:61)."""
import numpy as np
import pytest

from form_factors_b200 import emission, native, scenes

pytestmark = pytest.mark.gpu


def test_every_launch_shape_gives_identical_counts(ctx, oracle):
    shapes = native.trace_shapes()
    assert len(shapes) >= 6 and shapes[0]["blocks_per_sm"] == 8
    # a 2 560-face sphere (6.5 M matrix entries: one reduction per hit) and a
    # 200-face clutter (a small matrix: the warp histograms)
    for faces in (scenes.icosphere(3, 1.0, inward=True), scenes.clutter(90, 0.1, seed=4, enclosure_cells=2)):
        n = len(faces)
        w, total = emission.two_sided_weights(faces)
        front, rear = emission.ray_counts(300 * n, w, total)
        ctx.scene_set(faces)
        ctx.grid_build(cells_per_face=64)
        want = oracle.form_factor_counts(faces, front, rear, seed=17, epoch=2)
        for v in range(len(shapes)):
            ctx.set_trace_shape(v)
            assert ctx.trace_shape() == v
            got = ctx.form_factor_counts(front, rear, seed=17, epoch=2)
            assert np.array_equal(got, want), "shape %d (%s): %d entries differ" % (v, shapes[v], (got != want).sum())
        ctx.set_trace_shape(0)
    with pytest.raises(native.FFBError):
        ctx.set_trace_shape(len(shapes))


def test_autotune_applies_and_caches_its_choice(ctx, oracle):
    faces = scenes.clutter(400, 0.06, seed=8, enclosure_cells=5)
    n = len(faces)
    front, rear = emission.front_only(n, 700)
    ctx.scene_set(faces)
    first = ctx.autotune(front, rear, seed=5, force=True)
    assert not first["from_cache"] and first["timed"] == 5 + len(native.trace_shapes()) - 1
    assert 0 < first["sample_rays"] <= n * 700
    assert ctx.trace_shape() == first["shape"]
    info = ctx.grid_info()
    assert abs(info.nx * info.ny * info.nz / n - first["cells_per_face"]) < 0.6 * first["cells_per_face"] + 8
    again = ctx.autotune(front, rear, seed=5)
    assert again["from_cache"] and again["timed"] == 0
    assert again["shape"] == first["shape"] and again["cells_per_face"] == first["cells_per_face"]
    got = ctx.form_factor_counts(front, rear, seed=6)
    want = oracle.form_factor_counts(faces, front, rear, seed=6)
    assert np.array_equal(got, want)
    ctx.set_trace_shape(0)


def test_batch_autotune_matches_single_scene_counts(ctx):
    import torch
    sl = [scenes.parallel_plates(6, 1.0), scenes.icosphere(3, 1.0, inward=True),
          scenes.clutter(150, 0.08, seed=2, enclosure_cells=4)]
    rpf = [400, 150, 300]
    fronts = [np.full(len(f), r, np.int32) for f, r in zip(sl, rpf)]
    rears = [np.zeros(len(f), np.int32) for f in sl]
    seeds = np.array([11, 12, 13], np.uint64)
    ctx.batch_set(sl, cells_per_face=32)
    shapes = ctx.batch_autotune(np.concatenate(fronts), np.concatenate(rears))
    assert len(shapes) == 3 and all(0 <= v < len(native.trace_shapes()) for v in shapes)
    ctx.batch_prepare(np.concatenate(fronts), np.concatenate(rears), seeds)
    offs, words = ctx.batch_counts_layout()
    counts = torch.empty(words, dtype=torch.int32, device="cuda")
    ctx.batch_launch(counts, offs, advance_epoch=False)
    ctx.synchronize()
    got = counts.cpu().numpy().view(np.uint32)
    for i, f in enumerate(sl):
        n = len(f)
        ctx.scene_set(f)
        ctx.grid_build(cells_per_face=32)
        want = ctx.form_factor_counts(fronts[i], rears[i], seed=int(seeds[i]), epoch=0)
        assert np.array_equal(got[int(offs[i]):int(offs[i]) + n * n].reshape(n, n), want), "scene %d" % i
