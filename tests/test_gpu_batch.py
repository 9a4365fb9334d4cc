"""Batched scenes (ffb_batch_*: one single-scene launch per scene over side
streams, capturable as one CUDA graph) give, scene by scene, exactly the
counts of the single-scene path with the same seed and epoch; a CUDA graph
that captured the launches draws fresh rays on every replay."""
import numpy as np
import pytest

from form_factors_b200 import emission, native, scenes

pytestmark = pytest.mark.gpu


def _scene_list():
    return [scenes.parallel_plates(4, 1.0), scenes.unit_box(), scenes.icosphere(2, 1.0, inward=True),
            scenes.clutter(80, 0.1, seed=4, enclosure_cells=3), scenes.perpendicular_plates(5),
            scenes.icosphere(1, 0.5, inward=False)]


def test_batch_equals_single_scene_path(ctx):
    import torch

    sl = _scene_list()
    rng = np.random.default_rng(3)
    fronts = [rng.integers(50, 700, len(f)).astype(np.int32) for f in sl]
    rears = [rng.integers(0, 300, len(f)).astype(np.int32) for f in sl]
    seeds = np.array([11 + 1000 * i for i in range(len(sl))], np.uint64)
    ctx.batch_set(sl)
    ctx.batch_prepare(np.concatenate(fronts), np.concatenate(rears), seeds)
    offs, words = ctx.batch_counts_layout()
    counts = torch.empty(words, dtype=torch.int32, device="cuda")
    ctx.batch_launch(counts, offs, advance_epoch=True)  # epoch 1
    ctx.synchronize()  # the launch only enqueues on the context stream
    got_all = counts.cpu().numpy().view(np.uint32)
    for i, f in enumerate(sl):
        n = len(f)
        got = got_all[int(offs[i]):int(offs[i]) + n * n].reshape(n, n)
        ctx.scene_set(f)
        ctx.grid_build(cells_per_face=32)
        want = ctx.form_factor_counts(fronts[i], rears[i], seed=int(seeds[i]), epoch=1)
        assert np.array_equal(got, want), "scene %d" % i
        assert got.sum() > 0


def test_batch_graph_replays_draw_fresh_rays(ctx):
    import torch

    sl = _scene_list()[:3]
    fronts = [np.full(len(f), 300, np.int32) for f in sl]
    rears = [np.zeros(len(f), np.int32) for f in sl]
    ctx.batch_set(sl)
    ctx.batch_prepare(np.concatenate(fronts), np.concatenate(rears), np.array([5, 6, 7], np.uint64))
    offs, words = ctx.batch_counts_layout()
    counts = torch.empty(words, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        ctx.batch_launch(counts, offs, advance_epoch=True)
    results = []
    for _ in range(3):
        graph.replay()
        torch.cuda.synchronize()
        results.append(counts.cpu().numpy().copy())
    ctx.set_stream(None)
    # the capture itself does not run the work; replays k = 1, 2, 3 use epochs 1, 2, 3
    assert not np.array_equal(results[0], results[1]) and not np.array_equal(results[1], results[2])
    n0 = len(sl[0])
    ctx.scene_set(sl[0])
    ctx.grid_build(cells_per_face=32)
    for k, res in enumerate(results):
        want = ctx.form_factor_counts(fronts[0], rears[0], seed=5, epoch=k + 1)
        assert np.array_equal(res[:n0 * n0].view(np.uint32).reshape(n0, n0), want)
    del graph
