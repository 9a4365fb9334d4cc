"""GPU parity: every result of the CUDA path against the CPU oracle.

Bit-exact: hit indices and hit points of ffb_cast / ffb_cast_bruteforce vs the
reference definition (ray_caster/naive_cpu.cpp:65-97, restated in
oracle/ffo.c); emitted rays and the fused per-(source, hit) count matrix vs
the oracle's Philox emission + brute-force cast.
"""
import numpy as np
import pytest

from form_factors_b200 import emission, scenes
import rays as R

pytestmark = pytest.mark.gpu


def _scenes():
    return {
        "plates10": scenes.parallel_plates(10, 1.0),
        "perpendicular": scenes.perpendicular_plates(6),
        "unit_box": scenes.unit_box(),
        "sphere_out": scenes.icosphere(2, 1.0, inward=False),
        "clutter": scenes.clutter(300, 0.05, seed=3, enclosure_cells=5),
    }


def _assert_same_hits(hit, pts, ref_hit, ref_pts, what):
    bad = np.nonzero(hit != ref_hit)[0]
    assert bad.size == 0, "%s: %d/%d hit indices differ, first %s: got %s want %s" % (
        what, bad.size, hit.size, bad[:5], hit[bad[:5]], ref_hit[bad[:5]])
    m = ref_hit >= 0
    assert np.array_equal(pts[m].view(np.uint32), ref_pts[m].view(np.uint32)), what + ": hit points differ"
    assert np.isnan(pts[~m]).all(), what + ": miss points must be NaN"


@pytest.mark.parametrize("name", list(_scenes().keys()))
@pytest.mark.parametrize("skip", [True, False])
def test_cast_grid_matches_naive(ctx, oracle, name, skip):
    faces = _scenes()[name]
    rng = np.random.default_rng(7)
    rays = R.mixed_rays(rng, faces, 6000)
    ref_hit, ref_pts = oracle.cast_naive(faces, rays)
    ctx.scene_set(faces)
    for dims in (None, (1, 1, 1), (16, 16, 16), (37, 5, 23)):
        ctx.grid_build(dims=dims, skip_empty=skip)
        hit, pts = ctx.cast(rays)
        _assert_same_hits(hit, pts, ref_hit, ref_pts, "%s dims=%s skip=%s" % (name, dims, skip))


@pytest.mark.parametrize("name", ["plates10", "unit_box", "clutter"])
def test_cast_bruteforce_matches_naive(ctx, oracle, name):
    faces = _scenes()[name]
    rays = R.mixed_rays(np.random.default_rng(11), faces, 3000)
    ref_hit, ref_pts = oracle.cast_naive(faces, rays)
    ctx.scene_set(faces)
    hit, pts = ctx.cast(rays, brute=True)
    _assert_same_hits(hit, pts, ref_hit, ref_pts, name + " brute")


def test_emitted_rays_bit_exact(ctx, oracle):
    faces = np.concatenate([scenes.parallel_plates(3, 1.0), scenes.clutter(40, 0.05, seed=5, enclosure_cells=2)])
    n = len(faces)
    rng = np.random.default_rng(2)
    front = rng.integers(0, 40, n).astype(np.int32)
    rear = rng.integers(0, 40, n).astype(np.int32)
    ctx.scene_set(faces)
    for flags in (0, 1):
        got = ctx.emit(front, rear, seed=0x1234567890ABCDEF, epoch=3, flags=flags)
        want = oracle.emit(faces, front, rear, seed=0x1234567890ABCDEF, epoch=3, flags=flags)
        assert got.shape == want.shape
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), "flags=%d" % flags


@pytest.mark.parametrize("name", ["plates4", "box", "clutter"])
def test_form_factor_counts_bit_exact(ctx, oracle, name):
    faces = {"plates4": scenes.parallel_plates(4, 1.0), "box": scenes.unit_box(),
             "clutter": scenes.clutter(60, 0.1, seed=9, enclosure_cells=3)}[name]
    n = len(faces)
    w, total = emission.two_sided_weights(faces)
    front, rear = emission.ray_counts(2000 * n, w, total)
    ctx.scene_set(faces)
    ctx.grid_build()
    for flags in (0, 1):
        got = ctx.form_factor_counts(front, rear, seed=77, epoch=1, flags=flags)
        want = oracle.form_factor_counts(faces, front, rear, seed=77, epoch=1, flags=flags)
        assert np.array_equal(got, want), "%s flags=%d: %d entries differ" % (name, flags, (got != want).sum())
        st = ctx.stats()
        assert st.rays == int(front.sum() + rear.sum())
        assert st.hits == int(want.sum())


def test_form_factor_counts_mesh_rows(ctx, oracle):
    faces = scenes.parallel_plates(4, 0.5)
    n = len(faces)
    rows = np.repeat(np.arange(n // 8), 8).astype(np.int32)  # 8 faces per mesh
    front, rear = emission.front_only(n, 500)
    ctx.scene_set(faces)
    ctx.grid_build()
    got = ctx.form_factor_counts(front, rear, seed=5, face_to_row=rows, n_rows=n // 8)
    per_face = oracle.form_factor_counts(faces, front, rear, seed=5)
    m = n // 8
    want = np.zeros((m, m), np.uint64)
    np.add.at(want, (rows[:, None].repeat(n, 1), rows[None, :].repeat(n, 0)), per_face)
    assert np.array_equal(got.astype(np.uint64), want)


def test_wide_matrix_sparse_sources(ctx, oracle):
    """A 10 240-face matrix with few emitting faces: the warp histograms see
    keys spread over a 105 M-entry matrix."""
    faces = scenes.icosphere(4, 1.0, inward=True)  # 5120 faces
    faces = np.concatenate([faces, scenes.transform(faces, shift=(3, 0, 0))])  # 10240 faces
    n = len(faces)
    rng = np.random.default_rng(4)
    front = np.zeros(n, np.int32)
    sel = rng.choice(n, 24, replace=False)
    front[sel] = 300
    rear = np.zeros(n, np.int32)
    ctx.scene_set(faces)
    ctx.grid_build()
    got = ctx.form_factor_counts(front, rear, seed=99)
    want = oracle.form_factor_counts(faces, front, rear, seed=99)
    assert np.array_equal(got, want)


def test_row_blocks_concatenate_to_full_matrix(ctx):
    """Shards of source rows (one per GPU in a multi-GPU run) are independent:
    their blocks concatenate to the full matrix, bit for bit."""
    from form_factors_b200 import shard
    faces = scenes.clutter(200, 0.08, seed=6, enclosure_cells=4)
    n = len(faces)
    w, total = emission.two_sided_weights(faces)
    front, rear = emission.ray_counts(400 * n, w, total)
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=16)
    full = ctx.form_factor_counts(front, rear, seed=12, epoch=3)
    for world in (2, 3):
        blocks = [ctx.form_factor_counts_rows(front, rear, 12, b, e, epoch=3)
                  for b, e in shard.row_ranges(shard.rays_per_row(front, rear), world)]
        assert np.array_equal(np.concatenate(blocks), full)


def test_pipelined_host_output_matches_device_output(ctx):
    """Host outputs of 64 MB and more are traced in row blocks whose copies to
    the host overlap the next block: pageable and pinned host outputs, a row
    sub-range and a permuted face-to-row map give the device output bit for
    bit."""
    import torch
    faces = scenes.icosphere(4, 1.0, inward=True)  # 5120 faces
    faces = np.concatenate([faces, scenes.transform(faces, shift=(0.5, 0, 0))])  # 10240 faces
    n = len(faces)
    rng = np.random.default_rng(8)
    front = rng.integers(0, 40, n).astype(np.int32)
    front[rng.choice(n, 300, replace=False)] = 0
    rear = rng.integers(0, 3, n).astype(np.int32)
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=16)
    dev = torch.empty((n, n), dtype=torch.int32, device="cuda")
    ctx.form_factor_counts(front, rear, seed=31, epoch=2, out=dev)
    ctx.synchronize()
    want = dev.cpu().numpy().view(np.uint32)
    assert want.sum() > 0
    pageable = ctx.form_factor_counts(front, rear, seed=31, epoch=2)
    assert np.array_equal(pageable, want)
    pinned = torch.empty((n, n), dtype=torch.int32, pin_memory=True)
    ctx.form_factor_counts(front, rear, seed=31, epoch=2, out=pinned)
    assert np.array_equal(pinned.numpy().view(np.uint32), want)
    part = ctx.form_factor_counts_rows(front, rear, 31, 1234, 9876, epoch=2)
    assert np.array_equal(part, want[1234:9876])
    perm = rng.permutation(n).astype(np.int32)
    permuted = ctx.form_factor_counts(front, rear, seed=31, epoch=2, face_to_row=perm)
    expect = np.zeros_like(want)
    expect[perm[:, None], perm[None, :]] = want
    assert np.array_equal(permuted, expect)
