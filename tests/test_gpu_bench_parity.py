"""Bit-exact parity at the benchmarked configurations.

The closed enclosure the bench times -- an inward icosphere of 20 480
triangles holding two perpendicular 20x20 plates, N = 22 080 faces, 1000
front rays per face -- traced through the grid the bench uses (192 cells per
face, 162^3, per-octant empty-space jumps) and through the library default
(32 cells per face).  A sample of 200 source faces spread over the sphere
and both plates emits its full 1000 rays each (200 000 rays): every hit
index and hit point must equal the oracle's brute-force cast
(ray_caster/naive_cpu.cpp:65-97), and the fused kernel's count rows of those
faces must equal the rows the oracle tallies from its own emission and
brute-force hits (cpuFactorsCalculator/cpu_system.cpp:167-196).

The occluded-clutter configuration (2000 equilateral triangles of edge 0.05
in a 2028-triangle unit cube) is checked the same way at its stated
10 000 rays per face on a subset of 40 source faces, through the grid the
autotuner picks.
"""
import numpy as np
import pytest

from form_factors_b200 import scenes

pytestmark = pytest.mark.gpu

SEED = 0x5EED


def _sample_faces(n, n_sphere, k_sphere=180, k_plates=20):
    sphere = np.linspace(0, n_sphere - 1, k_sphere).astype(np.int64)
    plates = np.linspace(n_sphere, n - 1, k_plates).astype(np.int64)
    return np.unique(np.concatenate([sphere, plates]))


def _oracle_rows(oracle, faces, front, rear, sel, seed, epoch):
    """Rows `sel` of the per-face count matrix from the oracle's Philox
    emission (packed face by face, front then rear) and brute-force hits."""
    rays = oracle.emit(faces, front, rear, seed=seed, epoch=epoch)
    hit, pts = oracle.cast_naive(faces, rays)
    per_face = (front.astype(np.int64) + rear)
    src = np.repeat(np.arange(len(faces)), per_face)
    row_of = np.full(len(faces), -1, np.int64)
    row_of[sel] = np.arange(len(sel))
    rows = np.zeros((len(sel), len(faces)), np.uint32)
    m = hit >= 0
    np.add.at(rows, (row_of[src[m]], hit[m]), 1)
    return rays, hit, pts, rows


def _assert_same_hits(hit, pts, ref_hit, ref_pts, what):
    bad = np.nonzero(hit != ref_hit)[0]
    assert bad.size == 0, "%s: %d/%d hit indices differ, first %s: got %s want %s" % (
        what, bad.size, hit.size, bad[:5], hit[bad[:5]], ref_hit[bad[:5]])
    m = ref_hit >= 0
    assert np.array_equal(pts[m].view(np.uint32), ref_pts[m].view(np.uint32)), what + ": hit points differ"
    assert np.isnan(pts[~m]).all(), what + ": miss points must be NaN"


def _device_rows(ctx, front, rear, sel, seed, epoch, n):
    import torch
    counts = torch.empty((n, n), dtype=torch.int32, device="cuda")
    ctx.form_factor_counts(front, rear, seed, epoch=epoch, out=counts, n_rows=n)
    ctx.synchronize()
    rows = counts[torch.from_numpy(sel).cuda()].cpu().numpy().view(np.uint32)
    total = int(counts.sum(dtype=torch.int64).item())
    del counts
    torch.cuda.empty_cache()
    return rows, total


@pytest.fixture(scope="module")
def enclosure_case(oracle):
    faces = scenes.enclosure(5, 20)
    n = len(faces)
    assert n == 22080
    sel = _sample_faces(n, n - 1600)
    front = np.zeros(n, np.int32)
    front[sel] = 1000
    rear = np.zeros(n, np.int32)
    oracle.set_threads(0)
    rays, hit, pts, rows = _oracle_rows(oracle, faces, front, rear, sel, SEED, 7)
    return faces, front, rear, sel, rays, hit, pts, rows


@pytest.mark.parametrize("cells_per_face", [192.0, 32.0])
def test_enclosure_hits_bit_exact_at_bench_grid(ctx, enclosure_case, cells_per_face):
    faces, front, rear, sel, rays, ref_hit, ref_pts, _ = enclosure_case
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=cells_per_face, skip_empty=True)
    info = ctx.grid_info()
    if cells_per_face == 192.0:
        assert (info.nx, info.ny, info.nz) == (162, 162, 162)
    got_rays = ctx.emit(front, rear, seed=SEED, epoch=7)
    assert np.array_equal(got_rays.view(np.uint32), rays.view(np.uint32)), "emitted rays differ from the oracle"
    hit, pts = ctx.cast(rays)
    _assert_same_hits(hit, pts, ref_hit, ref_pts, "enclosure cpf=%g" % cells_per_face)
    assert (ref_hit >= 0).mean() > 0.999  # a closed enclosure: (almost) every ray lands


@pytest.mark.parametrize("cells_per_face", [192.0, 32.0])
def test_enclosure_count_rows_bit_exact_at_bench_grid(ctx, enclosure_case, cells_per_face):
    faces, front, rear, sel, _, ref_hit, _, ref_rows = enclosure_case
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=cells_per_face, skip_empty=True)
    ctx.set_stats(False)  # the bench's timed kernel variant (no counters)
    try:
        rows, total = _device_rows(ctx, front, rear, sel, SEED, 7, n)
    finally:
        ctx.set_stats(True)
    assert total == int((ref_hit >= 0).sum()), "hits outside the sampled rows"
    bad = np.argwhere(rows != ref_rows)
    assert bad.size == 0, "%d count entries differ, first %s" % (len(bad), bad[:5])


def test_clutter_config_bit_exact_at_stated_rays(ctx, oracle):
    """Occluded clutter at 10 000 rays per face (40 source faces, 20 of the
    clutter triangles and 20 of the cube), grid autotuned over 32^3-128^3."""
    faces = scenes.clutter(2000, 0.05, seed=1, enclosure_cells=13)
    n = len(faces)
    sel = np.unique(np.concatenate([np.linspace(0, 1999, 20), np.linspace(2000, n - 1, 20)]).astype(np.int64))
    front = np.zeros(n, np.int32)
    rear = np.zeros(n, np.int32)
    front[sel] = 5000
    rear[sel] = 5000
    ctx.scene_set(faces)
    best = ctx.autotune_grid(front, rear, seed=3,
                             candidates=[dict(dims=(d, d, d)) for d in (32, 64, 96, 128)], sample_every=1)
    assert best["dims"][0] in (32, 64, 96, 128)
    oracle.set_threads(0)
    rays, ref_hit, ref_pts, ref_rows = _oracle_rows(oracle, faces, front, rear, sel, 3, 2)
    hit, pts = ctx.cast(rays)
    _assert_same_hits(hit, pts, ref_hit, ref_pts, "clutter autotuned %s" % (best["dims"],))
    rows, total_hits = _device_rows(ctx, front, rear, sel, 3, 2, n)
    assert total_hits == int((ref_hit >= 0).sum())
    assert np.array_equal(rows, ref_rows)
