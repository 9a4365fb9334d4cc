"""Count matrices written to host buffers in row blocks (64 MB and more).

Each finished row block is packed on the device to the (column, count) pairs
of its nonzero entries; the pairs cross PCIe and host threads expand them
into the caller's rows with streaming stores, while the next block traces.
A block with more nonzeros than a quarter of its entries is copied dense.
Whatever the path, the host matrix must equal the device-resident output
of the same call bit for bit: pageable and pinned buffers, a destination
that is not 16-byte aligned, a row width that is not a multiple of four,
blocks without emitting faces, dense blocks, one host thread or several,
and host threads 0 (every block copied dense).  The device output itself is
pinned to the oracle by the parity tests.
"""
import numpy as np
import pytest

from form_factors_b200 import scenes

pytestmark = pytest.mark.gpu

SEED = 77


def _device(ctx, front, rear, epoch, rows=None, face_to_row=None, n_rows=None):
    import torch
    n = n_rows or ctx.n_faces
    b, e = rows if rows else (0, n)
    out = torch.empty((e - b, n), dtype=torch.int32, device="cuda")
    ctx.form_factor_counts_rows(front, rear, SEED, b, e, epoch=epoch, face_to_row=face_to_row, n_rows=n, out=out)
    ctx.synchronize()
    assert ctx.stats().d2h_bytes == 0
    return out.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def scene():
    faces = scenes.enclosure(4, 12)  # 5120 + 576 = 5696 faces: rows of 22 784 bytes
    return faces


@pytest.mark.parametrize("threads,wide", [(-1, False), (1, False), (3, False), (0, False), (-1, True)])
def test_packed_output_equals_device_output(ctx, scene, threads, wide):
    """wide: one row emits 70 000 rays, so a count may pass 2^16 and pairs
    take two words (column, count) instead of one."""
    import torch
    n = len(scene)
    assert 4 * n * n >= 64 << 20
    ctx.scene_set(scene)
    ctx.grid_build(cells_per_face=64, skip_empty=True)
    front = np.full(n, 30, np.int32)
    if wide:
        front[17] = 70000
    rear = np.zeros(n, np.int32)
    want = _device(ctx, front, rear, epoch=4)
    assert want.any()
    ctx.set_host_threads(threads)
    try:
        pageable = np.full((n, n), 0xDEADBEEF, np.uint32)
        ctx.form_factor_counts(front, rear, SEED, epoch=4, out=pageable)
        d2h = ctx.stats().d2h_bytes
        assert np.array_equal(pageable, want)
        pinned = torch.full((n, n), -1, dtype=torch.int32, pin_memory=True)
        ctx.form_factor_counts(front, rear, SEED, epoch=4, out=pinned)
        assert np.array_equal(pinned.numpy().view(np.uint32), want)
    finally:
        ctx.set_host_threads(-1)
    if threads == 0:
        assert d2h == 4 * n * n
    else:
        nnz = int(np.count_nonzero(want))
        pair = 8 if wide else 4
        assert pair * nnz < d2h < pair * nnz + 16 * n + 4096, "pairs plus block headers"


def test_unaligned_destination_and_odd_width(ctx):
    """A destination 4 bytes past a 16-byte boundary, and a row width that is
    not a multiple of four (head and tail words of every row)."""
    import torch
    faces = scenes.enclosure(4, 11)  # 5120 + 484 = 5604 faces
    faces = faces[:-1]               # 5603: odd width
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=64, skip_empty=True)
    front = np.full(n, 25, np.int32)
    rear = np.full(n, 2, np.int32)
    want = _device(ctx, front, rear, epoch=6)
    raw = torch.full((n * n + 3,), -1, dtype=torch.int32, pin_memory=True)
    for shift in (1, 2, 3):
        view = raw[shift:shift + n * n]
        assert view.data_ptr() % 16 != 0
        ctx.form_factor_counts(front, rear, SEED, epoch=6, out=view)
        assert np.array_equal(view.numpy().view(np.uint32).reshape(n, n), want), shift


def test_blocks_without_emitters_and_row_ranges(ctx, scene):
    """Row ranges whose blocks include ones where no face emits (all-zero
    rows written by the host threads), and sparse emitters."""
    n = len(scene)
    ctx.scene_set(scene)
    ctx.grid_build(cells_per_face=64, skip_empty=True)
    front = np.zeros(n, np.int32)
    front[:1500] = 40  # only the first rows emit: the second of the two row blocks has no emitting face
    rear = np.zeros(n, np.int32)
    want = _device(ctx, front, rear, epoch=8)
    got = np.full((n, n), 0xDEADBEEF, np.uint32)
    ctx.form_factor_counts(front, rear, SEED, epoch=8, out=got)
    assert np.array_equal(got, want)
    assert not got[1500:].any()
    front[4000:4003] = 500  # a few dense rows among empty ones
    want = _device(ctx, front, rear, epoch=8)
    part = ctx.form_factor_counts_rows(front, rear, SEED, 700, n, epoch=8)
    assert np.array_equal(part, want[700:])


def test_dense_matrices_and_dense_blocks(ctx):
    """A matrix whose rays could fill more than a quarter of its entries is
    copied dense as a whole; when only some rows are dense, a block whose
    pairs pass its cap is copied dense and the others come packed."""
    faces = scenes.icosphere(4, 1.0, inward=True)  # 5120 faces, 105 MB matrix
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=32, skip_empty=True)
    front = np.full(n, 12000, np.int32)
    rear = np.zeros(n, np.int32)
    want = _device(ctx, front, rear, epoch=1)
    assert np.count_nonzero(want) > n * n / 4
    got = ctx.form_factor_counts(front, rear, SEED, epoch=1)
    assert np.array_equal(got, want)
    assert ctx.stats().d2h_bytes == 4 * n * n
    # 1000 dense rows: within the global bound, but the first block (1 706
    # rows, half-size) holds them all and passes its own cap
    front[:] = 0
    front[:1000] = 12000
    want = _device(ctx, front, rear, epoch=2)
    got = ctx.form_factor_counts(front, rear, SEED, epoch=2)
    assert np.array_equal(got, want)
    d2h = ctx.stats().d2h_bytes
    assert 4 * 1706 * n <= d2h < 4 * 1706 * n + 16 * n + 4096, "block 0 dense, block 1 empty pairs"


def test_mesh_rows_host_output(ctx, scene):
    """Rows as meshes (face_to_row): several faces add into one row."""
    n = len(scene)
    ctx.scene_set(scene)
    ctx.grid_build(cells_per_face=64, skip_empty=True)
    rng = np.random.default_rng(3)
    m = 4200
    face_to_row = rng.integers(0, m, n).astype(np.int32)
    front = np.full(n, 20, np.int32)
    rear = np.zeros(n, np.int32)
    want = _device(ctx, front, rear, epoch=2, face_to_row=face_to_row, n_rows=m)
    got = ctx.form_factor_counts(front, rear, SEED, epoch=2, face_to_row=face_to_row, n_rows=m)
    assert np.array_equal(got, want)


def _same_floats(got, want):
    """Bit-identical floats, except that a NaN may have any NaN's bits (the
    device's 0 * inf and the host's differ in sign and payload)."""
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    assert np.array_equal(got[~nan].view(np.uint32), want[~nan].view(np.uint32))


@pytest.mark.parametrize("threads", [-1, 0])
def test_normalised_host_output(ctx, scene, threads):
    """ffb_form_factors into a host float matrix: the nonzero counts cross
    PCIe packed and host threads write (float)count * (1.f / outgoing[m]),
    the device normalisation's operations; rows without outgoing rays are
    0 * inf = NaN on both paths."""
    import torch
    n = len(scene)
    ctx.scene_set(scene)
    ctx.grid_build(cells_per_face=64, skip_empty=True)
    front = np.full(n, 30, np.int32)
    front[::97] = 0  # rows with no outgoing rays
    rear = np.zeros(n, np.int32)
    outgoing = (front + rear).astype(np.int32)
    dev = torch.empty((n, n), dtype=torch.float32, device="cuda")
    ctx.form_factors(front, rear, SEED, epoch=5, outgoing=outgoing, out=dev)
    ctx.synchronize()
    want = dev.cpu().numpy()
    assert np.isnan(want[0]).all() and not np.isnan(want[1]).any()
    ctx.set_host_threads(threads)
    try:
        got = np.full((n, n), 7.0, np.float32)
        ctx.form_factors(front, rear, SEED, epoch=5, outgoing=outgoing, out=got)
        d2h = ctx.stats().d2h_bytes
    finally:
        ctx.set_host_threads(-1)
    _same_floats(got, want)
    if threads != 0:
        assert d2h < n * n, "pairs, not the dense matrix"


def test_normalised_host_output_dense_blocks_and_meshes(ctx, scene):
    """A block of a normalised host output whose pairs pass its cap is
    normalised on the device and copied dense; mesh rows (face_to_row) take
    the packed path."""
    faces = scenes.icosphere(4, 1.0, inward=True)
    n = len(faces)
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=32, skip_empty=True)
    front = np.zeros(n, np.int32)
    front[:1000] = 12000
    front[3000:] = 40
    rear = np.zeros(n, np.int32)
    want = ctx.form_factors(front, rear, SEED, epoch=1, out=_device_floats(n))
    ctx.synchronize()
    got = ctx.form_factors(front, rear, SEED, epoch=1)
    _same_floats(got, want.cpu().numpy())
    d2h = ctx.stats().d2h_bytes
    assert 4 * 1706 * n <= d2h < 4 * n * n, "block 0 (1 706 rows) dense, block 1 as pairs"
    n = len(scene)
    ctx.scene_set(scene)
    ctx.grid_build(cells_per_face=64, skip_empty=True)
    rng = np.random.default_rng(9)
    m = 4300
    face_to_row = rng.integers(0, m, n).astype(np.int32)
    front = np.full(n, 25, np.int32)
    rear = np.full(n, 3, np.int32)
    want = ctx.form_factors(front, rear, SEED, epoch=3, face_to_row=face_to_row, n_rows=m, out=_device_floats(m))
    ctx.synchronize()
    got = ctx.form_factors(front, rear, SEED, epoch=3, face_to_row=face_to_row, n_rows=m)
    _same_floats(got, want.cpu().numpy())


def _device_floats(n):
    import torch
    return torch.empty((n, n), dtype=torch.float32, device="cuda")


def test_host_threads_setting(ctx):
    """-1 is the default (min(12, hardware threads)), 0 to 256 are taken as
    given, anything else is refused with FFB_ERR_ARG."""
    import os
    from form_factors_b200 import native
    assert ctx.host_threads() == min(12, os.cpu_count())
    for n in (0, 1, 256):
        ctx.set_host_threads(n)
        assert ctx.host_threads() == n
    for bad in (-2, 257):
        with pytest.raises(native.FFBError) as err:
            ctx.set_host_threads(bad)
        assert err.value.code == -301
    ctx.set_host_threads(-1)
    assert ctx.host_threads() == min(12, os.cpu_count())
