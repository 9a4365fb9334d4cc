"""GPU parity of the CSV export (csv_export::export_csv,
import_export/csv_export.cpp:26-46): the text formatted by the CUDA kernels
is byte-identical to the file the reference's own export writes for the same
matrix (oracle/_ref, live) and to the committed golden bytes, through every
entry point: floats or counts, host or device buffers, file, one or several
segments.
"""
import os

import numpy as np
import pytest

from form_factors_b200 import native

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "csv_ref.npz")


def normalised(counts, outgoing):
    """The reference's row normalisation in float32 (cpu_system.cpp:193-195)."""
    ratio = np.float32(1.0) / outgoing.astype(np.float32)
    return (counts.astype(np.float32) * ratio[:, None]).astype(np.float32)


def sparse_counts(rng, n, per_row, rays):
    counts = np.zeros((n, n), np.uint32)
    rows = np.repeat(np.arange(n), per_row)
    cols = rng.integers(0, n, rows.size)
    np.add.at(counts, (rows, cols), rng.integers(1, rays // per_row + 1, rows.size).astype(np.uint32))
    outgoing = np.maximum(counts.sum(1, dtype=np.int64) + rng.integers(0, 50, n), 1).astype(np.int32)
    return counts, outgoing


def test_golden_matrix(ctx):
    g = np.load(GOLDEN)
    assert ctx.csv_format(ff=g["ff"]) == g["text"].tobytes()


def test_random_floats_match_reference_export(ctx, reference, tmp_path):
    rng = np.random.default_rng(11)
    n = 61
    bits = rng.integers(0, 2 ** 32, n * n, dtype=np.uint64).astype(np.uint32)
    ff = bits.view(np.float32).reshape(n, n)
    want = reference.csv_text(ff, tmp_path)
    assert ctx.csv_length(ff=ff) == len(want)
    assert ctx.csv_format(ff=ff) == want


def test_counts_epilogue_equals_normalise_then_format(ctx, reference, tmp_path):
    rng = np.random.default_rng(12)
    counts, outgoing = sparse_counts(rng, 300, 40, 4000)
    want = reference.csv_text(normalised(counts, outgoing), tmp_path)
    assert ctx.csv_format(counts=counts, outgoing=outgoing) == want
    assert ctx.csv_format(ff=ctx.normalise(counts, outgoing)) == want


def test_several_segments_device_and_host_buffers(ctx, reference, tmp_path):
    """4200^2 = 17.6 M entries: two segments of 2^24 entries."""
    import torch
    rng = np.random.default_rng(13)
    n = 4200
    counts, outgoing = sparse_counts(rng, n, 30, 1000)
    want = reference.csv_text(normalised(counts, outgoing), tmp_path)
    d_counts = torch.from_numpy(counts.view(np.int32)).cuda()
    d_out = torch.from_numpy(outgoing).cuda()
    assert ctx.csv_length(counts=d_counts, outgoing=d_out) == len(want)
    dev = torch.empty(len(want) + 64, dtype=torch.uint8, device="cuda")
    n_bytes = ctx.csv_format(counts=d_counts, outgoing=d_out, out=dev)
    assert n_bytes == len(want)
    assert dev[:n_bytes].cpu().numpy().tobytes() == want
    host = np.empty(len(want), np.uint8)
    assert ctx.csv_format(counts=counts, outgoing=outgoing, out=host) == len(want)
    assert host.tobytes() == want


def test_export_files(ctx, reference, tmp_path):
    rng = np.random.default_rng(14)
    counts, outgoing = sparse_counts(rng, 500, 20, 2000)
    ff = normalised(counts, outgoing)
    want = reference.csv_text(ff, tmp_path)
    p1, p2 = str(tmp_path / "a.csv"), str(tmp_path / "b.csv")
    ctx.csv_export(p1, ff=ff)
    ctx.csv_export(p2, counts=counts, outgoing=outgoing)
    assert open(p1, "rb").read() == want
    assert open(p2, "rb").read() == want


def test_export_large_file_pipelined(ctx, reference, tmp_path):
    """A multi-segment export: the host writes one segment while the GPU
    formats the next."""
    rng = np.random.default_rng(15)
    counts, outgoing = sparse_counts(rng, 4500, 10, 500)
    want = reference.csv_text(normalised(counts, outgoing), tmp_path)
    p = str(tmp_path / "big.csv")
    ctx.csv_export(p, counts=counts, outgoing=outgoing)
    assert os.path.getsize(p) == len(want)
    assert open(p, "rb").read() == want


def test_empty_matrix_and_errors(ctx, reference, tmp_path):
    p = str(tmp_path / "empty.csv")
    ctx.csv_export(p, ff=np.zeros((0, 0), np.float32))
    assert os.path.getsize(p) == 0
    assert reference.export_csv(str(tmp_path / "ref_empty.csv"), np.zeros((0, 0), np.float32)) == 0
    bad = str(tmp_path / "no_such_dir" / "x.csv")
    with pytest.raises(native.FFBError) as e:
        ctx.csv_export(bad, ff=np.ones((2, 2), np.float32))
    assert e.value.code == -309
    assert reference.export_csv(bad, np.ones((2, 2), np.float32)) == -31  # -CSV_EXPORT_FILE_ERROR
    small = np.empty(5, np.uint8)
    with pytest.raises(native.FFBError) as e:
        ctx.csv_format(ff=np.ones((4, 4), np.float32), out=small)
    assert e.value.code == -301
