"""Row sharding of the form-factor matrix across ranks (one process per GPU).

Source rows are independent (the per-source-face loop of
cpuFactorsCalculator/cpu_system.cpp:167-196 splits by source without any
exchange): rank r traces only the rays of the faces whose row falls in its
contiguous block and owns those rows of the matrix; nothing is exchanged
while tracing.  Blocks are balanced by the rays they emit.  When a rank
needs the whole matrix, `gather_rows` assembles the blocks with one
all_gather of padded row blocks (NCCL between GPUs, gloo on CPU).
`solve_rows` is the per-rank step of a sharded solve; on a GPU rank its
rows function is Context.form_factor_counts_rows.
"""
import numpy as np


def row_ranges(rays_per_row, world):
    """Contiguous [begin, end) row blocks, one per rank, each with about the
    same number of rays; every row belongs to exactly one block and no block
    is empty while there are at least `world` rows."""
    w = np.asarray(rays_per_row, np.float64)
    n = len(w)
    if world < 1:
        raise ValueError("world must be >= 1")
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        b = max(b, bounds[-1] + (1 if bounds[-1] < n else 0))
        b = min(b, n - (world - r)) if n >= world else min(b, n)
        bounds.append(max(b, bounds[-1]))
    bounds.append(n)
    return [(bounds[i], bounds[i + 1]) for i in range(world)]


def rays_per_row(front, rear, face_to_row=None, n_rows=None):
    f = np.asarray(front, np.int64) + np.asarray(rear, np.int64)
    if face_to_row is None:
        return f
    out = np.zeros(n_rows if n_rows is not None else int(np.max(face_to_row)) + 1, np.int64)
    np.add.at(out, np.asarray(face_to_row), f)
    return out


def gather_rows(block, begin, end, n_rows, group=None):
    """All ranks: returns the full (n_rows, n_cols) matrix assembled from every
    rank's rows [begin, end) block (a torch tensor on the rank's device, or on
    CPU for gloo)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    meta = torch.tensor([begin, end], dtype=torch.int64, device=block.device)
    metas = [torch.zeros_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    rows_max = max(int(m[1] - m[0]) for m in metas)
    n_cols = block.shape[1]
    pad = torch.zeros((rows_max, n_cols), dtype=block.dtype, device=block.device)
    pad[: end - begin] = block
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    full = torch.empty((n_rows, n_cols), dtype=block.dtype, device=block.device)
    for m, part in zip(metas, parts):
        b, e = int(m[0]), int(m[1])
        full[b:e] = part[: e - b]
    return full


def rank_rows(front, rear, rank, world, face_to_row=None, n_rows=None):
    """This rank's [begin, end) block of source rows, balanced by rays."""
    return row_ranges(rays_per_row(front, rear, face_to_row, n_rows), world)[rank]


def solve_rows(rows_fn, front, rear, rank, world, n_rows, face_to_row=None, gather=False, group=None):
    """The per-rank step of a row-sharded solve.  rows_fn(begin, end) returns
    the (end - begin, n_rows) count block of this rank's source rows (on a GPU
    rank: Context.form_factor_counts_rows into a device tensor); no data
    moves between ranks while it runs.  With gather=True every rank then
    receives the full matrix through one all_gather.  Returns
    ((begin, end), block or full matrix)."""
    begin, end = rank_rows(front, rear, rank, world, face_to_row, n_rows)
    block = rows_fn(begin, end)
    if not gather:
        return (begin, end), block
    return (begin, end), gather_rows(block, begin, end, n_rows, group)
