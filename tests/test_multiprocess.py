"""Row sharding across ranks (the multi-GPU path): balanced contiguous row
blocks, and the per-rank step shard.solve_rows -- the same call the GPU
ranks of bench.py make -- run on world_size gloo ranks reproduces the full
matrix.  Its rows function is the CPU oracle here (the rows of the faces the
rank emits); on GPUs it is Context.form_factor_counts_rows."""
import os
import socket

import numpy as np
import pytest

from form_factors_b200 import emission, scenes, shard


def test_row_ranges_cover_every_row_once():
    rng = np.random.default_rng(0)
    for n in (1, 2, 5, 17, 400):
        for world in (1, 2, 3, 8):
            w = rng.integers(0, 50, n)
            r = shard.row_ranges(w, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == n
            assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
            assert all(b <= e for b, e in r)
            if n >= world:
                assert all(e > b for b, e in r)


def test_row_ranges_balance_rays():
    w = np.full(1000, 10)
    r = shard.row_ranges(w, 4)
    sizes = [w[b:e].sum() for b, e in r]
    assert max(sizes) - min(sizes) <= 10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    from oracle_lib import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        oracle = Oracle()
        oracle.set_threads(2)
        faces = scenes.parallel_plates(3, 0.7)
        n = len(faces)
        w, total = emission.two_sided_weights(faces)
        front, rear = emission.ray_counts(300 * n, w, total)

        def rows_fn(b, e):
            emit = (np.arange(n) >= b) & (np.arange(n) < e)
            fr = np.where(emit, front, 0).astype(np.int32)
            re = np.where(emit, rear, 0).astype(np.int32)
            return torch.from_numpy(oracle.form_factor_counts(faces, fr, re, seed=4)[b:e].astype(np.int64))

        (b, e), full = shard.solve_rows(rows_fn, front, rear, rank, world, n, gather=True)
        assert (b, e) == shard.row_ranges(shard.rays_per_row(front, rear), world)[rank]
        if rank == 0:
            want = oracle.form_factor_counts(faces, front, rear, seed=4).astype(np.int64)
            np.save(os.path.join(out_dir, "ok.npy"), np.array([np.array_equal(full.numpy(), want)]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gathered_row_blocks_equal_full_matrix(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    assert bool(np.load(tmp_path / "ok.npy")[0])
