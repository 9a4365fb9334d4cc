"""ffb_cast_bruteforce_static: the brute-force cast for callers that cannot
allocate device memory (their device memory is owned by another allocator, or
their host forbids device allocations after start-up).  It keeps its scratch
in a static device array instead of allocating, so it is checked here on two
calls in a row, the second overwriting the array the first one filled,
against the context entry point ffb_cast_bruteforce and against the CPU
oracle's brute-force definition (ray_caster/naive_cpu.cpp:65-97).  Hit
indices and points must be bit-identical (the tolerance of every hit
comparison in these tests)."""
import ctypes as C

import numpy as np
import pytest

from form_factors_b200 import build, native, scenes
import rays as R

pytestmark = pytest.mark.gpu


def _same(got_hit, got_pts, want_hit, want_pts, what):
    assert np.array_equal(got_hit, want_hit), what + ": hit indices differ"
    m = want_hit >= 0
    assert m.any() and (~m).any()
    assert np.array_equal(got_pts[m].view(np.uint32), want_pts[m].view(np.uint32)), what + ": hit points differ"
    assert np.isnan(got_pts[~m]).all(), what + ": miss points must be NaN"


def test_static_scratch_cast_matches_context_cast_and_oracle(oracle):
    import torch

    build.build()
    ctx = native.Context(0)
    cases = [(scenes.parallel_plates(10, 1.0), 3), (scenes.clutter(300, 0.05, seed=2, enclosure_cells=5), 4)]
    for faces, seed in cases:
        rays = R.mixed_rays(np.random.default_rng(seed), faces, 5000)
        ctx.scene_set(faces)
        want_hit, want_pts = ctx.cast(rays, brute=True)
        ref_hit, ref_pts = oracle.cast_naive(faces, rays)
        n = len(rays)
        f_dev = torch.from_numpy(faces).cuda()
        r_dev = torch.from_numpy(rays).cuda()
        hit = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        pts = torch.full((n, 3), 7.0, dtype=torch.float32, device="cuda")
        native.cast_bruteforce_static(f_dev, r_dev, hit, pts)
        torch.cuda.synchronize()
        got_hit = hit.cpu().numpy()
        got_pts = pts.cpu().numpy()
        _same(got_hit, got_pts, want_hit, want_pts, "static vs context")
        _same(got_hit, got_pts, ref_hit, ref_pts, "static vs oracle")
    ctx.close()


def test_static_scratch_rejects_oversize_scene():
    import torch

    build.build()
    faces = torch.zeros((16385, 9), dtype=torch.float32, device="cuda")
    rays = torch.zeros((4, 6), dtype=torch.float32, device="cuda")
    hit = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(native.FFBError) as err:
        native.cast_bruteforce_static(faces, rays, hit)
    assert err.value.code == -306
    assert "16384" in str(err.value)


def test_static_scratch_rejects_host_buffers():
    """Every buffer must be device memory of the current device: a host array
    is refused with FFB_ERR_ARG before anything is enqueued."""
    import torch

    lib = native.load()
    faces = torch.zeros((8, 9), dtype=torch.float32, device="cuda")
    rays_host = np.zeros((4, 6), np.float32)
    hit = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = lib.ffb_cast_bruteforce_static(C.c_void_p(faces.data_ptr()), 8, rays_host.ctypes.data_as(C.c_void_p), 4,
                                        C.c_void_p(hit.data_ptr()), None, None)
    assert rc == -301, lib.ffb_last_error()
    assert b"device memory" in lib.ffb_last_error()
