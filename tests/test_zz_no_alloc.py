"""ffb_cast_bruteforce_static: the brute-force cast for callers that cannot
allocate device memory (their device memory is owned by another allocator, or
their host forbids device allocations after start-up).  It keeps its scratch
in a static device array instead of allocating, so it is checked here against
the context entry point ffb_cast_bruteforce on two calls in a row, the second
overwriting the array the first one filled.  Hit indices and points must be
bit-identical (the tolerance of every hit comparison in these tests)."""
import numpy as np
import pytest

from form_factors_b200 import build, native, scenes
import rays as R

pytestmark = pytest.mark.gpu


def test_static_scratch_cast_matches_context_cast():
    import torch

    build.build()
    ctx = native.Context(0)
    cases = [(scenes.parallel_plates(10, 1.0), 3), (scenes.clutter(300, 0.05, seed=2, enclosure_cells=5), 4)]
    for faces, seed in cases:
        rays = R.mixed_rays(np.random.default_rng(seed), faces, 5000)
        ctx.scene_set(faces)
        want_hit, want_pts = ctx.cast(rays, brute=True)
        n = len(rays)
        f_dev = torch.from_numpy(faces).cuda()
        r_dev = torch.from_numpy(rays).cuda()
        hit = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        pts = torch.full((n, 3), 7.0, dtype=torch.float32, device="cuda")
        native.cast_bruteforce_static(f_dev, r_dev, hit, pts)
        torch.cuda.synchronize()
        got_hit = hit.cpu().numpy()
        got_pts = pts.cpu().numpy()
        assert np.array_equal(got_hit, want_hit)
        m = want_hit >= 0
        assert m.any() and (~m).any()
        assert np.array_equal(got_pts[m].view(np.uint32), want_pts[m].view(np.uint32))
        assert np.isnan(got_pts[~m]).all()
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
