"""Grid structure checks that need no ray.

1. Binning is conservative: every face is listed in every cell that the
   triangle meets once the cell is grown by the binning margin on each axis
   (an exact separating-axis test in float64 with 0.9 of the margin, so that
   only cells the float32 build must include are required).  Faces the
   reference treats as degenerate are never binned and are skipped.  The
   traversal's
   exactness rests on this (a hit point computed on a triangle lies within
   the margin of the triangle).
2. Each empty cell's eight octant distances equal the side of the largest
   cube of empty cells that extends from it in the octant's directions
   (capped at 127), computed here by the corner recurrence
   side(c) = 1 + min(side of the 7 neighbours further along the octant).
3. Each cell's references are in ascending face order.
"""
import itertools

import numpy as np
import pytest

from form_factors_b200 import scenes

pytestmark = pytest.mark.gpu

CAP = 127


def _slivers(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.1, 0.9, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    b = a + 0.6 * d
    c = a + 0.3 * d + rng.normal(scale=1e-3, size=(n, 3))  # nearly on the a-b line
    return np.concatenate([a, b, c], axis=1).astype(np.float32)


def _cases():
    return {
        "clutter": (scenes.clutter(300, 0.05, seed=3, enclosure_cells=5), (24, 20, 28)),
        "sphere": (scenes.icosphere(3, 1.0, inward=True), (22, 22, 22)),
        "slivers": (np.concatenate([_slivers(200, 5), scenes.unit_box()]), (17, 23, 19)),
    }


def _cell_lists(rec, refs):
    occ = (rec[..., 1] & 0x80000000) == 0
    lists = {}
    for z, y, x in zip(*np.nonzero(occ)):
        b, e = int(rec[z, y, x, 0]), int(rec[z, y, x, 1])
        lists[(x, y, z)] = refs[b:e]
    return occ, lists


def _live(face9):
    """A face the reference can hit: finite, and dot(n, n) >= 1e-8 for its
    float32 normal n = (p1 - p0) x (p2 - p0) (math/operations.h:31); the
    build bins no other face."""
    p = np.asarray(face9, np.float32).reshape(3, 3)
    if not np.isfinite(p).all():
        return False
    u, v = p[1] - p[0], p[2] - p[0]
    n = [u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]]
    nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2]
    return float(nn) >= 1e-8


def _overlaps(tri, centres, h):
    """Exact (float64) separating-axis test of a triangle against boxes of
    half-extent h around the given centres (k, 3): a boolean per box."""
    v = tri[None, :, :] - centres[:, None, :]  # (k, 3 vertices, 3)
    e = [tri[1] - tri[0], tri[2] - tri[1], tri[0] - tri[2]]
    axes = [np.eye(3)[a] for a in range(3)] + [np.cross(e[0], e[1])]
    axes += [np.cross(ei, np.eye(3)[a]) for ei in e for a in range(3)]
    keep = np.ones(len(centres), bool)
    for ax in axes:
        if not np.any(ax):
            continue
        p = v @ ax
        r = np.abs(ax) @ h
        keep &= ~((p.min(1) > r) | (p.max(1) < -r))
    return keep


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_binning_is_conservative(ctx, name):
    faces, dims = _cases()[name]
    ctx.scene_set(faces)
    ctx.grid_build(dims=dims)
    info = ctx.grid_info()
    rec, refs = ctx.grid_export()
    _, lists = _cell_lists(rec, refs)
    lists = {k: set(v.tolist()) for k, v in lists.items()}
    lo = np.array(info.lo, np.float64)
    cs = np.array(info.cell, np.float64)
    n = np.array([info.nx, info.ny, info.nz])
    m = 0.9 * float(info.margin)
    h = cs / 2 + m
    tris = faces.reshape(-1, 3, 3).astype(np.float64)
    missing = []
    required = 0
    for f, t in enumerate(tris):
        if not _live(faces[f]):
            continue
        i0 = np.clip(np.floor((t.min(0) - m - lo) / cs).astype(int) - 1, 0, n - 1)
        i1 = np.clip(np.floor((t.max(0) + m - lo) / cs).astype(int) + 1, 0, n - 1)
        cells = np.array(list(itertools.product(*[range(i0[a], i1[a] + 1) for a in range(3)])))
        need = cells[_overlaps(t, lo + (cells + 0.5) * cs, h)]
        required += len(need)
        for x, y, z in need.tolist():
            if f not in lists.get((x, y, z), ()):
                missing.append((f, (x, y, z)))
    assert required > 0
    assert not missing, "%d of %d required (face, cell) pairs missing, first %s" % (
        len(missing), required, missing[:5])
    assert int(info.n_refs) >= required


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_octant_distances(ctx, name):
    faces, dims = _cases()[name]
    ctx.scene_set(faces)
    ctx.grid_build(dims=dims)
    rec, refs = ctx.grid_export()
    occ, lists = _cell_lists(rec, refs)
    for cell in lists.values():
        assert np.all(np.diff(cell) > 0), "references of a cell must ascend"
    nz, ny, nx = occ.shape
    empty = ~occ
    packed = rec[..., 0].astype(np.uint64) | (rec[..., 1].astype(np.uint64) & 0x7FFFFFFF) << 32
    for o in range(8):
        s = [(-1 if (o >> a) & 1 else 1) for a in range(3)]  # x, y, z
        side = np.full((nz + 1, ny + 1, nx + 1), CAP, np.int64)  # one cell of padding past the far end
        xs = range(nx - 1, -1, -1) if s[0] > 0 else range(nx)
        ys = range(ny - 1, -1, -1) if s[1] > 0 else range(ny)
        zs = range(nz - 1, -1, -1) if s[2] > 0 else range(nz)
        for z in zs:
            for y in ys:
                for x in xs:
                    if occ[z, y, x]:
                        side[z, y, x] = 0
                        continue
                    best = CAP
                    for dz, dy, dx in itertools.product((0, 1), repeat=3):
                        if dx == dy == dz == 0:
                            continue
                        best = min(best, side[z + dz * s[2], y + dy * s[1], x + dx * s[0]])
                    side[z, y, x] = min(CAP, 1 + best)
        want = side[:nz, :ny, :nx]
        got = ((packed >> np.uint64(32 * (o >> 2) + 8 * (o & 3))) & np.uint64(0x7F)).astype(np.int64)
        bad = np.argwhere(empty & (got != want))
        assert bad.size == 0, "octant %d: %d cells differ, first (z, y, x) %s got %s want %s" % (
            o, len(bad), bad[:3].tolist(), got[tuple(bad[0])], want[tuple(bad[0])])


def test_export_without_skip_marks_unit_steps(ctx):
    faces = scenes.clutter(100, 0.08, seed=2, enclosure_cells=3)
    ctx.scene_set(faces)
    ctx.grid_build(dims=(12, 12, 12), skip_empty=False)
    rec, _ = ctx.grid_export()
    empty = (rec[..., 1] & 0x80000000) != 0
    assert empty.any()
    assert np.all(rec[empty][:, 0] == 0x01010101)
    assert np.all(rec[empty][:, 1] == 0x81010101)
