"""GPU OBJ import against the reference's importer (obj_import::scene,
import_export/obj_import.cpp:167-340, run live from oracle/_ref): faces bit
for bit, meshes, materials byte for byte and the status code, on generated
files in every supported style, on error cases, on a large file; and the
parsed scene traced straight from the device."""
import os

import numpy as np
import pytest

from form_factors_b200 import native, scenes
import obj_text as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "obj_ref.npz")


def _write(tmp_path, name, data):
    p = tmp_path / name
    p.write_bytes(data if isinstance(data, bytes) else data.encode())
    return str(p)


def _compare(ctx, reference, path):
    info = ctx.obj_load(path)
    rc, faces, meshes, materials = reference.obj_scene(path)
    assert info["status"] == rc, (info, rc)
    if rc != 0:
        return info
    got_faces, got_meshes, got_materials = ctx.obj_result(info)
    assert np.array_equal(got_faces.view(np.uint32), faces.view(np.uint32))
    assert np.array_equal(got_meshes, meshes)
    assert got_materials.tobytes() == materials.tobytes()
    return info


def _scene_with_meshes(seed):
    faces = scenes.clutter(240, 0.08, seed=seed, enclosure_cells=2)
    n = len(faces)
    cuts = sorted(set([0] + list(np.random.default_rng(seed).integers(1, n, 9)) + [n]))
    meshes = [(a, b - a) for a, b in zip(cuts[:-1], cuts[1:])]
    return faces, meshes


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_obj_with_materials_matches_reference(ctx, reference, tmp_path, seed):
    faces, meshes = _scene_with_meshes(seed)
    names = ["steel", "glass", "paint_%d" % seed]
    rng = np.random.default_rng(100 + seed)
    _write(tmp_path, "scene.mtl", O.mtl_text(names, rng))
    path = _write(tmp_path, "scene.obj", O.obj_text(faces, meshes, names, mtllib="scene.mtl", seed=seed))
    info = _compare(ctx, reference, path)
    assert info["n_faces"] == len(faces) and info["n_meshes"] == len(meshes) and info["n_materials"] == 3


def test_obj_plain_crlf_matches_reference(ctx, reference, tmp_path):
    faces = scenes.icosphere(3, 1.0, inward=True)
    path = _write(tmp_path, "crlf.obj", O.obj_text(faces, seed=7, crlf=True))
    info = _compare(ctx, reference, path)
    assert info["n_meshes"] == 1 and info["n_materials"] == 1  # one mesh, the black body


def test_obj_golden(ctx, tmp_path):
    g = np.load(GOLDEN)
    _write(tmp_path, "golden.mtl", g["mtl"].tobytes())
    info = ctx.obj_parse(g["obj"].tobytes(), filename=str(tmp_path / "golden.obj"))
    assert info["status"] == 0
    faces, meshes, materials = ctx.obj_result(info)
    assert np.array_equal(faces.view(np.uint32), g["faces"].view(np.uint32))
    assert np.array_equal(meshes, g["meshes"])
    assert materials.tobytes() == g["materials"].tobytes()


ERROR_CASES = {
    "bad vertex": ("v 1 2 3\nv 1 x 3\nf 1 1 1\n", None, 2),
    "bad face": ("v 1 2 3\nv 4 5 6\nv 7 8 9\nf 1 2\n", None, 4),
    "face v/vt": ("v 1 2 3\nv 4 5 6\nv 7 8 9\nf 1/1 2/2 3/3\n", None, 4),
    "unknown material": ("mtllib m.mtl\no a\nusemtl nothere\nv 1 2 3\n", "newmtl one\n" + "".join(
        "%s 0.5\n" % p for p in O.MATERIAL_PROPS) + "\n", 3),
    "missing library": ("mtllib absent.mtl\nv 1 2 3\n", None, 1),
    "not enough properties": ("mtllib m.mtl\nv 1 2 3\n", "newmtl one\nshell.density 1\n\n", 1),
    "invalid property": ("mtllib m.mtl\nv 1 2 3\n", "newmtl one\nshell.density abc\n", 1),
    "earliest error wins": ("v 1 2 3\nv bad\nmtllib absent.mtl\n", None, 2),
    "mtllib error first": ("mtllib absent.mtl\nv bad\n", None, 1),
}


@pytest.mark.parametrize("case", sorted(ERROR_CASES))
def test_obj_errors_match_reference(ctx, reference, tmp_path, case):
    obj, mtl, line = ERROR_CASES[case]
    if mtl is not None:
        _write(tmp_path, "m.mtl", mtl)
    path = _write(tmp_path, "e.obj", obj)
    info = _compare(ctx, reference, path)
    assert info["status"] < 0
    assert info["error_line"] == line


def test_large_obj_and_trace_from_device(ctx, reference, tmp_path):
    """200 000 faces: the import equals the reference's, and the scene set
    from the device traces to the same counts as the same faces from the host."""
    faces = np.concatenate([scenes.clutter(190000, 0.004, seed=4, enclosure_cells=40)])[:200000]
    path = _write(tmp_path, "big.obj", O.obj_text(faces, seed=9))
    info = _compare(ctx, reference, path)
    ctx.obj_scene_set(info["n_faces"])
    ctx.grid_build()
    front = np.full(info["n_faces"], 2, np.int32)
    rear = np.zeros(info["n_faces"], np.int32)
    rows = (np.arange(info["n_faces"]) % 64).astype(np.int32)
    a = ctx.form_factor_counts(front, rear, seed=3, face_to_row=rows, n_rows=64)
    got_faces, _, _ = ctx.obj_result(info)
    ctx.scene_set(got_faces)
    ctx.grid_build()
    b = ctx.form_factor_counts(front, rear, seed=3, face_to_row=rows, n_rows=64)
    assert np.array_equal(a, b) and a.sum() > 0
