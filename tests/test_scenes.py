"""Seeded scene generator: shapes, the no-face-parallel-to-y rule, file formats."""
import json
import os

import numpy as np
import pytest


def test_config0_shape(scenes):
    d = scenes.config0()
    assert d.n_triangles == 22  # 10 wall quads + the light quad
    assert len(d.spheres) == 2
    assert {"white", "red", "green", "light", "glossy", "ball"} <= set(d.shaders)


def test_no_flat_face_parallel_to_y(scenes):
    # The reference's frame n x (0,1,0) is NaN for such faces (scene.hpp:48-50).
    for desc in (scenes.config0(), scenes.config1(level=3)):
        for g in desc.groups:
            n = g.n.astype(np.float64)
            assert np.all(np.hypot(n[:, 0], n[:, 2]) > 1e-3)


def test_config1_counts(scenes):
    d = scenes.config1(level=3)
    assert d.n_triangles == 22 + 20 * 4 ** 3
    names = [g.name for g in d.groups]
    assert len(names) == len(set(names))


def test_icosphere_patches(scenes):
    v, f = scenes.icosphere(3)
    assert len(f) == 20 * 64 and len(v) == 10 * 64 + 2
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)


def test_crm_and_obj_round_trip(scenes, tmp_path):
    d = scenes.config0()
    p = str(tmp_path / "m.crm")
    scenes.write_crm(p, d.groups)
    back = scenes.read_crm(p)
    assert [g.name for g in back] == [g.name for g in d.groups]
    for a, b in zip(d.groups, back):
        assert np.array_equal(a.v, b.v) and np.array_equal(a.n, b.n) and np.array_equal(a.f, b.f)
    path = scenes.write_scene(d, str(tmp_path), fmt="obj")
    doc = json.load(open(path))
    assert doc["scene"]["assets"][0] == ["import", {"path": "config0.obj"}]
    text = open(os.path.join(tmp_path, "config0.obj")).read()
    assert text.count("usemtl") == len(d.groups)


def test_pinhole_rays_match_lens_formula(scenes):
    d = scenes.config0()
    o, dirs = scenes.pinhole_rays(d.camera, 64, 64, 16, np.array([[32, 32]]), np.array([0]))
    # the centre pixel's first sub-sample looks along the target direction
    t = np.asarray(d.camera["target"])
    assert np.dot(dirs[0], t / np.linalg.norm(t)) > 0.9999


@pytest.mark.parametrize("encoding", ["ascii", "binary_little_endian", "binary_big_endian"])
@pytest.mark.parametrize("quads,extras", [(False, False), (True, True)])
def test_ply_import_reads_what_obj_import_reads(cr, scenes, tmp_path, encoding, quads, extras):
    """The PLY reader (cr_mesh_file_info parses without a GPU) sees the same
    triangles, in the same order, as the OBJ reader: 4-gons fan back into
    their two triangles and unknown properties and elements are skipped."""
    d = scenes.config0()
    obj, ply = str(tmp_path / "m.obj"), str(tmp_path / "m.ply")
    scenes.write_obj(obj, d.groups)
    scenes.write_ply(ply, d.groups, encoding=encoding, quads=quads, extras=extras)
    go, vo, to, co = cr.mesh_file_info(obj)
    gp, vp, tp, cp = cr.mesh_file_info(ply)
    assert go == len(d.groups) and gp == 1          # PLY: one "DefaultMaterial" group
    assert to == tp == d.n_triangles
    assert vp == sum(len(g.v) for g in d.groups)
    assert cp == pytest.approx(co, rel=1e-12)


def test_ply_without_normals_and_bad_files(cr, scenes, tmp_path):
    d = scenes.config1(level=2)
    ply = str(tmp_path / "n.ply")
    scenes.write_ply(ply, d.groups, normals=False)
    assert cr.mesh_file_info(ply)[2] == d.n_triangles
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
                    b"element face 1\nproperty list uchar int vertex_indices\nend_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 7\n")
    with pytest.raises(cr.CrError, match="out of range"):
        cr.mesh_file_info(str(bad))
    trunc = tmp_path / "trunc.ply"
    trunc.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
                      b"property float z\nend_header\n\x00\x00")
    with pytest.raises(cr.CrError, match="truncated"):
        cr.mesh_file_info(str(trunc))
    with pytest.raises(cr.CrError):
        cr.mesh_file_info(str(tmp_path / "missing.ply"))


def test_obj_faces_without_material_bind_to_default_material(cr, tmp_path):
    """OBJ faces before any usemtl get the material name assimp gives a mesh
    without one, "DefaultMaterial"; the shader lookup fails (before any GPU
    work) when the scene does not define it."""
    import ctypes as C
    import json
    (tmp_path / "m.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    doc = {"scene": {"camera": [{"position": [0, 0, -1], "target": [0, 0, 1]}],
                     "assets": [["import", {"path": "m.obj"}]], "shaders": {}}}
    out = C.c_void_p()
    rc = cr.lib().cr_scene_create(json.dumps(doc).encode(), str(tmp_path).encode(), C.byref(out))
    assert rc == -1 and b"DefaultMaterial" in cr.lib().cr_last_error()
