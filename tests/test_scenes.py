"""Seeded scene generator: shapes, the no-face-parallel-to-y rule, file formats."""
import json
import os

import numpy as np


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
