"""Scene files whose mesh is a PLY render exactly like the same mesh as an OBJ:
the importer binds the PLY's single mesh to the shader "DefaultMaterial" (the
name assimp gives a mesh without a material) and the reference JSON schema
is otherwise unchanged."""
import json
import os

import numpy as np
import pytest

from conftest import require_gpu
from gpu_util import render_film

pytestmark = pytest.mark.gpu


def _one_material_scene(scenes):
    d = scenes.config0()
    merged = scenes.Group("DefaultMaterial", np.concatenate([g.v for g in d.groups]),
                          np.concatenate([g.n for g in d.groups]),
                          np.concatenate([g.f + o for g, o in zip(d.groups, np.cumsum([0] + [len(g.v) for g in d.groups[:-1]]))]).astype(np.uint32))
    d.groups = [merged]
    d.shaders["DefaultMaterial"] = ["Lambert", {"R": [0.7, 0.7, 0.7], "color": [1, 1, 1]}]
    d.shaders["lamp"] = ["Emission", {"color": [1, 1, 1], "strength": 20.0}]
    d.spheres = list(d.spheres) + [{"o": [2.8, 1.5, 4.6], "r": 0.4, "shader": "lamp"}]
    return d


def test_ply_scene_renders_like_obj_scene(cr, scenes, tmp_path):
    require_gpu()
    d = _one_material_scene(scenes)
    films, hits = [], []
    from golden.make_golden import make_rays
    rays = make_rays(d, 2048, 3)
    for fmt in ("obj", "ply"):
        mesh = str(tmp_path / f"m.{fmt}")
        if fmt == "obj":
            scenes.write_obj(mesh, d.groups)
        else:
            scenes.write_ply(mesh, d.groups, encoding="binary_little_endian", quads=True, extras=True)
        js = scenes.scene_json(d, os.path.basename(mesh))
        sc = cr.Scene.from_json(json.dumps(js), str(tmp_path))
        assert sc.info()["triangles"] == d.n_triangles
        hits.append(sc.trace(rays))
        films.append(render_film(cr, sc, 32, 32, 64, seeds=[5], estimator=cr.MIS))
    assert (hits[0]["prim"] == hits[1]["prim"]).all() and (hits[0]["tri"] == hits[1]["tri"]).all()
    np.testing.assert_array_equal(hits[0]["t"], hits[1]["t"])
    np.testing.assert_allclose(films[0].sum, films[1].sum, rtol=1e-12, atol=1e-300)
    assert films[0].mean.mean() > 0.01
