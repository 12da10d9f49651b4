"""The reference's traversal work, counted by the harness's `work` command
(oracle/_ref/cr_ref: Mesh::intersect's depth-first walk restated over the
reference's own BVH and faces, src/core/primitive/mesh.cu:200-267), which the
bench sets beside this build's node and primitive counts on the same rays."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest


def _work(oracle, scenes, desc, rays):
    with tempfile.TemporaryDirectory() as tmp:
        path = scenes.write_scene(desc, tmp)
        rp = os.path.join(tmp, "rays.f32")
        np.ascontiguousarray(rays, np.float32).tofile(rp)
        r = subprocess.run([oracle.REF_BIN, "work", os.path.basename(path), rp], cwd=tmp, capture_output=True,
                           text=True, timeout=300, check=True)
    return json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])


def test_reference_work_counts(oracle, scenes):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/cr_ref not built")
    d = scenes.config0()
    rng = np.random.default_rng(3)
    n = 256
    px = np.stack([rng.integers(0, d.width, n), rng.integers(0, d.height, n)], 1)
    o, dr = scenes.pinhole_rays(d.camera, d.width, d.height, d.spp, px, rng.integers(0, d.spp, n))
    rays = np.concatenate([o, dr, np.zeros((n, 1), np.float32)], 1)
    w = _work(oracle, scenes, d, rays)
    n_meshes = len(d.groups)
    assert w["rays"] == n
    # every ray asks each of the 2 spheres and reads each mesh's root record
    assert w["spheres"] == 2 * n
    assert w["nodes"] >= n * n_meshes
    # a mesh small enough to be one leaf has its faces tested by every ray
    assert w["faces"] >= n
    # the same rays twice: twice the work
    w2 = _work(oracle, scenes, d, np.concatenate([rays, rays]))
    assert (w2["nodes"], w2["faces"], w2["spheres"]) == (2 * w["nodes"], 2 * w["faces"], 2 * w["spheres"])
