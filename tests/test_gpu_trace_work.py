"""cr_trace_work: the counting build of the traversal kernel on a batch of
queries (wide nodes fetched, primitives tested), and the bench's comparison
of bytes per query with the reference's layout on the same rays."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, require_gpu

pytestmark = pytest.mark.gpu


def test_trace_work_counts(cr, scenes):
    require_gpu()
    d = scenes.config1(level=5, width=160, height=120)
    s = cr.Scene.from_desc(d)
    try:
        rng = np.random.default_rng(4)
        n = 4096
        px = np.stack([rng.integers(0, d.width, n), rng.integers(0, d.height, n)], 1)
        o, dr = scenes.pinhole_rays(d.camera, d.width, d.height, d.spp, px, rng.integers(0, d.spp, n))
        rays = np.concatenate([o, dr, np.zeros((n, 1), np.float32)], 1)
        nodes, prims = s.trace_work(rays)
        assert nodes >= n and prims >= n  # every ray of the closed box hits something
        nodes2, prims2 = s.trace_work(np.concatenate([rays, rays]))
        assert (nodes2, prims2) == (2 * nodes, 2 * prims)
        an, ap = s.trace_work(rays, any_hit=True)
        assert an > 0 and ap > 0
        assert s.trace_work(rays[:0]) == (0, 0)
    finally:
        s.close()


def test_layout_comparison_against_reference(cr, scenes, oracle):
    require_gpu()
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/cr_ref not built")
    sys.path.insert(0, ROOT)
    import bench
    import tempfile
    d = scenes.config0()
    s = cr.Scene.from_desc(d)
    try:
        with tempfile.TemporaryDirectory() as tmp:
            path = scenes.write_scene(d, tmp)
            out = bench.layout_comparison(s, d, path, n=512)
        assert out["ours"]["bytes_per_ray"] > 48 and out["reference"]["bytes_per_ray"] > 48
        assert out["reference"]["sphere_tests_per_ray"] == 2.0
        assert out["ratio"] > 0
    finally:
        s.close()
