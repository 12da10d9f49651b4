"""Ray binning (cr_render_desc.bin_rays): the secondary and shadow traversal
queues are sorted by (ray octant, origin cell) before tracing.  Every ray's
result is its own, so a binned render must give the same film, bit for bit,
and trace the same rays as the render in queue order, for both estimators,
with waves that split the image and with spheres among the primitives.
"""
import numpy as np
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu


def _film(cr, scene, W, H, spp, seed, estimator, bin_rays, wave_paths=0, max_bounce=7):
    import torch
    n = W * H
    f = (torch.zeros(n * 3, dtype=torch.float64, device="cuda"), torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
         torch.zeros(n, dtype=torch.int32, device="cuda"))
    d = cr.render_desc(W, H, spp, max_bounce=max_bounce, estimator=estimator, seed=seed, wave_paths=wave_paths,
                       bin_rays=bin_rays, count_work=True)
    st = scene.render_device(d, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in f], st


@pytest.mark.parametrize("estimator", ["KOISHI", "MIS"])
def test_binned_render_equals_queue_order(cr, scenes, estimator):
    require_gpu()
    est = getattr(cr, estimator)
    s = cr.Scene.from_desc(scenes.config1(level=5, width=160, height=120))
    try:
        for wave in (0, 20000):
            a, sa = _film(cr, s, 160, 120, 8, 5, est, -1, wave)
            b, sb = _film(cr, s, 160, 120, 8, 5, est, 1, wave)
            for x, y in zip(a, b):
                assert np.array_equal(x, y)
            assert sa.rays_extend == sb.rays_extend and sa.rays_shadow == sb.rays_shadow
            assert sa.extend_launches == sb.extend_launches
    finally:
        s.close()


def test_binned_render_with_spheres(cr, scenes):
    """The small box scene: two spheres among the BVH primitives."""
    require_gpu()
    s = cr.Scene.from_desc(scenes.config0(width=96, height=96))
    try:
        a, _ = _film(cr, s, 96, 96, 16, 11, cr.MIS, -1)
        b, _ = _film(cr, s, 96, 96, 16, 11, cr.MIS, 1)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    finally:
        s.close()


def test_autotune_reports_binning(cr, scenes):
    require_gpu()
    s = cr.Scene.from_desc(scenes.config1(level=5, width=128, height=96))
    try:
        t = s.autotune(cr.render_desc(128, 96, 16, max_bounce=7, estimator=cr.KOISHI, seed=3))
        assert t.bin_rays in (1, -1)
        # later renders with bin_rays = 0 take the tuned choice and still render
        f, _ = _film(cr, s, 128, 96, 4, 9, cr.KOISHI, 0)
        assert np.isfinite(f[0]).all() and (f[2] == 4).all()
    finally:
        s.close()
