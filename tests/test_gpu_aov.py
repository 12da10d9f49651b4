"""The reference's debug kernels (Normal, Visibility, HalfVector) on the GPU
against the reference's own renders of them (tests/golden/c0_aov_*.npz) and
the FP64 oracle, and their selection by name (cr_scene_set_kernel, cr -k)."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import require_gpu
from gpu_util import render_film, zscores

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("kernel", ["Normal", "Visibility", "HalfVector"])
def test_debug_kernel_matches_reference(cr, scenes, kernel):
    require_gpu()
    g = np.load(os.path.join(GOLDEN, f"c0_aov_{kernel.lower()}.npz"))
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    ref = O.Film(g["sum"], g["sumsq"], g["count"])
    s = cr.Scene.from_desc(scenes.config0()).set_kernel(kernel)
    f = render_film(cr, s, W, H, spp, seeds=[41], estimator=cr.KOISHI)
    assert np.all(f.count == spp)
    if kernel == "Normal":
        d = np.abs(f.mean - ref.mean)
        assert (d > 1e-3).mean() < 0.02, (d > 1e-3).mean()
        assert abs(f.mean.mean() - ref.mean.mean()) < 1e-4
    else:
        z = zscores(f, ref)
        assert (z > 3).mean() < 0.01, (z > 3).mean()
        assert abs(f.mean.mean() / ref.mean.mean() - 1) < 0.01


def test_visibility_on_a_mesh_scene_matches_oracle(cr, scenes):
    """Visibility where much of the image is in shadow: the level-5 mesh in the
    box, against the FP64 oracle."""
    require_gpu()
    d = scenes.config1(level=5)
    W, H, spp = 48, 36, 256
    o = O.OracleScene(d).render(W, H, spp, 7, O.AOV_VISIBILITY, seed=3)
    f = render_film(cr, cr.Scene.from_desc(d).set_kernel("Visibility"), W, H, spp, seeds=[5], estimator=cr.KOISHI)
    z = zscores(f, o)
    assert (z > 3).mean() < 0.01, (z > 3).mean()
    assert 0.1 < o.mean.mean() < 0.99


def test_kernel_selection_errors(cr, scenes):
    require_gpu()
    s = cr.Scene.from_desc(scenes.config0())
    with pytest.raises(cr.CrError):
        s.set_kernel("Bogus")
    s.set_kernel("Normal")
    with pytest.raises(cr.CrError):  # guiding belongs to the Radiance kernel
        s.render(8, 8, 1, estimator=cr.MIS, guiding=True)
    film, _ = s.render(8, 8, 1)
    assert np.isfinite(film).all() and film.max() <= 1.0
