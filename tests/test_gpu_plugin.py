"""The reference-side binding, run for real: the CudaWavefront Tracer plugin
(cuda-raytracer_b200/plugin/cudaWavefront.hpp) registered in the reference's
Factory<Tracer> (as src/core/tracer/tracer.impl.cu:8-11 registers
CPUMulticore), created by name and driven through Tracer::execute
(src/core/tracer/tracer.hpp:20-21) on a Scene the reference itself built,
inside the reference harness (oracle/_ref/cr_ref_plugin).

Its 8-bit image must equal the library's own render of the same scene with
the same seed and the reference's light table, and agree with the
reference's CPU render (tests/golden/c0_film.npz) within Monte Carlo error.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden, require_gpu

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "cr_ref_plugin")


def to_image8(film):
    """util::Image<3>'s conversion (src/util/image.hpp:29-34): float, clamped
    to [0, 1], times 255, truncated to a byte."""
    f = np.clip(film.astype(np.float32), np.float32(0), np.float32(1)) * np.float32(255)
    return f.astype(np.uint8)


def run_plugin(desc, W, H, spp, seed):
    from cuda_raytracer_b200 import scenes
    with tempfile.TemporaryDirectory() as tmp:
        path = scenes.write_scene(desc, tmp)
        out = os.path.join(tmp, "img.u8")
        r = subprocess.run([EXE, "plugin", os.path.basename(path), str(W), str(H), str(spp), out, str(seed)],
                           cwd=tmp, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        return np.fromfile(out, np.uint8).reshape(H, W, 3)


@pytest.mark.skipif(not os.path.exists(EXE), reason="plugin harness not built (make -C oracle plugin)")
def test_plugin_renders_through_factory_tracer(cr, scenes):
    require_gpu()
    g = golden("c0_film.npz")
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    desc = scenes.config0()
    img = run_plugin(desc, W, H, spp, seed=1)
    # The library's own render with the reference's light table (the plugin
    # hands the reference Mesh's table over) and the same seed: the same
    # sample paths up to float rounding, so the 8-bit images agree exactly on
    # nearly every pixel.
    lt = golden("c0_lights.npz")
    sc = cr.Scene.from_desc(desc)
    sc.set_light_table(int(lt["group"]), lt["table"], float(lt["pdf"]))
    film, _ = sc.render(W, H, spp, max_bounce=int(g["max_bounce"]), estimator=cr.KOISHI, seed=1)
    ours = to_image8(film)
    same = (ours == img).mean()
    assert same > 0.98, same
    assert np.abs(ours.astype(int) - img.astype(int)).max() <= 8
    # Against the reference's CPU render: within 3 sigma (plus one 8-bit step)
    # of its clamped mean, per pixel channel.
    ref_mean = g["sum"] / g["count"][..., None]
    ref_var = np.maximum(g["sumsq"] / g["count"][..., None] - ref_mean ** 2, 0) / g["count"][..., None]
    got = img.astype(np.float64) / 255
    tol = 3 * np.sqrt(2 * ref_var) + 1.0 / 255
    inside = np.abs(got - np.clip(ref_mean, 0, 1)) <= tol
    assert inside.mean() > 0.98, inside.mean()
    sc.close()
