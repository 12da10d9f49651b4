"""Concurrent renders of distinct scenes (include/cr.h promises them): two
host threads, each with its own stream and scene, rendering at the same time.

The films must equal the same renders made one after the other (renders are
deterministic), and guided renders started concurrently on two fresh scenes,
whose first launches set the guide kernels' shared-memory limit, must both
run and give finite films.
"""
import threading

import numpy as np
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu


def _render(cr, scene, W, H, spp, seed, estimator, stream, guiding=False, wave_paths=0):
    import torch
    n = W * H
    f = (torch.zeros(n * 3, dtype=torch.float64, device="cuda"), torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
         torch.zeros(n, dtype=torch.int32, device="cuda"))
    d = cr.render_desc(W, H, spp, max_bounce=7, estimator=estimator, seed=seed, guiding=guiding,
                       wave_paths=wave_paths)
    scene.render_device(d, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream.cuda_stream, stats=False)
    stream.synchronize()
    return [t.cpu().numpy() for t in f]


def _run_threads(targets):
    out, errs = [None] * len(targets), []

    def wrap(i, fn):
        try:
            out[i] = fn()
        except Exception as e:  # surfaced in the main thread
            errs.append(e)

    ts = [threading.Thread(target=wrap, args=(i, fn)) for i, fn in enumerate(targets)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    assert not errs, errs
    return out


def test_two_threads_two_streams_two_scenes_match_sequential(cr, scenes):
    require_gpu()
    import torch
    a = cr.Scene.from_desc(scenes.config0())
    b = cr.Scene.from_desc(scenes.config_materials(cosine=False))
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    ref_a = _render(cr, a, 64, 48, 64, 3, cr.KOISHI, sa)
    ref_b = _render(cr, b, 48, 48, 64, 4, cr.MIS, sb)
    got_a, got_b = _run_threads([lambda: _render(cr, a, 64, 48, 64, 3, cr.KOISHI, sa),
                                 lambda: _render(cr, b, 48, 48, 64, 4, cr.MIS, sb)])
    for got, ref in ((got_a, ref_a), (got_b, ref_b)):
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-12, atol=0)
        np.testing.assert_allclose(got[1], ref[1], rtol=1e-12, atol=0)
        np.testing.assert_array_equal(got[2], ref[2])
    a.close(), b.close()


def test_concurrent_guided_renders_on_fresh_scenes(cr, scenes):
    require_gpu()
    import torch
    c = cr.Scene.from_desc(scenes.config0())
    d = cr.Scene.from_desc(scenes.config3(width=64, height=64))
    sc, sd = torch.cuda.Stream(), torch.cuda.Stream()
    # 16 waves of 65,536 paths: 2 training steps per wave, and the guide is
    # sampled (its inference kernel launched) once 8 steps have run
    fc, fd = _run_threads([lambda: _render(cr, c, 64, 64, 256, 5, cr.MIS, sc, guiding=True, wave_paths=65536),
                           lambda: _render(cr, d, 64, 64, 256, 6, cr.MIS, sd, guiding=True, wave_paths=65536)])
    for f in (fc, fd):
        assert np.isfinite(f[0]).all() and f[2].min() > 0
    # the guide trained past its warm-up (and was then sampled) on both scenes
    assert cr.Guide(c).info()["step"] > 8 and cr.Guide(d).info()["step"] > 8
    c.close(), d.close()
