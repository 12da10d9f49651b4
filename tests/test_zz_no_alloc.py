"""cr_render_device_noalloc: the render entry point for callers that cannot
allocate device memory while rendering (frame callbacks or real-time loops
where a cudaMalloc/cudaFree would synchronise the device, or applications that
budget all device memory at start-up).

Its film must equal the one cr_render_device produces for the same request,
on two calls in a row (the second call reuses the fixed array the first one
left filled).  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import require_gpu
from gpu_util import render_film

pytestmark = pytest.mark.gpu


def _noalloc_film(cr, scene, desc, n, films=None):
    import torch
    if films is None:
        films = (torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
                 torch.zeros(n * 3, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.int32, device="cuda"))
    s, q, c = films
    stream = torch.cuda.current_stream().cuda_stream
    rc = cr.lib().cr_render_device_noalloc(scene.h, C.byref(desc), C.c_void_p(s.data_ptr()),
                                           C.c_void_p(q.data_ptr()), C.c_void_p(c.data_ptr()), C.c_void_p(stream))
    assert rc == 0, cr.lib().cr_last_error()
    torch.cuda.synchronize()
    return s.cpu().numpy(), q.cpu().numpy(), c.cpu().numpy()


@pytest.mark.parametrize("wave_paths", [0, 10000])
def test_noalloc_matches_render_device_on_two_calls(cr, scenes, wave_paths):
    require_gpu()
    import torch
    scene = cr.Scene.from_desc(scenes.config0())
    W, H, spp = 40, 30, 64
    ref = render_film(cr, scene, W, H, spp, seeds=[5], estimator=cr.KOISHI, max_bounce=7,
                      wave_paths=wave_paths or 262144)
    for call in range(2):
        d = cr.render_desc(W, H, spp, max_bounce=7, estimator=cr.KOISHI, seed=5, wave_paths=wave_paths)
        films = [torch.zeros(W * H * 3, dtype=torch.float64, device="cuda") for _ in range(2)]
        films.append(torch.zeros(W * H, dtype=torch.int32, device="cuda"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        s, q, c = _noalloc_film(cr, scene, d, W * H, films)
        free1 = torch.cuda.mem_get_info()[0]
        if call == 1:
            # the first call may load kernel code lazily; the second allocates
            # nothing on the device
            assert free1 == free0, (free0, free1)
        # Same request, same random streams, same waves: the films agree to
        # the FP64 summation tolerance the render tests use (1e-12 relative),
        # and the sample counts exactly.
        np.testing.assert_allclose(s.reshape(H, W, 3), ref.sum, rtol=1e-12, atol=0)
        np.testing.assert_allclose(q.reshape(H, W, 3), ref.sumsq, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(c.reshape(H, W), ref.count.astype(np.int64))


def test_noalloc_rejects_sizes_beyond_its_array(cr, scenes):
    require_gpu()
    scene = cr.Scene.from_desc(scenes.config0())
    lib = cr.lib()
    dummy = C.c_void_p(1 << 20)  # never dereferenced: the request is rejected first
    d = cr.render_desc(16, 16, 4, max_bounce=7, wave_paths=262144 + 1)
    assert lib.cr_render_device_noalloc(scene.h, C.byref(d), dummy, dummy, dummy, None) == -1
    assert b"exceeds the no-allocation maximum" in lib.cr_last_error()
    d = cr.render_desc(16, 16, 4, max_bounce=65)
    assert lib.cr_render_device_noalloc(scene.h, C.byref(d), dummy, dummy, dummy, None) == -1
    assert b"max_bounce" in lib.cr_last_error()


def test_noalloc_refuses_guided_renders_before_touching_the_scene(cr, scenes):
    """A guided request needs the scene's guide and its training records, which
    are allocated: the entry point refuses it up front (CR_ERR_UNSUPPORTED)
    and leaves the scene's guide unset."""
    require_gpu()
    scene = cr.Scene.from_desc(scenes.config0())
    lib = cr.lib()
    dummy = C.c_void_p(1 << 20)  # never dereferenced: the request is rejected first
    d = cr.render_desc(16, 16, 4, max_bounce=7, estimator=cr.MIS, guiding=True)
    assert lib.cr_render_device_noalloc(scene.h, C.byref(d), dummy, dummy, dummy, None) == -5
    assert b"guided" in lib.cr_last_error()
    # the scene's guide was never set up (cr_guide_info reports no guide)
    step = C.c_uint32()
    assert lib.cr_guide_info(scene.h, None, None, C.byref(step), None) == -4
