"""Wave state comes from a memory pool of the library's own, which keeps freed
memory mapped between renders; cr_trim_memory hands it back.  Renders before
and after a trim agree bit for bit, and the trim returns the cached memory to
the device (its free memory rises by at least the wave state of the render)."""
import numpy as np
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu


def test_trim_returns_cached_wave_memory(cr, scenes):
    require_gpu()
    import torch
    s = cr.Scene.from_desc(scenes.config0(width=128, height=128))
    kw = dict(max_bounce=7, estimator=cr.KOISHI, seed=5, wave_paths=1 << 22)
    a, _ = s.render(128, 128, 256, **kw)
    s.close()  # the scene's wave buffers go back to the pool, which keeps them
    torch.cuda.synchronize()
    free_kept, _ = torch.cuda.mem_get_info()
    cr.trim_memory()
    torch.cuda.synchronize()
    free_trimmed, _ = torch.cuda.mem_get_info()
    # 4M paths of wave state: several hundred MB
    assert free_trimmed - free_kept >= 256 << 20, (free_kept, free_trimmed)
    s2 = cr.Scene.from_desc(scenes.config0(width=128, height=128))
    b, _ = s2.render(128, 128, 256, **kw)
    s2.close()
    assert np.array_equal(a, b)
    cr.trim_memory()
