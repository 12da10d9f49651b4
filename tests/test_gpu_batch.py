"""Batched renders (cr_batch_*): several scenes of different size, resolution
and spp in shared waves under one captured CUDA graph give the same films as
rendering each scene on its own with the same seeds."""
import numpy as np
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu


def _films(torch, w, h):
    n = w * h
    return (torch.zeros(n * 3, dtype=torch.float64, device="cuda"), torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
            torch.zeros(n, dtype=torch.int32, device="cuda"))


@pytest.fixture(scope="module")
def batch_scenes(cr, scenes):
    require_gpu()
    a = cr.Scene.from_desc(scenes.config0())
    b = cr.Scene.from_desc(scenes.config2(3, max_triangles=6000))
    c = cr.Scene.from_desc(scenes.config2(7, max_triangles=20000))
    o = cr.Scene.from_desc(scenes.config0_ortho())  # the orthographic lens
    # (scene, width, height, spp, seed): uneven sizes; scene a twice with other seeds
    return [(a, 48, 40, 16, 11), (b, 64, 64, 8, 12), (a, 33, 17, 5, 13), (c, 80, 48, 4, 14), (o, 40, 24, 6, 15)]


def _single(cr, torch, job, estimator, seed_add=0, acc=None):
    sc, w, h, spp, seed = job
    f = acc or _films(torch, w, h)
    d = cr.render_desc(w, h, spp, max_bounce=7, estimator=estimator, seed=seed + seed_add)
    sc.render_device(d, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    return f


def _assert_same(got, ref):
    torch_sync()
    for g, r in zip(got, ref):
        g, r = g.cpu().numpy(), r.cpu().numpy()
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-300)


def torch_sync():
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("estimator", [0, 1])
def test_batch_matches_single_renders(cr, batch_scenes, estimator):
    """Same paths, same random keys: each job's film equals the stand-alone
    render of its scene (up to the order of FP64 additions at wave edges)."""
    import torch
    films = [_films(torch, j[1], j[2]) for j in batch_scenes]
    jobs = [(j[0], j[1], j[2], j[3], j[4], f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
            for j, f in zip(batch_scenes, films)]
    b = cr.Batch(jobs, max_bounce=7, estimator=estimator, stream=torch.cuda.current_stream().cuda_stream)
    st = b.render(0)
    assert st.samples == sum(j[1] * j[2] * j[3] for j in batch_scenes)
    assert st.rays_extend >= st.samples and st.ms_total > 0
    for job, f in zip(batch_scenes, films):
        ref = _single(cr, torch, job, estimator)
        _assert_same(f, ref)
        assert int(f[2].sum().item()) > 0
    b.close()


def test_batch_graph_replays_accumulate(cr, batch_scenes):
    """Replays of the captured graph with new seed offsets add independent
    samples: two replays equal two stand-alone renders with seeds s and s+1."""
    import torch
    films = [_films(torch, j[1], j[2]) for j in batch_scenes]
    jobs = [(j[0], j[1], j[2], j[3], j[4], f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
            for j, f in zip(batch_scenes, films)]
    b = cr.Batch(jobs, max_bounce=7, estimator=1, stream=torch.cuda.current_stream().cuda_stream)
    b.render(0, stats=False)
    b.render(1, stats=True)
    for job, f in zip(batch_scenes, films):
        ref = _single(cr, torch, job, 1)
        ref = _single(cr, torch, job, 1, seed_add=1, acc=ref)
        _assert_same(f, ref)
    b.close()


@pytest.mark.parametrize("wave", [1000, 4099])
def test_batch_graph_loops_over_many_waves(cr, batch_scenes, wave):
    """Small waves: the graph's device-side loop runs many times (waves that
    cut jobs and pixels at odd places), with the same films as stand-alone
    renders, and the graph holds one wave's kernels, not every wave's."""
    import torch
    films = [_films(torch, j[1], j[2]) for j in batch_scenes]
    jobs = [(j[0], j[1], j[2], j[3], j[4], f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
            for j, f in zip(batch_scenes, films)]
    b = cr.Batch(jobs, max_bounce=7, estimator=1, stream=torch.cuda.current_stream().cuda_stream)
    b.set_tuning(wave_paths=wave)
    st = b.render(0)
    total = sum(j[1] * j[2] * j[3] for j in batch_scenes)
    assert st.samples == total and st.waves == -(-total // wave) and st.waves > 10
    assert st.graph_nodes == 1 + 4 + 3 * 8  # init; begin, generate, 8 x 3 stages, accumulate, end
    assert st.launches == 1 + st.waves * (st.graph_nodes - 1)
    assert st.rays_extend >= total
    for job, f in zip(batch_scenes, films):
        _assert_same(f, _single(cr, torch, job, 1))
    # a replay adds the next seed's samples
    b.render(1, stats=False)
    for job, f in zip(batch_scenes, films):
        ref = _single(cr, torch, job, 1)
        _assert_same(f, _single(cr, torch, job, 1, seed_add=1, acc=ref))
    b.close()


def test_batch_set_tuning_validates(cr, batch_scenes):
    import torch
    f = _films(torch, 8, 8)
    b = cr.Batch([(batch_scenes[0][0], 8, 8, 1, 1, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())])
    for bad in ({"refill_min": 33}, {"traverse_blocks_per_sm": 9}, {"shade_threads": 96}):
        with pytest.raises(cr.CrError):
            b.set_tuning(**bad)
    b.close()


def test_batch_autotune_keeps_results(cr, batch_scenes):
    """The autotuned launch configuration changes the waves, not the film."""
    import torch
    films = [_films(torch, j[1], j[2]) for j in batch_scenes]
    jobs = [(j[0], j[1], j[2], j[3], j[4], f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
            for j, f in zip(batch_scenes, films)]
    b = cr.Batch(jobs, max_bounce=7, estimator=0, stream=torch.cuda.current_stream().cuda_stream)
    t = b.autotune()
    assert t.candidates_tried >= 5 and t.msamples_per_s > 0
    b.render(0)
    for job, f in zip(batch_scenes, films):
        _assert_same(f, _single(cr, torch, job, 0))
    b.close()


def test_batch_rejects_bad_jobs(cr, batch_scenes):
    import torch
    f = _films(torch, 8, 8)
    sc = batch_scenes[0][0]
    ok = (sc, 8, 8, 1, 1, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
    for bad in ((sc, 0, 8, 1, 1, *ok[5:]), (sc, 8, 8, 0, 1, *ok[5:]), (sc, 8, 8, 1, 1, 0, *ok[6:])):
        with pytest.raises(cr.CrError):
            cr.Batch([ok, bad])
    with pytest.raises(cr.CrError):
        cr.Batch([ok], estimator=7)
