"""The CUDA path guide against the FP64 guide oracle (forward outputs and
training gradients), and guided rendering against plain MIS rendering (the
guide changes the variance, never the expectation)."""
import numpy as np
import pytest

import guide_oracle as G
import oracle as O
from conftest import require_gpu
from gpu_util import render_film, zscores

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def guided(cr, scenes):
    require_gpu()
    s = cr.Scene.from_desc(scenes.config0())
    g = cr.Guide(s).reset(seed=5)
    rng = np.random.default_rng(7)
    grid = rng.uniform(-0.5, 0.5, (G.LEVELS, G.T, G.FEAT)).astype(np.float32)
    W = rng.uniform(-0.3, 0.3, (G.LAYERS, 64, 64)).astype(np.float32)
    W[0][:, 43:] = 0
    b = rng.uniform(-0.1, 0.1, (G.LAYERS, 64)).astype(np.float32)
    g.set_params(grid, W, b)
    info = g.info()
    return s, g, grid.astype(np.float64), W.astype(np.float64), b.astype(np.float64), info


def _inputs(rng, n):
    x = rng.uniform(0.5, 5.0, (n, 3))
    wo = rng.normal(size=(n, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    nn = rng.normal(size=(n, 3)); nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    return np.concatenate([x, wo, nn], 1).astype(np.float32)


def test_forward_matches_fp64(guided):
    s, g, grid, W, b, info = guided
    rng = np.random.default_rng(1)
    inp = _inputs(rng, 200)
    out = g.forward(inp)
    for i in range(0, 200, 5):
        h0, _ = G.encode(grid, info["bmin"].astype(np.float64), info["binv"].astype(np.float64),
                         inp[i, :3].astype(np.float64), inp[i, 3:6].astype(np.float64), inp[i, 6:9].astype(np.float64))
        ref, _ = G.forward(W, b, h0)
        np.testing.assert_allclose(out[i], ref, rtol=2e-4, atol=2e-4 * np.abs(ref).max())


def test_tc_forward_matches_fp64(guided):
    """The BF16 tensor-core forward (tcgen05, FP32 accumulation) the renderer
    samples with, against the FP64 network: BF16 rounding of the inputs,
    activations and weights bounds the error to about 1% of the output
    scale.  1000 rows: three full CTA iterations of 256 rows and a ragged tail."""
    s, g, grid, W, b, info = guided
    rng = np.random.default_rng(11)
    n = 1000
    inp = _inputs(rng, n)
    out = g.forward(inp, tensor_cores=True)
    fp32 = g.forward(inp)
    ref = np.zeros((n, 64))
    for i in range(n):
        h0, _ = G.encode(grid, info["bmin"].astype(np.float64), info["binv"].astype(np.float64),
                         inp[i, :3].astype(np.float64), inp[i, 3:6].astype(np.float64), inp[i, 6:9].astype(np.float64))
        ref[i], _ = G.forward(W, b, h0)
    scale = np.abs(ref).max()
    err = np.abs(out - ref)
    assert err.max() < 0.03 * scale, err.max() / scale
    rel = np.linalg.norm(out - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert np.median(rel) < 0.01, np.median(rel)
    # the FP32 CUDA-core path is far closer: the gap is the BF16 rounding
    assert np.abs(fp32 - ref).max() < 1e-3 * scale


@pytest.mark.parametrize("n", [0, 1, 3, 255, 257])
def test_tc_forward_ragged_sizes(guided, n):
    """Empty, single-row and ragged batches (any n, the output row offsets
    stay 16-byte aligned) agree with the FP32 path to BF16 accuracy."""
    s, g, grid, W, b, info = guided
    rng = np.random.default_rng(100 + n)
    inp = _inputs(rng, n)
    out = g.forward(inp, tensor_cores=True)
    assert out.shape == (n, 64)
    if n:
        ref = g.forward(inp)
        assert np.abs(out - ref).max() < 0.03 * np.abs(ref).max()


def test_guide_configure_validates(guided):
    s, g, grid, W, b, info = guided
    import cuda_raytracer_b200 as crm
    cfg = g.configure()
    assert cfg["train_paths"] == 32768 and cfg["steps_per_wave"] == 64 and cfg["warmup_steps"] == 8
    assert cfg["product_target"] == 1 and cfg["guided_bounces"] == 0
    for bad in ({"lr": 0.0}, {"select_prob": 1.0}, {"train_paths": 0}, {"steps_per_wave": 65}):
        with pytest.raises(crm.CrError):
            g.configure(**bad)
    assert g.configure() == cfg  # a rejected schedule changes nothing


def test_gradients_match_fp64(guided):
    s, g, grid, W, b, info = guided
    rng = np.random.default_rng(2)
    n = 64
    inp = _inputs(rng, n)
    om = rng.normal(size=(n, 3)); om /= np.linalg.norm(om, axis=1, keepdims=True)
    wts = rng.uniform(0.05, 3.0, n)
    wts[::9] = 0.0  # some records carry no weight
    recs = np.concatenate([inp, om, wts[:, None]], 1).astype(np.float32)
    ggrid, gW, gb = g.gradients(recs)
    rW, rb, rgrid = G.gradients(grid, W, b, info["bmin"].astype(np.float64), info["binv"].astype(np.float64),
                                recs.astype(np.float64))
    for got, ref in ((gW, rW), (gb, rb), (ggrid, rgrid)):
        got = got.reshape(ref.shape)
        rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert rel < 2e-3, rel


def test_tc_gradients_match_fp64(guided):
    """The tensor-core training pass (BF16 operands, FP32 accumulation) against
    the BF16-emulating FP64 restatement, record by record and in one batch of
    300 records (three 128-row tiles with a ragged tail).

    The emulation rounds where the kernel rounds, so only the order of the
    FP32 accumulations separates them; on most records the two agree to a few
    FP32 ulps.  Some records' gradients are ill-conditioned: their lower-layer
    gradients are small differences of large terms, so that BF16 rounding
    alone moves them by tens of percent (the emulation against exact FP64),
    and an accumulation-order difference that flips one BF16 rounding moves
    them as much.  Such a record may leave the emulation by no more than
    twice its own BF16 sensitivity; the batch is compared on the
    well-conditioned records."""
    s, g, grid, W, b, info = guided
    rng = np.random.default_rng(3)
    n = 300
    inp = _inputs(rng, n)
    om = rng.normal(size=(n, 3)); om /= np.linalg.norm(om, axis=1, keepdims=True)
    wts = rng.uniform(0.05, 3.0, n)
    wts[::7] = 0.0
    recs = np.concatenate([inp, om, wts[:, None]], 1).astype(np.float32)
    bmin, binv = info["bmin"].astype(np.float64), info["binv"].astype(np.float64)
    rel = lambda a, e: np.linalg.norm(a - e) / max(np.linalg.norm(e), 1e-300)
    close, well = 0, []
    for i in np.nonzero(wts > 0)[0]:
        r64 = recs[i:i + 1].astype(np.float64)
        _, gW, gb = g.gradients(recs[i:i + 1], tensor_cores=True)
        gW, gb = gW.reshape(W.shape), gb.reshape(b.shape)
        eW, eb, _ = G.gradients_bf16(grid, W, b, bmin, binv, r64)
        xW, xb, _ = G.gradients(grid, W, b, bmin, binv, r64)
        for l in range(G.LAYERS):
            sens = rel(eW[l], xW[l])
            assert rel(gW[l], eW[l]) <= 2.0 * sens + 5e-3, (i, l, rel(gW[l], eW[l]), sens)
            assert rel(gb[l], eb[l]) <= 2.0 * rel(eb[l], xb[l]) + 5e-3, (i, l)
        close += rel(gW, eW) < 5e-3
        if rel(eW, xW) < 0.05:
            well.append(i)
    assert close >= 0.9 * int((wts > 0).sum()), close
    assert len(well) >= 0.8 * int((wts > 0).sum()), len(well)
    # one batch of the well-conditioned records (zero-weight rows kept as padding)
    sel = recs[[i for i in range(n) if i in set(well) or wts[i] == 0]]
    ggrid, gW, gb = g.gradients(sel, tensor_cores=True)
    rW, rb, rgrid = G.gradients(grid, W, b, bmin, binv, sel.astype(np.float64))
    eW, eb, egrid = G.gradients_bf16(grid, W, b, bmin, binv, sel.astype(np.float64))
    errs = {}
    for name, got, ref, emu in (("W", gW, rW, eW), ("b", gb, rb, eb), ("grid", ggrid, rgrid, egrid)):
        got = got.reshape(ref.shape)
        errs[name] = (rel(got, ref), rel(got, emu))
    for l in range(G.LAYERS):
        errs[f"W{l}"] = (0.0, rel(gW.reshape(rW.shape)[l], eW[l]))
    for name, (exact, emulated) in errs.items():
        assert emulated < 5e-3, (name, errs)
        assert exact < 0.15, (name, errs)


def test_gradients_where_every_lobe_density_underflows(guided):
    """Every lobe sharp (kappa near 2000) and far from the recorded
    directions: the mixture density underflows in FP32, yet the log-space
    responsibilities give the FP64 oracle's gradients."""
    s, g, grid, W, b, info = guided
    b2 = b.copy()
    b2[4][3:40:5] = 2000.0
    g.set_params(None, None, b2.astype(np.float32))
    try:
        rng = np.random.default_rng(21)
        n = 64
        inp = _inputs(rng, n)
        om = rng.normal(size=(n, 3)); om /= np.linalg.norm(om, axis=1, keepdims=True)
        recs = np.concatenate([inp, om, rng.uniform(0.1, 2.0, (n, 1))], 1).astype(np.float32)
        ggrid, gW, gb = g.gradients(recs)
        rW, rb, rgrid = G.gradients(grid, W, b2, info["bmin"].astype(np.float64), info["binv"].astype(np.float64),
                                    recs.astype(np.float64))
        for got, ref in ((gW, rW), (gb, rb), (ggrid, rgrid)):
            got = got.reshape(ref.shape)
            assert np.isfinite(got).all()
            assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 5e-3
    finally:
        g.set_params(None, None, b.astype(np.float32))


@pytest.mark.parametrize("tensor_cores", [False, True])
def test_selection_gradients_match_fp64(guided, tensor_cores):
    """Learned selection: records carry the BSDF density of their direction
    and the loss fits the one-sample mixture s q + (1 - s) p_bsdf; the
    gradients of both passes, selection logit included, against FP64 (the
    tensor-core pass against the BF16-emulating FP64 restatement)."""
    s, g, grid, W, b, info = guided
    g.configure(learn_select=1)
    try:
        rng = np.random.default_rng(9)
        n = 300
        inp = _inputs(rng, n)
        om = rng.normal(size=(n, 3)); om /= np.linalg.norm(om, axis=1, keepdims=True)
        wts = rng.uniform(0.05, 3.0, n)
        wts[::7] = 0.0
        pb = rng.uniform(0.0, 1.5, n)
        pb[::5] = 0.0
        recs = np.concatenate([inp, om, wts[:, None], pb[:, None]], 1).astype(np.float32)
        ggrid, gW, gb = g.gradients(recs, tensor_cores=tensor_cores)
        bmin, binv = info["bmin"].astype(np.float64), info["binv"].astype(np.float64)
        fn = G.gradients_bf16 if tensor_cores else G.gradients
        rW, rb, rgrid = fn(grid, W, b, bmin, binv, recs.astype(np.float64), learn_select=True)
        tol = 5e-3 if tensor_cores else 2e-3
        for got, ref in ((gW, rW), (gb, rb), (ggrid, rgrid)):
            got = got.reshape(ref.shape)
            rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert rel < tol, rel
        # the selection logit's bias gradient itself
        assert abs(gb.reshape(rb.shape)[4, 40] - rb[4, 40]) <= tol * np.abs(rb[4]).max() + 1e-6
        assert abs(rb[4, 40]) > 0
    finally:
        g.configure(learn_select=0)


@pytest.mark.parametrize("guided_bounces", [3, 0, 1])
def test_guided_render_is_unbiased(cr, scenes, guided_bounces):
    """Guided MIS and plain MIS films agree within 3 sigma: one-sample MIS of
    the learned mixture with the BSDF keeps the estimator unbiased while the
    guide trains online during the render, whichever vertices (the first 3,
    all but the last, the first) sample the guide."""
    require_gpu()
    d = scenes.config0()
    s = cr.Scene.from_desc(d)
    gd = cr.Guide(s).reset(seed=3)
    # sample the guide from the third wave on
    gd.configure(steps_per_wave=2, warmup_steps=4, guided_bounces=guided_bounces, max_steps=600,
                 learn_select=int(guided_bounces == 3))
    W, H, spp = 32, 32, 256
    plain = render_film(cr, s, W, H, spp, seeds=[21, 22], estimator=cr.MIS)
    import torch
    n = W * H
    acc = [torch.zeros(n * 3, dtype=torch.float64, device="cuda"), torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
           torch.zeros(n, dtype=torch.int32, device="cuda")]
    for seed in (31, 32):
        desc = cr.render_desc(W, H, spp, max_bounce=7, estimator=cr.MIS, seed=seed, guiding=True, wave_paths=65536)
        s.render_device(desc, acc[0].data_ptr(), acc[1].data_ptr(), acc[2].data_ptr(),
                        stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    guided = O.Film(acc[0].cpu().numpy().reshape(H, W, 3), acc[1].cpu().numpy().reshape(H, W, 3),
                    acc[2].cpu().numpy().astype(np.uint32).reshape(H, W))
    assert cr.Guide(s).info()["step"] == 16  # 2 renders x 4 waves, two steps each
    z = zscores(guided, plain)
    assert (z > 3).mean() < 0.01, (z > 3).mean()
    # the image means: their difference against its standard error (all pixels)
    diff = guided.mean.sum() - plain.mean.sum()
    se = np.sqrt((guided.var_of_mean + plain.var_of_mean).sum())
    assert abs(diff) < 4 * se, (diff / se, guided.mean.mean(), plain.mean.mean())


def test_guide_train_spends_the_budget_exactly(cr, scenes):
    """cr_guide_train: scratch passes of about one recorded wave each until the
    budget is spent, then guided renders run with the frozen guide; a guide
    without a budget is refused."""
    require_gpu()
    import torch
    s = cr.Scene.from_desc(scenes.config0())
    try:
        g = cr.Guide(s).reset(seed=3)
        g.configure(max_steps=96, steps_per_wave=16, train_paths=8192, warmup_steps=4)
        d = cr.render_desc(256, 256, 1, max_bounce=7, estimator=cr.MIS, seed=9, guiding=True)
        passes = g.train(d)
        # 16 x 8192 = 131,072 paths per pass at 2 spp of 256 x 256: 16 steps per pass
        assert g.info()["step"] == 96 and passes == 6
        f = [torch.zeros(256 * 256 * 3, dtype=torch.float64, device="cuda"),
             torch.zeros(256 * 256 * 3, dtype=torch.float64, device="cuda"),
             torch.zeros(256 * 256, dtype=torch.int32, device="cuda")]
        d4 = cr.render_desc(256, 256, 4, max_bounce=7, estimator=cr.MIS, seed=11, guiding=True)
        st = s.render_device(d4, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
        torch.cuda.synchronize()
        assert g.info()["step"] == 96  # frozen
        # inference on bounces 0..6 of every wave (never the last vertex), on
        # each bounce's whole extension queue; no training time once frozen
        assert st.guide_launches == 7 * st.waves
        assert st.samples <= st.guide_rows < st.rays_extend
        assert st.ms_guide > 0 and st.ms_guide_train == 0
        assert np.isfinite(f[0].cpu().numpy()).all() and int(f[2].sum().item()) > 0
        g.configure(max_steps=0)
        with pytest.raises(cr.CrError):
            g.train(d)
    finally:
        s.close()
