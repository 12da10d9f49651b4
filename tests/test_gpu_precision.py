"""Precision study on the 1.31M-triangle workload (FP32 CUDA path against the
FP64 oracle): hit-id agreement and relative t error on primary and secondary
rays, and the per-pixel error of a converged MIS render.  The figures are
printed on one line starting with PRECISION (pytest -s shows it)."""
import json

import numpy as np
import pytest

from conftest import require_gpu
from gpu_util import render_film, zscores

pytestmark = pytest.mark.gpu

W, H = 1024, 768


@pytest.fixture(scope="module")
def c1(cr, scenes, oracle):
    require_gpu()
    desc = scenes.config1(level=8)
    return desc, cr.Scene.from_desc(desc), oracle.OracleScene(desc)


def _rays(scenes, desc, sc, n, seed):
    """n primary rays (random pixels and sample indices of the 1024x768x256
    image) and n secondary rays leaving their hit points in random directions
    of the hemisphere facing the camera ray's origin side."""
    rng = np.random.default_rng(seed)
    px = np.stack([rng.integers(0, W, n), rng.integers(0, H, n)], 1)
    o, d = scenes.pinhole_rays(desc.camera, W, H, 256, px, rng.integers(0, 256, n))
    prim = np.zeros((n, 7), np.float32)
    prim[:, :3], prim[:, 3:6], prim[:, 6] = o, d, np.inf
    h = sc.trace(prim)
    ok = h["prim"] >= 0
    p = (o + d * (h["t"][:, None] * (1 - 1e-4))).astype(np.float32)[ok]
    nd = rng.normal(size=(len(p), 3))
    nd /= np.linalg.norm(nd, axis=1, keepdims=True)
    back = -d[ok]
    nd = np.where((nd * back).sum(1, keepdims=True) < 0, -nd, nd)  # towards the side the ray came from
    sec = np.zeros((len(p), 7), np.float32)
    sec[:, :3], sec[:, 3:6], sec[:, 6] = p, nd.astype(np.float32), np.inf
    return prim, sec


def test_c1_precision_study(cr, scenes, oracle, c1):
    desc, sc, orc = c1
    prim, sec = _rays(scenes, desc, sc, 100_000, 2024)
    report = {}
    for name, rays in (("primary", prim), ("secondary", sec)):
        hits = sc.trace(rays)
        p, tri, t, _, _ = orc.trace(rays)
        same = (hits["prim"] == p) & (hits["tri"] == tri)
        both = same & (p >= 0) & (p < len(desc.groups))
        err = np.abs(hits["t"][both].astype(np.float64) - t[both])
        # |cos| between the ray and the hit triangle's plane normal
        cosv = np.zeros(int(both.sum()))
        for gi in np.unique(p[both]):
            g = desc.groups[gi]
            sel = p[both] == gi
            f = g.f[tri[both][sel]]
            v0, v1, v2 = (g.v[f[:, k]].astype(np.float64) for k in range(3))
            nrm = np.cross(v1 - v0, v2 - v0)
            nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
            cosv[sel] = np.abs((nrm * rays[both][sel, 3:6]).sum(1))
        # FP32 world coordinates (|o| up to ~6) carry ~1e-6 of absolute error, so
        # the relative bound applies away from the ray origin; t of a grazing hit
        # moves by that error over |cos|
        far = t[both] >= 0.05
        steep = far & (cosv >= 0.05)
        rel = err / t[both]
        scale = np.abs(rays[both, :3]).max(1) + 1.0
        report[name] = {"rays": int(len(rays)), "hit_id_agreement": float(same.mean()),
                        "rel_t_err_max": float(rel[steep].max()), "rel_t_err_p999": float(np.quantile(rel[steep], 0.999)),
                        "rel_t_err_mean": float(rel[steep].mean()),
                        "grazing_or_near_origin_hits": int((~steep).sum()),
                        "rel_t_err_max_grazing_or_near": float(rel[~steep].max()) if (~steep).any() else 0.0,
                        "abs_t_err_times_cos_over_origin_scale_max": float((err * np.maximum(cosv, 1e-3) / scale).max())}
        assert same.mean() >= 0.999, (name, report[name])
        assert rel[steep].max() <= 1e-5, (name, report[name])
        assert (err * np.maximum(cosv, 1e-3) / scale).max() <= 1e-6, (name, report[name])
    # MIS render of a 64 x 48 window at the image centre, FP32 and FP64 at the
    # same spp: the glossy materials (roughness down to 0.05) make per-pixel
    # estimates heavy-tailed, so the two films get the same number of samples
    # and the check also runs on 4 x 4 blocks
    win = (W // 2 - 32, H // 2 - 24, W // 2 + 32, H // 2 + 24)
    spp = 512
    o = orc.render(W, H, spp, 7, oracle.MIS, seed=9, window=win)
    g = render_film(cr, sc, W, H, spp, seeds=[21], estimator=cr.MIS, window=win)
    z = zscores(g, o)
    den = o.mean ** 2 + 1e-2
    raw = float((((g.mean - o.mean) ** 2) / den).mean())
    noise = float(((g.var_of_mean + o.var_of_mean) / den).mean())
    blk = lambda a: a.reshape(12, 4, 16, 4, 3).sum((1, 3))
    zb = np.abs(blk(g.mean) - blk(o.mean)) / np.sqrt(blk(g.var_of_mean) + blk(o.var_of_mean))
    diff = (g.mean - o.mean).sum() / np.sqrt((g.var_of_mean + o.var_of_mean).sum())
    report["render"] = {"window": list(win), "spp_each": spp, "relmse_fp32_vs_fp64": raw,
                        "relmse_expected_from_noise": noise, "frac_pixels_beyond_3_sigma": float((z > 3).mean()),
                        "frac_4x4_blocks_beyond_3_sigma": float((zb > 3).mean()),
                        "image_mean_diff_in_standard_errors": float(diff)}
    print("PRECISION " + json.dumps(report))
    assert (z > 3).mean() < 0.02, report["render"]
    assert (zb > 3).mean() < 0.03, report["render"]
    assert abs(diff) < 4, report["render"]
    # the FP32 path adds no error beyond the Monte Carlo noise of the two films
    assert raw < 1.3 * noise, report["render"]
