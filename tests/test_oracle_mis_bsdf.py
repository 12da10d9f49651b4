"""The MIS estimator's restatement of the remaining shaders (rough dielectric
GlassBSDF and RefractionBSDF after Walter et al. 2007, Transparent as a delta
pass-through, Blackhole, Mixed of two leaves), checked for consistency on
the CPU: the mean sample weight times a smooth test function equals the same
integral taken over uniform directions with the evaluated f (so sampling,
density and f agree), the density integrates to the probability of a
non-delta sample, and no more energy leaves than arrives."""
import numpy as np
import pytest

BECK = ["Beckmann", {"roughness": 0.3}]
CASES = {
    "glass": ["GlassBSDF", {"ior": 1.5, "distribution": BECK}],
    "glass_rough": ["GlassBSDF", {"ior": 1.33, "distribution": ["Beckmann", {"roughness": 0.7}]}],
    "refraction": ["RefractionBSDF", {"ior": 1.5, "distribution": BECK}],
    "coat": ["Mixed", {"fac": ["Fresnel", {"ior": 1.5}], "shaders": [["Lambert", {"R": [0.5, 0.5, 0.5]}],
                                                                    ["GlossyBSDF", {"distribution": BECK}]]}],
    "veil": ["Mixed", {"fac": ["Constant", {"value": 0.3}], "shaders": [["Lambert", {"R": [0.8, 0.8, 0.8]}],
                                                                       ["Transparent", {"color": [0.9, 0.9, 0.9]}]]}],
    "blackhole": ["Blackhole", {}],
}
N = 60000


def _g(w):
    return 1.0 + 0.5 * w[:, 0] - 0.3 * w[:, 1] + 0.25 * w[:, 2]


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("entering", [True, False])
def test_mis_bsdf_sampling_matches_evaluation(oracle, name, entering):
    sh = oracle.OracleShader(CASES[name])
    rng = np.random.default_rng(3)
    wo = np.tile(np.array([0.35, 0.2, 0.915]) / np.linalg.norm([0.35, 0.2, 0.915]), (N, 1))
    wi, w, pdf, delta = sh.mis_sample(wo, rng.random((N, 3)), entering)
    lum = w.mean(1)
    # the sampling-based integral of f |cos| g over the sphere (continuous part)
    a = lum * _g(wi) * ~delta
    # the same by uniform directions over the sphere and the evaluated f
    u = rng.normal(size=(N, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    f, p = sh.mis_eval(wo, u, entering)
    b = f.mean(1) * np.abs(u[:, 2]) * _g(u) * 4 * np.pi
    se = np.sqrt(a.var() / N + b.var() / N) + 1e-12
    assert abs(a.mean() - b.mean()) < 4 * se, (a.mean(), b.mean(), se)
    # the density integrates to the probability of a non-delta sample
    valid = (lum > 0) & ~delta
    dens = p * 4 * np.pi
    assert abs(dens.mean() - valid.mean()) < 4 * np.sqrt(dens.var() / N + 0.25 / N) + 1e-12, (dens.mean(), valid.mean())
    if delta.any():  # the delta lobe: its selection probability times its colour, straight through
        assert np.allclose(wi[delta], -wo[delta])
        assert abs((lum * delta).mean() - 0.3 * 0.9) < 0.02
    # energy: with the radiance scaling of refraction undone, at most what arrives
    eo, et = (1.0, 1.5) if entering else (1.5, 1.0)
    if name == "glass_rough":
        eo, et = (1.0, 1.33) if entering else (1.33, 1.0)
    scale = np.where(wi[:, 2] < 0, (et / eo) ** 2, 1.0) if name in ("glass", "glass_rough", "refraction") else 1.0
    albedo = (lum * scale).mean()
    assert albedo <= 1.0 + 4 * (lum * scale).std() / np.sqrt(N)
    if name == "blackhole":
        assert albedo == 0
    if name in ("glass", "refraction"):
        assert albedo > 0.8  # a moderately rough dielectric loses little to masking


def test_mis_glass_splits_by_fresnel(oracle):
    """At near-normal incidence from outside about 4% reflects (Fresnel at
    ior 1.5); from inside past the critical angle everything reflects."""
    sh = oracle.OracleShader(["GlassBSDF", {"ior": 1.5, "distribution": ["Beckmann", {"roughness": 0.05}]}])
    rng = np.random.default_rng(5)
    wo = np.tile([0.0, 0.0, 1.0], (20000, 1))
    wi, w, _, _ = sh.mis_sample(wo, rng.random((20000, 3)), True)
    refl = wi[:, 2] > 0
    assert 0.03 < refl.mean() < 0.05
    g = np.tile(np.array([0.8, 0.0, 0.6]), (20000, 1))  # 53 degrees, beyond the 41.8 degree critical angle
    wi, w, _, _ = sh.mis_sample(g, rng.random((20000, 3)), False)
    live = w.max(1) > 0
    assert (wi[live, 2] > 0).mean() > 0.97


def test_mis_strategies_agree_on_the_materials_scene(oracle, scenes):
    """The MIS estimator over glass, refraction, pass-through, black and mixed
    surfaces: the power-heuristic combination (estimator 1), BSDF sampling
    alone (2) and the light-sampling weights alone (3) estimate the same image
    (emitter hits after a pass-through count in full in every one, as no
    light sample can reach them)."""
    d = scenes.config_materials(cosine=False, point_light=False)
    o = oracle.OracleScene(d)
    W, H, spp = 20, 20, 512
    films = {v: o.render(W, H, spp, 7, v, seed=61 + v) for v in (1, 2, 3)}
    for v in (2, 3):
        a, b = films[1], films[v]
        z = np.abs(a.mean - b.mean) / np.sqrt(a.var_of_mean + b.var_of_mean + 1e-30)
        assert (z > 3).mean() < 0.02, (v, (z > 3).mean())
        assert abs(b.mean.mean() / a.mean.mean() - 1) < 0.03, (v, a.mean.mean(), b.mean.mean())


def test_mis_point_light_falls_off_with_distance(oracle, scenes):
    """With the point light alone lighting the Lambert box (the panel made a
    black Lambert, the spheres removed), the MIS estimator's direct light at a
    camera ray's hit is albedo / pi * I cos / r^2, I = color * strength."""
    d = scenes.config_materials(cosine=False)
    d.shaders = dict(d.shaders, light=["Lambert", {"R": [0, 0, 0]}])
    d.spheres = []
    o = oracle.OracleScene(d)
    W = H = 16
    film = o.render(W, H, 1, 0, oracle.MIS, seed=3)  # one ray per pixel, no continuation
    px = np.stack(np.meshgrid(np.arange(W), np.arange(H)), -1).reshape(-1, 2)
    ro, rd = scenes.pinhole_rays(d.camera, W, H, 1, px, np.zeros(len(px), int))
    rays = np.concatenate([ro, rd, np.full((len(px), 1), np.inf, np.float32)], 1).astype(np.float32)
    prim, tri, t, _, _ = o.trace(rays)
    pl = d.point_lights[0]
    lpos = np.array(pl["position"], np.float64)
    inten = np.array(pl["color"], np.float32) * np.float32(pl["strength"])
    alb = {g.name: np.array(d.shaders[g.name][1].get("R", [1, 1, 1])) for g in d.groups}
    checked = 0
    for i in range(len(px)):
        if prim[i] < 0:
            continue
        g = d.groups[prim[i]]
        p = ro[i].astype(np.float64) + rd[i].astype(np.float64) * t[i]
        n = g.n[g.f[tri[i]][0]].astype(np.float64)
        if np.dot(n, rd[i]) > 0:
            n = -n
        dl = lpos - p
        r2 = dl @ dl
        cos = max(0.0, dl @ n / np.sqrt(r2))
        seg = np.concatenate([p + n * 1e-4, dl / np.sqrt(r2), [np.sqrt(r2) * (1 - 1e-3)]]).astype(np.float32)
        vis = 0.0 if o.occluded(seg[None])[0] else 1.0
        expect = alb[g.name] / np.pi * inten * cos / r2 * vis
        got = film.mean[px[i, 1], px[i, 0]]
        np.testing.assert_allclose(got, expect, rtol=1e-4, atol=1e-7)
        checked += 1
    assert checked > 200
