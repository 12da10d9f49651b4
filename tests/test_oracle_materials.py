"""The oracle's restatement of the reference's remaining shaders (GlassBSDF,
RefractionBSDF, Transparent, Blackhole, Mixed with Constant and Fresnel fac,
the Cosine distribution) and of the pointLight, against answers of the
reference itself (tests/golden/shaders.npz and materials_*.npz, made by
tests/golden/make_golden.py --materials-only from the reference's compiled
CPU code)."""
import json

import numpy as np
import pytest

from conftest import golden
from golden.make_golden import SHADE_K, scene_hash, shade_records, shader_configs

# float (reference) against FP64 (oracle) on the same draws
F_RTOL, F_ATOL, WI_ATOL = 2e-4, 1e-6, 1e-3


@pytest.fixture(scope="module")
def mats(scenes):
    return scenes.config_materials()


def test_fixtures_unchanged(mats):
    g = golden("shaders.npz")
    assert json.loads(str(g["configs"])) == shader_configs()
    wo, wi, u = shade_records()
    assert np.array_equal(g["wo"], wo) and np.array_equal(g["wi"], wi) and np.array_equal(g["u"], u)
    assert g["u"].shape[1] == SHADE_K
    for f in ("materials_film.npz", "materials_aov_visibility.npz", "materials_aov_halfvector.npz"):
        assert str(golden(f)["scene_hash"]) == scene_hash(mats, full=True)


@pytest.mark.parametrize("index", range(len(shader_configs())))
def test_shader_execute_matches_reference(oracle, index):
    """Per record: the same number of draws, and f / wi / emission within
    float rounding of the reference's own Shader::execute on the same draws."""
    g = golden("shaders.npz")
    cfg = shader_configs()[index]
    out = g["out"][index]
    o = oracle.OracleShader(cfg)
    fe, _, ee, ue = o.execute(0, g["wo"], g["u"], g["wi"])
    fs, ws, es, us = o.execute(1, g["wo"], g["u"], g["wi"])
    assert np.array_equal(ue, out[:, 6]) and np.array_equal(us, out[:, 16]), cfg
    np.testing.assert_allclose(fe, out[:, 0:3], rtol=F_RTOL, atol=F_ATOL)
    np.testing.assert_allclose(ee, out[:, 3:6], rtol=F_RTOL, atol=F_ATOL)
    np.testing.assert_allclose(ws, out[:, 7:10], rtol=0, atol=WI_ATOL)
    np.testing.assert_allclose(fs, out[:, 10:13], rtol=F_RTOL, atol=F_ATOL)
    np.testing.assert_allclose(es, out[:, 13:16], rtol=F_RTOL, atol=F_ATOL)


def test_shader_fixture_exercises_every_branch():
    """The records reach both Mixed branches, Fresnel reflection and
    refraction, total internal reflection (wi left as given) and emission."""
    g = golden("shaders.npz")
    cfgs = shader_configs()
    out = g["out"]
    glass = [i for i, c in enumerate(cfgs) if c[0] == "GlassBSDF"][0]
    refr = [i for i, c in enumerate(cfgs) if c[0] == "RefractionBSDF"][0]
    # refraction past the critical angle keeps wi and returns f = 0
    tir = np.all(out[refr][:, 10:13] == 0, 1)
    assert 0 < tir.mean() < 0.5
    assert np.allclose(out[refr][tir, 7:10], g["wi"][tir])
    # glass: some samples reflect (wo, wi same side), some transmit
    same = g["wo"][:, 2] * out[glass][:, 9] > 0
    live = np.any(out[glass][:, 10:13] != 0, 1)
    assert 0 < (same & live).mean() and 0 < (~same & live).mean()
    nested = len(cfgs) - 1
    em = np.any(out[nested][:, 3:6] != 0, 1)
    assert 0 < em.mean() < 0.5          # the Emission leaf of the nested Mixed
    assert set(np.unique(out[nested][:, 6])) >= {1, 2, 3}  # 1, 2 or 3 draws


def test_materials_render_matches_reference(oracle, mats):
    """Reference semantics through the new shaders and the point light: per
    pixel within 3 sigma of the combined Monte Carlo error.  The reference
    drops about 0.04% of its samples as non-finite (float arithmetic), the
    FP64 oracle none."""
    g = golden("materials_film.npz")
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    f = oracle.OracleScene(mats).render(W, H, spp, int(g["max_bounce"]), oracle.KOISHI, seed=43)
    ref = oracle.Film(g["sum"], g["sumsq"], g["count"])
    assert ref.count.sum() >= 0.999 * W * H * spp and np.all(f.count == spp)
    z = np.abs(f.mean - ref.mean) / np.sqrt(f.var_of_mean + ref.var_of_mean + 1e-30)
    assert (z > 3).mean() < 0.01, (z > 3).mean()
    assert (z > 5).mean() == 0
    assert abs(f.mean.mean() / ref.mean.mean() - 1) < 0.01


@pytest.mark.parametrize("kernel", ["Visibility", "HalfVector"])
def test_point_light_debug_kernels_match_reference(oracle, mats, kernel):
    """Light 0 of the materials scene is the point light: PointLight::sample
    (pointLight.hpp:21-29) through the reference's debug kernels."""
    g = golden(f"materials_aov_{kernel.lower()}.npz")
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    est = oracle.AOV_VISIBILITY if kernel == "Visibility" else oracle.AOV_HALFVECTOR
    f = oracle.OracleScene(mats).render(W, H, spp, 7, est, seed=47)
    ref = oracle.Film(g["sum"], g["sumsq"], g["count"])
    if kernel == "HalfVector":
        # one deterministic direction per sub-pixel sample: pixels agree except at edges
        d = np.abs(f.mean - ref.mean)
        assert (d > 1e-3).mean() < 0.02, (d > 1e-3).mean()
    else:
        floor = (1e-6 * np.maximum(np.abs(f.mean), np.abs(ref.mean))) ** 2
        z = np.abs(f.mean - ref.mean) / np.sqrt(f.var_of_mean + ref.var_of_mean + floor + 1e-30)
        assert (z > 3).mean() < 0.01, (z > 3).mean()
    assert abs(f.mean.mean() / ref.mean.mean() - 1) < 0.01


def test_mis_refuses_reference_only_scenes(oracle, mats):
    with pytest.raises(RuntimeError, match="-2"):
        oracle.OracleScene(mats).render(8, 8, 1, 7, oracle.MIS, seed=1)


def random_shader(rng, depth=0):
    """A random shader config of the reference's registry, Mixed nested up to
    three deep."""
    beck = lambda: ["Beckmann", {"roughness": float(rng.uniform(0.05, 0.8))}]
    dist = lambda: beck() if rng.random() < 0.7 else ["Cosine", {}]
    col = lambda: [float(x) for x in rng.uniform(0.2, 1.0, 3)]
    kinds = ["Lambert", "GlossyBSDF", "Emission", "Transparent", "Blackhole", "RefractionBSDF", "GlassBSDF"]
    if depth < 3:
        kinds += ["Mixed"] * 3
    k = kinds[rng.integers(len(kinds))]
    if k == "Lambert":
        return [k, {"R": col(), "color": col()}]
    if k == "GlossyBSDF":
        return [k, {"distribution": dist(), "color": col()}]
    if k == "Emission":
        return [k, {"color": col(), "strength": float(rng.uniform(1, 10))}]
    if k == "Transparent":
        return [k, {"color": col()}]
    if k == "Blackhole":
        return [k, {}]
    if k in ("RefractionBSDF", "GlassBSDF"):
        return [k, {"ior": float(rng.uniform(1.1, 2.0)), "distribution": dist(), "color": col()}]
    fac = ["Constant", {"value": float(rng.uniform(0, 1))}] if rng.random() < 0.5 else \
        ["Fresnel", {"ior": float(rng.uniform(1.1, 2.0))}]
    return ["Mixed", {"fac": fac, "shaders": [random_shader(rng, depth + 1), random_shader(rng, depth + 1)]}]


def fuzz_records(rng, n, k=16):
    d = rng.normal(size=(2 * n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d[:n].astype(np.float32), d[n:].astype(np.float32), rng.random((n, k)).astype(np.float32)


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference harness not built")
def test_random_shader_trees_match_reference(oracle, tmp_path):
    """Shader::execute of 24 random shader trees (nested Mixed with every
    leaf kind, both distributions and both facs), the reference's own code on
    scripted draws (the harness's `shade` command) against the oracle."""
    rng = np.random.default_rng(2024)
    for i in range(24):
        cfg = random_shader(rng)
        wo, wi, u = fuzz_records(rng, 256)
        (tmp_path / "s.json").write_text(json.dumps(cfg))
        np.concatenate([wo, wi, u], 1).astype(np.float32).tofile(tmp_path / "r.f32")
        oracle.ref_run("shade", "s.json", "r.f32", u.shape[1], "o.f32", cwd=str(tmp_path))
        out = np.fromfile(tmp_path / "o.f32", np.float32).reshape(256, 17)
        o = oracle.OracleShader(cfg)
        fe, _, ee, ue = o.execute(0, wo, u, wi)
        fs, ws, es, us = o.execute(1, wo, u, wi)
        same = (ue == out[:, 6]) & (us == out[:, 16])
        assert same.sum() >= 255, (cfg, np.nonzero(~same))
        np.testing.assert_allclose(fe[same], out[same, 0:3], rtol=F_RTOL, atol=F_ATOL, err_msg=json.dumps(cfg))
        np.testing.assert_allclose(ee[same], out[same, 3:6], rtol=F_RTOL, atol=F_ATOL)
        np.testing.assert_allclose(ws[same], out[same, 7:10], rtol=0, atol=WI_ATOL)
        np.testing.assert_allclose(fs[same], out[same, 10:13], rtol=F_RTOL, atol=F_ATOL)
        np.testing.assert_allclose(es[same], out[same, 13:16], rtol=F_RTOL, atol=F_ATOL)
