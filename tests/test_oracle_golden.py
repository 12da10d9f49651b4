"""The FP64 oracle against answers of the reference itself (tests/golden/,
made by tests/golden/make_golden.py from the reference's compiled CPU path)."""
import numpy as np
import pytest

from conftest import golden
from golden.make_golden import ico_scene, scene_hash


@pytest.fixture(scope="module")
def c0(scenes):
    return scenes.config0()


def test_fixture_scenes_unchanged(c0):
    assert str(golden("c0_trace.npz")["scene_hash"]) == scene_hash(c0)
    assert str(golden("ico_trace.npz")["scene_hash"]) == scene_hash(ico_scene())


def test_light_table_matches_reference(oracle, c0):
    g = golden("c0_lights.npz")
    o = oracle.OracleScene(c0, light_seed=int(g["seed"]))
    pts, pdf = o.light_table(0)
    # Same generator, same face order (padding copies included), same float
    # arithmetic; only FMA contraction may differ between the two builds.
    np.testing.assert_allclose(pts, g["table"], rtol=0, atol=2e-6)
    assert abs(pdf - float(g["pdf"])) <= 1e-7 * abs(pdf)
    assert int(g["n_faces"]) == 4  # 2 triangles padded to 4 (mesh.cu:137-141)


def _hit_ids(o, rays, prim_kind):
    prim, tri, t, _, _ = o.trace(rays)
    kind = np.where(prim >= 0, np.asarray(prim_kind)[np.maximum(prim, 0)], -1)
    # group index for meshes, sphere index for spheres
    n_mesh = sum(1 for k in prim_kind if k == 0)
    index = np.where(kind == 0, prim, np.where(kind == 1, prim - n_mesh, -1))
    return kind, index, tri, t


@pytest.mark.parametrize("fixture,make", [("c0_trace.npz", None), ("ico_trace.npz", ico_scene)])
def test_hit_ids_match_reference(oracle, c0, fixture, make):
    g = golden(fixture)
    desc = make() if make else c0
    o = oracle.OracleScene(desc)
    kind, index, tri, t = _hit_ids(o, g["rays"], o.prim_kind)
    same = (kind == g["kind"]) & (index == g["index"]) & (tri == g["tri"])
    # Disagreements are allowed only at documented near-ties: equal distance
    # within 1e-6 relative (shared edges, padding duplicates).
    rt = g["t"].astype(np.float64)
    tie = np.abs(t - rt) <= 1e-6 * np.maximum(np.abs(rt), 1e-6)
    assert np.all(same | tie), np.nonzero(~(same | tie))[0][:10]
    assert same.mean() > 0.995
    hit = g["kind"] >= 0
    assert np.all((kind >= 0) == hit)
    np.testing.assert_allclose(t[hit], rt[hit], rtol=2e-5)


def test_occlusion_matches_reference(oracle, c0):
    g = golden("c0_occlude.npz")
    o = oracle.OracleScene(c0)
    occ = o.occluded(g["segs"])
    assert (occ == g["occluded"]).mean() >= 0.999
    assert 0.05 < g["occluded"].mean() < 0.95  # the fixture exercises both answers


def test_koishi_render_matches_reference(oracle, c0):
    """Oracle (reference semantics, FP64) vs the reference's own render: per
    pixel within 3 sigma of the combined Monte Carlo standard error."""
    g = golden("c0_film.npz")
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    o = oracle.OracleScene(c0)
    f = o.render(W, H, spp, int(g["max_bounce"]), oracle.KOISHI, seed=23)
    ref = oracle.Film(g["sum"], g["sumsq"], g["count"])
    assert np.all(ref.count == spp) and np.all(f.count == spp)
    z = np.abs(f.mean - ref.mean) / np.sqrt(f.var_of_mean + ref.var_of_mean + 1e-30)
    assert (z > 3).mean() < 0.01, (z > 3).mean()
    assert (z > 5).mean() == 0
    # image-level agreement of the mean
    rel = abs(f.mean.mean() - ref.mean.mean()) / ref.mean.mean()
    assert rel < 0.01


@pytest.mark.parametrize("kernel", ["Normal", "Visibility", "HalfVector"])
def test_debug_kernels_match_reference(oracle, c0, kernel):
    """The oracle's restatement of the reference's debug kernels against the
    reference's own renders of them (NormalKernel, VisibilityKernel,
    HalfVectorKernel through the harness).  Normal is deterministic per
    sub-pixel sample: pixels agree except where an object edge splits the
    pixel's samples; the two light-sampling kernels agree within 3 sigma."""
    g = golden(f"c0_aov_{kernel.lower()}.npz")
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    est = {"Normal": oracle.AOV_NORMAL, "Visibility": oracle.AOV_VISIBILITY, "HalfVector": oracle.AOV_HALFVECTOR}[kernel]
    f = oracle.OracleScene(c0).render(W, H, spp, 7, est, seed=29)
    ref = oracle.Film(g["sum"], g["sumsq"], g["count"])
    assert np.all(ref.count == spp) and np.all(f.count == spp)
    if kernel == "Normal":
        d = np.abs(f.mean - ref.mean)
        assert (d > 1e-3).mean() < 0.02, (d > 1e-3).mean()
        assert abs(f.mean.mean() - ref.mean.mean()) < 1e-4
    else:
        floor = (1e-6 * np.maximum(np.abs(f.mean), np.abs(ref.mean))) ** 2
        z = np.abs(f.mean - ref.mean) / np.sqrt(f.var_of_mean + ref.var_of_mean + floor + 1e-30)
        assert (z > 3).mean() < 0.01, (z > 3).mean()
        assert abs(f.mean.mean() / ref.mean.mean() - 1) < 0.01


def test_orthographic_render_matches_reference(oracle, scenes):
    """OrthographicLens::sample (lens.hpp:40-53) through the reference's own
    render of config 0 (tests/golden/c0_ortho_film.npz)."""
    g = golden("c0_ortho_film.npz")
    d = scenes.config0_ortho()
    assert str(g["scene_hash"]) == scene_hash(d, full=True) and str(g["lens"]) == "orthographic"
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    f = oracle.OracleScene(d).render(W, H, spp, int(g["max_bounce"]), oracle.KOISHI, seed=61)
    ref = oracle.Film(g["sum"], g["sumsq"], g["count"])
    z = np.abs(f.mean - ref.mean) / np.sqrt(f.var_of_mean + ref.var_of_mean + 1e-30)
    assert (z > 3).mean() < 0.01 and (z > 5).mean() == 0, ((z > 3).mean(), z.max())
    assert abs(f.mean.mean() / ref.mean.mean() - 1) < 0.01


def _sphere_t_allowance(desc, rays, idx, t):
    """1e-5 relative, plus what FP32 ray-sphere arithmetic loses on small far
    spheres: the direction is unit length to ~1e-7 and the reference's
    |oc|^2 - (d.oc)^2 cancels, both moving t by about |oc|^2 * 1e-7 / sqrt(det),
    with sqrt(det) = |cos| r at the hit."""
    cen = np.array([desc.spheres[i]["o"] for i in idx], np.float64)
    rad = np.array([desc.spheres[i]["r"] for i in idx], np.float64)
    ro, rd = rays[:, :3].astype(np.float64), rays[:, 3:6].astype(np.float64)
    nrm = (ro + rd * t[:, None] - cen) / rad[:, None]
    cos = np.abs((nrm * rd).sum(1))
    return 1e-5 * t + 5e-7 * ((cen - ro) ** 2).sum(1) / np.maximum(cos * rad, 1e-3)


def test_sphere_field_matches_reference(oracle):
    """Closest hits on 300 spheres: the oracle against the reference's own
    Sphere::intersect over every sphere (tests/golden/spheres_trace.npz)."""
    from golden.make_golden import sphere_field
    g = golden("spheres_trace.npz")
    d = sphere_field()
    assert str(g["scene_hash"]) == scene_hash(d)
    p, tri, t, _, _ = oracle.OracleScene(d).trace(g["rays"])
    kind = np.where(p < 0, -1, 1)
    assert np.array_equal(kind, g["kind"]) and np.array_equal(np.where(p < 0, -1, p), g["index"])
    hit = p >= 0
    assert 0.3 < hit.mean() < 0.9
    err = np.abs(t[hit] - g["t"][hit])
    assert (err <= _sphere_t_allowance(d, g["rays"][hit], p[hit], t[hit])).all()


def test_ico_render_matches_reference(oracle):
    """The reference estimator on the displaced icosphere (5120 triangles,
    Lambert and Beckmann patches, 20 meshes) against the reference's own
    render (tests/golden/ico_film.npz).  The Beckmann patches down to
    roughness 0.05 make the image mean heavy-tailed: two reference renders of
    this scene differ by 0.6 % in it, three times their sample standard
    error, so the image-level check allows 2 %."""
    g = golden("ico_film.npz")
    d = ico_scene()
    assert str(g["scene_hash"]) == scene_hash(d, full=True)
    W, H, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    f = oracle.OracleScene(d).render(W, H, spp, int(g["max_bounce"]), oracle.KOISHI, seed=67)
    ref = oracle.Film(g["sum"], g["sumsq"], g["count"])
    z = np.abs(f.mean - ref.mean) / np.sqrt(f.var_of_mean + ref.var_of_mean + 1e-30)
    assert (z > 3).mean() < 0.01 and (z > 5).mean() == 0, ((z > 3).mean(), z.max())
    assert abs(f.mean.mean() / ref.mean.mean() - 1) < 0.02
