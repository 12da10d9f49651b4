"""The oracle against the known-answer tests in the reference's own unit tests.

test/sphere.cu:7-18 pins Sphere::intersect on two rays; test/intersect.cu:7-71
pins Seg::intersect_bbox on fifteen segments against the unit box;
test/math.cu:6-29 pins refract (both ways through an ior 1.33 surface) and the
Fresnel scala (ior 1.4 at 45 degrees).  The oracle must reproduce every
expected answer.
"""
import numpy as np
import pytest


def _norm(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v)


def test_sphere_kats(oracle):
    # test/sphere.cu:12-18: Sphere((0,0,0), 1); ray from (2,0,0) along -x hits,
    # along normalize(-1,0,1) misses.
    hit, t = oracle.sphere_hit([0, 0, 0], 1.0, [2, 0, 0, *_norm([-1, 0, 0])])
    assert hit and abs(t - 1.0) < 1e-12
    hit, _ = oracle.sphere_hit([0, 0, 0], 1.0, [2, 0, 0, *_norm([-1, 0, 1])])
    assert not hit


# test/intersect.cu:9-70: (origin, direction before normalisation, expected).
SEG_BOX_KATS = [
    ((2, 0, 0), (-1, 0, 1), True),
    ((2, 0, 0), (-1, 0, 1.01), False),
    ((2, 0, 0), (-1.01, 0, 1), True),
    ((2, 0, 0), (-0.99, 0, 1), False),
    ((2, 2, 0), (-1, -1, 1), True),
    ((2, 2, 0), (-1, -1, 1.01), False),
    ((2, 2, 0), (-1, -1, 0), True),
    ((2, 2, 0), (-0.99, -0.99, 0), False),
    ((0, 0, 2), (0, 0, -2), True),
    ((0, 0, 2), (0, 0, -1), True),
    ((0, 0, 2), (0, 0, -0.99), False),
    ((0, 0, 1e5), (0, 0, -2e5), True),
    ((0.5, 0.5, 1e5), (0, 0, -2e5), True),
    ((0.5, 0.5, 0.5), (0, 0, 0.1), True),
    ((1e-5, 1e-5, 1e-5), (1 - 2e-5, 1 - 2e-5, 1 - 2e-5), True),
]


@pytest.mark.parametrize("o,d,expected", SEG_BOX_KATS)
def test_segment_box_kats(oracle, o, d, expected):
    d32 = np.asarray(d, np.float32)
    ln = np.float32(np.sqrt(np.sum(d32.astype(np.float64) ** 2)))
    seg = [*o, *(d32 / ln), ln]  # Seg{o, normalize(d), length(d)}
    assert oracle.seg_box(seg, [0, 0, 0], [1, 1, 1]) == expected


def test_seg_box_kat_count():
    # test/intersect.cu holds fifteen EXPECT_EQ cases; all are restated above.
    assert len(SEG_BOX_KATS) == 15


# test/math.cu:8-29.  refract and Fresnel are reached through the shaders that
# use them: RefractionBSDF with the Cosine distribution draws h = +z exactly for
# draws (0.5, 0.5) (H::sampleCos's centre), and a Mixed over [Blackhole,
# Transparent] takes Transparent exactly when its draw is below the Fresnel fac.
MATH_KATS = {
    "refract_in": ((1, 0, 1), (-0.531659, -0.0, -0.846958)),
    "refract_out": ((-0.531659, 0, -0.846958), (0.707107, 0.0, 0.707107)),
    "fresnel_1.4": 0.0365785,
}
REFRACT = ["RefractionBSDF", {"ior": 1.33, "distribution": ["Cosine", {}]}]
FRESNEL = ["Mixed", {"fac": ["Fresnel", {"ior": 1.4}], "shaders": [["Blackhole", {}], ["Transparent", {}]]}]


def math_kat_inputs():
    """(wo, draws) for the two refractions and the two sides of the Fresnel fac."""
    wo = np.array([_norm(MATH_KATS["refract_in"][0]), _norm(MATH_KATS["refract_out"][0])])
    f = MATH_KATS["fresnel_1.4"]
    u_fr = np.array([[f - 1e-4, 0.5, 0.5, 0.5], [f + 1e-4, 0.5, 0.5, 0.5]])
    return wo, np.full((2, 3), 0.5), np.repeat(_norm([1, 0, 1])[None], 2, 0), u_fr


def test_math_kats(oracle):
    wo, u, wo_fr, u_fr = math_kat_inputs()
    f, wi, _, used = oracle.OracleShader(REFRACT).execute(1, wo, u)
    assert np.all(used == 3)
    np.testing.assert_allclose(wi[0], MATH_KATS["refract_in"][1], atol=1e-4)
    np.testing.assert_allclose(wi[1], MATH_KATS["refract_out"][1], atol=1e-4)
    # entering scales by 1/eta^2 = ior^2; leaving keeps the colour
    np.testing.assert_allclose(f[:, 0], [1.33 ** 2, 1.0], rtol=1e-6)
    f, wi, _, _ = oracle.OracleShader(FRESNEL).execute(1, wo_fr, u_fr)
    assert np.all(f[0] == 1) and np.allclose(wi[0], -wo_fr[0])  # below the fac: Transparent
    assert np.all(f[1] == 0)                                      # above it: Blackhole

