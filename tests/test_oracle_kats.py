"""The oracle against the known-answer tests in the reference's own unit tests.

test/sphere.cu:7-18 pins Sphere::intersect on two rays; test/intersect.cu:7-71
pins Seg::intersect_bbox on fifteen segments against the unit box.  The
oracle must reproduce every expected answer.
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
