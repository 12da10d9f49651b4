"""cr_measure_peaks: the in-run L2 and FP32 rooflines are plausible for a B200
(L2 reads above the HBM copy figure, FP32 between 10 and 200 TFLOP/s)."""
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu


def test_measure_peaks(cr):
    require_gpu()
    l2, fp32 = cr.measure_peaks()
    assert 4000.0 < l2 < 100000.0, l2
    assert 10.0 < fp32 < 200.0, fp32


def test_gather_peak_is_measured(cr):
    """Random record gathers from an L2-resident array: a positive rate below
    the streaming L2 read rate, and refused for unsupported record sizes."""
    require_gpu()
    import cuda_raytracer_b200 as crm
    l2, _ = cr.measure_peaks()
    for rb in (80, 48):
        g = cr.measure_gather(rb, 64 << 20)
        assert 100 < g < 1.5 * l2, (rb, g, l2)
    with pytest.raises(crm.CrError):
        cr.measure_gather(64, 64 << 20)
