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
