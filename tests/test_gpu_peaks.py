"""cfs_fp_peaks (the floating-point roofline's denominator): the measured
CUDA-core rates are positive and plausible for a B200-class device, and packed
FFMA2 is at least as fast as scalar FFMA."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp_peaks_plausible(cfsb):
    p = cfsb.fp_peaks(0)
    assert 10.0 < p["fp32_ffma"] < 400.0, p
    assert 10.0 < p["fp32_ffma2"] < 800.0, p
    assert 1.0 < p["fp64_dfma"] < 200.0, p
    assert p["fp32_ffma2"] > 0.9 * p["fp32_ffma"], p
