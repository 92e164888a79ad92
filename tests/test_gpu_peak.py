"""The FMA peak microbenchmark the plain form's roofline is reported against
(kmb_measure_fma_peak): FP32 scalar, packed FP32 pairs (fma.rn.f32x2) and FP64
give plausible B200 figures, and an unknown precision is rejected."""
import ctypes

import pytest

from onedal_b200 import _native

pytestmark = pytest.mark.gpu


def _peak(dtype):
    g = ctypes.c_double()
    rc = _native.load_library().kmb_measure_fma_peak(0, dtype, ctypes.byref(g))
    return rc, g.value / 1e3


def test_fma_peaks_are_plausible():
    rc32, f32 = _peak(_native.KMB_F32)
    rc2, f32x2 = _peak(_native.KMB_FMA_PEAK_F32X2)
    rc64, f64 = _peak(_native.KMB_F64)
    assert rc32 == rc2 == rc64 == _native.KMB_OK
    # 148 SMs x 128 FP32 lanes x 2 flops x ~1.9 GHz = 72 TFLOP/s
    assert 30.0 < f32 < 120.0, f32
    assert 0.8 * f32 < f32x2 < 2.5 * f32, (f32, f32x2)
    assert 0.1 < f64 < f32, (f64, f32)


def test_fma_peak_rejects_unknown_precision():
    g = ctypes.c_double()
    assert _native.load_library().kmb_measure_fma_peak(0, 7, ctypes.byref(g)) == _native.KMB_EINVAL
