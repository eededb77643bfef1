"""The FMA throughput measurement behind the FP64 denominator: positive,
plausible for a B200 (tens of FP64 TFLOP/s), and FP32 above FP64."""
import ctypes

import pytest

from canoe_b200._abi import check, load

pytestmark = pytest.mark.gpu


def test_fma_peaks_plausible():
    lib = load()
    p64, p32 = ctypes.c_double(0.), ctypes.c_double(0.)
    check(lib.canoe_measure_fma_peak(0, ctypes.byref(p64)), "fp64")
    check(lib.canoe_measure_fma_peak(1, ctypes.byref(p32)), "fp32")
    assert 5.0 < p64.value < 200.0, p64.value
    assert p32.value > p64.value, (p32.value, p64.value)
