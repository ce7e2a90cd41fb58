"""The library's peak microbenchmarks (the roofline denominators) return plausible B200 figures."""
import pytest

from ggbtddft_b200 import engine

pytestmark = pytest.mark.gpu


def test_measured_peaks_are_plausible():
    p = engine.measure_peaks()
    # B200: FP64 ~37-40 TFLOP/s on both the FMA and the mma.sync paths, int8 ~4.5 POP/s dense
    assert 10.0 < p["fp64_fma_tflops"] < 80.0, p
    assert 5.0 < p["fp64_mma_tflops"] < 160.0, p
    assert p["fp64_tflops"] == max(p["fp64_fma_tflops"], p["fp64_mma_tflops"])
    assert 1000.0 < p["int8_tops"] < 9000.0, p
    print(p)
