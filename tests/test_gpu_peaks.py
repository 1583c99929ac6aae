"""Same-run peak microbenchmarks through the C ABI (pmg_measure_peaks): the copy bandwidth and
the FP64 / FP32 FMA rates must be positive and of the B200's order (HBM3e copy in the TB/s,
FMA rates in the tens of TFLOP/s, FP32 above FP64), and sizes outside the documented range
are refused."""
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu


def test_measure_peaks_plausible():
    p = pmg.measure_peaks(0, 512 << 20)
    assert p["copy_bytes"] == 512 << 20
    assert p["sm_count"] == torch.cuda.get_device_properties(0).multi_processor_count
    assert 1000.0 < p["copy_gbs"] < 20000.0
    assert 1.0 < p["fp64_fma_tflops"] < 200.0
    assert 1.0 < p["fp32_fma_tflops"] < 400.0
    assert p["fp32_fma_tflops"] > p["fp64_fma_tflops"]


@pytest.mark.parametrize("nbytes", [1 << 20, 17 << 30])
def test_measure_peaks_rejects_sizes(nbytes):
    with pytest.raises(pmg.PmgError) as e:
        pmg.measure_peaks(0, nbytes)
    assert e.value.status == -1  # PMG_EINVAL
