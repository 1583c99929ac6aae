"""Vector kernels through the C ABI: the FP64-accumulated dot product and the precision
conversion used on entry to and exit from the FP32 V-cycle, against torch fp64 references."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 255, 256, 257, 100_003, 3_000_000])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_vector_dot(n, dtype):
    g = torch.Generator(device="cuda").manual_seed(n)
    a = torch.rand(n, generator=g, device="cuda", dtype=torch.float64).to(dtype)
    b = torch.rand(n, generator=g, device="cuda", dtype=torch.float64).to(dtype)
    ref = float(torch.dot(a.double(), b.double()))
    got = pmg.vector_dot(a, b)
    assert abs(got - ref) <= 1e-13 * abs(ref) * max(1.0, np.log2(n))
    assert pmg.vector_dot(a, b) == got  # deterministic


def test_vector_copy_converts():
    x = torch.rand(12345, device="cuda", dtype=torch.float64)
    y = torch.empty(12345, device="cuda", dtype=torch.float32)
    pmg.vector_copy(y, x)
    z = torch.empty_like(x)
    pmg.vector_copy(z, y)
    torch.cuda.synchronize()
    assert torch.equal(y, x.float()) and torch.equal(z, y.double())


def test_vector_dot_rejects_bad_dtype():
    a = torch.zeros(4, device="cuda")
    L = pmg.lib()
    import ctypes
    r = ctypes.c_double()
    assert L.pmg_vector_dot(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(a.data_ptr()), 7, 4,
                            ctypes.byref(r), None) == -1
