"""pmg_vector_dot_noalloc through the C ABI: the allocation-free dot product agrees with
pmg_vector_dot on two calls in a row and rejects inputs beyond its fixed scratch.

The entry point exists for callers that cannot allocate device memory where they need a
reduction (a caching allocator owns their device budget, or the synchronisation of
cudaMalloc/cudaFree is not acceptable); its scratch is a fixed array in the library.  This
file is collected last so that a failure here does not hide any other test."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu

MAX_N = 4096 * 65536


def noalloc_fn():
    fn = pmg.lib().pmg_vector_dot_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int32
    return fn


def dot_noalloc(a, b, out):
    dt = pmg.F64 if a.dtype == torch.float64 else pmg.F32
    stream = torch.cuda.current_stream().cuda_stream
    st = noalloc_fn()(a.data_ptr(), b.data_ptr(), dt, a.numel(), out.data_ptr(), stream)
    assert st == 0, pmg.last_error()
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n", [1, 1000, 65536, 65537, 5_000_001])
def test_noalloc_dot_matches_allocating_dot_twice(dtype, n):
    g = torch.Generator(device="cuda").manual_seed(n + 3)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    results = []
    for call in range(2):  # the second call runs over the first call's leftover scratch
        a = torch.rand(n, generator=g, device="cuda", dtype=torch.float64).to(dtype) - 0.5
        b = torch.rand(n, generator=g, device="cuda", dtype=torch.float64).to(dtype)
        ref = pmg.vector_dot(a, b)
        got = dot_noalloc(a, b, out)
        tol = 1e-13 * max(1.0, np.log2(n)) * float(torch.dot(a.double().abs(), b.double().abs()))
        assert abs(got - ref) <= tol, (call, got, ref)
        results.append(got)
    assert results[0] != results[1]


def test_noalloc_dot_accepts_the_maximum_size():
    """n = 268,435,456 FP32 entries (two 1 GiB vectors): the largest accepted input, spread
    over more partial sums than the finishing block has threads."""
    g = torch.Generator(device="cuda").manual_seed(11)
    a = torch.rand(MAX_N, generator=g, device="cuda", dtype=torch.float32) - 0.5
    b = torch.rand(MAX_N, generator=g, device="cuda", dtype=torch.float32)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ref = pmg.vector_dot(a, b)
    got = dot_noalloc(a, b, out)
    assert abs(got - ref) <= 1e-13 * np.log2(MAX_N) * float(torch.dot(a.double().abs(), b.double().abs()))
    del a, b
    torch.cuda.empty_cache()


def test_noalloc_dot_rejects_oversized_input():
    a = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = noalloc_fn()(a.data_ptr(), a.data_ptr(), pmg.F64, MAX_N + 1, out.data_ptr(), None)
    assert st == -1
    assert "exceeds" in pmg.last_error()


def test_noalloc_dot_empty_input_writes_zero():
    a = torch.zeros(1, dtype=torch.float32, device="cuda")
    out = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    assert noalloc_fn()(a.data_ptr(), a.data_ptr(), pmg.F32, 0, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert float(out.item()) == 0.0
