// Same-run peak microbenchmarks: a STREAM-style device copy and FP64 / FP32 FMA throughput.
//
// The roofline fractions of the cell kernels are quoted against peaks; these kernels measure
// them on the GPU and at the clocks of the run that quotes them.  No counterpart in the
// reference, which times with deal.II Timer and reports no roofline.
//  * copy: dst = src over two buffers of `copy_bytes` (larger than L2), 16-byte vector
//    loads/stores, grid-stride; GB/s counts the bytes read plus the bytes written.
//  * FMA: every thread runs kChains independent chains a = fma(a, b, c) for `iters`
//    iterations (no memory traffic inside the loop); TFLOP/s counts 2 flops per FMA.
#include <algorithm>

#include "pmg_internal.hpp"

namespace pmg {
namespace {

constexpr int kThreads = 256;
constexpr int kChains = 8;

__global__ void __launch_bounds__(kThreads) copy16_kernel(const int4 *__restrict__ src, int4 *__restrict__ dst,
                                                          int64_t n) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

template <typename T>
__global__ void __launch_bounds__(kThreads) fma_kernel(T *__restrict__ out, T b, T c, int iters) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = T(threadIdx.x + k) * T(1e-3);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  T s = T(0);
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  out[int64_t(blockIdx.x) * blockDim.x + threadIdx.x] = s; // keeps the chains live
}

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  EventPair() {
    PMG_CUDA(cudaEventCreate(&a));
    PMG_CUDA(cudaEventCreate(&b));
  }
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  float ms() {
    float t = 0.f;
    PMG_CUDA(cudaEventSynchronize(b));
    PMG_CUDA(cudaEventElapsedTime(&t, a, b));
    return t;
  }
};

template <typename T> double fma_tflops(int sms, cudaStream_t s) {
  const int grid = sms * 8, iters = 1 << 15, reps = 5;
  DeviceBuffer out(size_t(grid) * kThreads * sizeof(T));
  const T b = T(0.999999), c = T(1e-6);
  fma_kernel<T><<<grid, kThreads, 0, s>>>(static_cast<T *>(out.get()), b, c, iters); // warm-up
  PMG_LAUNCH_CHECK();
  EventPair ev;
  PMG_CUDA(cudaEventRecord(ev.a, s));
  for (int r = 0; r < reps; ++r)
    fma_kernel<T><<<grid, kThreads, 0, s>>>(static_cast<T *>(out.get()), b, c, iters);
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaEventRecord(ev.b, s));
  const double flops = 2.0 * double(grid) * kThreads * kChains * double(iters) * reps;
  return flops / (ev.ms() * 1e-3) / 1e12;
}

} // namespace

void measure_peaks(int device, int64_t copy_bytes, pmg_peaks *out) {
  PMG_REQUIRE(out != nullptr, "null output");
  PMG_REQUIRE(copy_bytes >= (int64_t(256) << 20), "copy_bytes must be at least 256 MiB (larger than L2)");
  PMG_REQUIRE(copy_bytes <= (int64_t(16) << 30), "copy_bytes must be at most 16 GiB");
  PMG_CUDA(cudaSetDevice(device));
  int sms = 0;
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  cudaStream_t s = nullptr;
  PMG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{s};

  const int64_t n16 = copy_bytes / 16;
  {
    DeviceBuffer a(size_t(n16) * 16), b(size_t(n16) * 16);
    PMG_CUDA(cudaMemsetAsync(a.get(), 0, size_t(n16) * 16, s));
    const int grid = sms * 4;
    const int reps = 10;
    auto launch = [&] {
      copy16_kernel<<<grid, kThreads, 0, s>>>(static_cast<const int4 *>(a.get()), static_cast<int4 *>(b.get()), n16);
    };
    launch();
    launch();
    PMG_LAUNCH_CHECK();
    EventPair ev;
    PMG_CUDA(cudaEventRecord(ev.a, s));
    for (int r = 0; r < reps; ++r) launch();
    PMG_LAUNCH_CHECK();
    PMG_CUDA(cudaEventRecord(ev.b, s));
    out->copy_gbs = 2.0 * double(n16) * 16.0 * reps / (ev.ms() * 1e-3) / 1e9;
  }
  out->fp64_fma_tflops = fma_tflops<double>(sms, s);
  out->fp32_fma_tflops = fma_tflops<float>(sms, s);
  out->copy_bytes = n16 * 16;
  out->sm_count = sms;
  PMG_CUDA(cudaStreamSynchronize(s));
}

} // namespace pmg
