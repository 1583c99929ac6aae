// pmg_vector_dot_noalloc: the dot product of pmg_vector_dot without any device allocation.
//
// Some callers cannot call cudaMalloc at the point where they need a reduction: code that
// runs under a fixed device-memory budget already reserved by its own allocator (a
// framework's caching allocator that owns the whole GPU, an embedded or real-time host that
// pre-allocates everything at start-up), or code that must not pay for the device-wide
// synchronisation cudaMalloc/cudaFree can imply.  For them this entry point keeps its
// scratch -- one FP64 partial sum per block -- in a file-scope __device__ array that every
// GPU loading the library holds until the process exits.
//
// Limits and rules:
//  * each block reduces one chunk of consecutive entries, a multiple of the block size
//    chosen from n so that about eight blocks per SM share the vector (at most kMaxBlocks
//    partial sums); n may be at most kMaxN = 268,435,456 entries, larger n is rejected with
//    PMG_EINVAL;
//  * for a given n and device the reduction order is fixed (deterministic), but it is not
//    pmg_vector_dot's order, so the two may differ in the last bits;
//  * the result is written to a caller-owned device double, ordered on the stream; the
//    host is not synchronised;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, that device current); make that first call
//    before any stream capture.  The address is kept per device ordinal for the life of the
//    process: it assumes the device's primary context is not reset (cudaDeviceReset) and
//    that the calls run in that primary context;
//  * every call shares the one array: calls whose kernels overlap on the GPU (different
//    streams without ordering) race and give wrong results;
//  * every block writes its partial before the final kernel reads exactly those partials,
//    so the array never needs clearing; it keeps the last call's partials.
#include <algorithm>
#include <mutex>

#include "pmg_internal.hpp"

namespace pmg {
namespace {

constexpr int kMaxBlocks = 4096; // partial sums held by the scratch array
constexpr int kThreads = 256;
constexpr int64_t kMaxN = int64_t(kMaxBlocks) * 256 * kThreads;

static __device__ __align__(256) double g_dot_partials[kMaxBlocks];

template <typename T>
__global__ void __launch_bounds__(kThreads) dot_chunk_kernel(const T *__restrict__ a,
                                                             const T *__restrict__ b, int64_t n,
                                                             int64_t chunk,
                                                             double *__restrict__ partials) {
  const int64_t base = int64_t(blockIdx.x) * chunk;
  const int64_t end = min(base + chunk, n);
  double v = 0.0;
  for (int64_t i = base + threadIdx.x; i < end; i += kThreads) v += (double)a[i] * (double)b[i];
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = (threadIdx.x < kThreads / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = w;
  }
}

// fixed-order tree over the n_blocks partials (deterministic)
__global__ void __launch_bounds__(1024) dot_finish_kernel(const double *__restrict__ partials,
                                                          int n_blocks, double *__restrict__ out) {
  __shared__ double s[1024];
  double v = 0.0;
  for (int i = threadIdx.x; i < n_blocks; i += 1024) v += partials[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// device address of g_dot_partials, looked up once per device with that device current
double *scratch_address(int device) {
  static std::mutex mu;
  static double *addr[64] = {nullptr};
  PMG_REQUIRE(device >= 0 && device < 64, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void *p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_dot_partials);
    if (rc != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      fail(PMG_ECUDA, std::string("cudaGetSymbolAddress of the dot scratch failed: ") +
                          cudaGetErrorString(rc));
    }
    addr[device] = static_cast<double *>(p);
  }
  return addr[device];
}

} // namespace

void vector_dot_noalloc(const void *a, const void *b, int dtype, int64_t n, double *result,
                        cudaStream_t s) {
  PMG_REQUIRE(a && b && result, "null pointer");
  PMG_REQUIRE(dtype == PMG_F64 || dtype == PMG_F32, "bad dtype");
  PMG_REQUIRE(n >= 0, "n must be >= 0");
  if (n > kMaxN)
    fail(PMG_EINVAL, "n = " + std::to_string(n) + " exceeds the no-allocation dot limit of " +
                         std::to_string(kMaxN) + " entries");
  int device = 0;
  PMG_CUDA(cudaGetDevice(&device));
  double *partials = scratch_address(device);
  int sms = 0;
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  // chunk: a multiple of the block size, about eight blocks per SM, at most kMaxBlocks blocks
  const int64_t target = std::min<int64_t>(kMaxBlocks, 8 * (int64_t)std::max(sms, 1));
  const int64_t per_block = (n + target - 1) / target;
  const int64_t chunk = std::max<int64_t>(kThreads, (per_block + kThreads - 1) / kThreads * kThreads);
  const int n_blocks = (int)((n + chunk - 1) / chunk);
  if (n_blocks > 0) {
    if (dtype == PMG_F64)
      dot_chunk_kernel<double><<<n_blocks, kThreads, 0, s>>>(static_cast<const double *>(a),
                                                             static_cast<const double *>(b), n, chunk, partials);
    else
      dot_chunk_kernel<float><<<n_blocks, kThreads, 0, s>>>(static_cast<const float *>(a),
                                                            static_cast<const float *>(b), n, chunk, partials);
    PMG_LAUNCH_CHECK();
  }
  dot_finish_kernel<<<1, 1024, 0, s>>>(partials, n_blocks, result);
  PMG_LAUNCH_CHECK();
}

} // namespace pmg
