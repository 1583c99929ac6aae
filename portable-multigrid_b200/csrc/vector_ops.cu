// Vector kernels of the Chebyshev smoother, the V-cycle and CG: fused updates (one pass
// over HBM per update instead of deal.II's chain of sadd/add/DiagonalMatrix::vmult calls)
// and deterministic dot products accumulated in FP64 whatever the vector type.
#include <mutex>

#include "pmg_internal.hpp"
#include "vector_ops.hpp"

namespace pmg {
namespace vec {
namespace {

constexpr int kBlock = 256;
constexpr int kMaxPartials = 1024;

// SM count of the current device (cached per device)
int current_sms() {
  static std::mutex mu;
  static int sms[64] = {0};
  int dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  int &n = sms[dev & 63];
  if (n == 0) PMG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

// grid of an elementwise grid-stride kernel: eight 256-thread blocks per SM at most
inline int grid_for(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kBlock - 1) / kBlock, 8 * (int64_t)current_sms()));
}

#define GRID_STRIDE(i, n)                                                                     \
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n);                  \
       i += (int64_t)gridDim.x * blockDim.x)

template <typename T> __global__ void fill_mod11_k(T *x, int64_t n, double mean) {
  GRID_STRIDE(i, n) x[i] = (T)((double)(i % 11) - mean);
}

template <typename TD, typename TS> __global__ void convert_k(TD *d, const TS *s, int64_t n) {
  GRID_STRIDE(i, n) d[i] = (TD)s[i];
}

template <typename T>
__global__ void cheb_init_k(T *dst, T *xo, const T *src, const T *invd, T scale, int64_t n) {
  GRID_STRIDE(i, n) {
    dst[i] = scale * invd[i] * src[i];
    if (xo) xo[i] = T(0);
  }
}

template <typename T>
__global__ void cheb_first_step_k(T *dst, T *xo, const T *src, const T *Ax, const T *invd, T scale,
                                  int64_t n) {
  GRID_STRIDE(i, n) {
    const T x = dst[i];
    xo[i] = x;
    dst[i] = x + scale * invd[i] * (src[i] - Ax[i]);
  }
}

// the same first step into another vector: x0 is kept as the previous iterate
template <typename T>
__global__ void cheb_first_step_into_k(T *out, const T *x0, const T *src, const T *Ax, const T *invd,
                                       T scale, int64_t n) {
  GRID_STRIDE(i, n) {
    const T x = x0[i];
    out[i] = x + scale * invd[i] * (src[i] - Ax[i]);
  }
}

// the update written over the previous iterate (out == prev allowed; prev == nullptr: zero)
template <typename T>
__global__ void cheb_update_into_k(T *out, const T *cur, const T *prev, const T *src, const T *Ax,
                                   const T *invd, T f1, T f2, int64_t n) {
  GRID_STRIDE(i, n) {
    const T x = cur[i];
    const T xo = prev ? prev[i] : T(0);
    out[i] = x + f1 * (x - xo) + f2 * invd[i] * (src[i] - Ax[i]);
  }
}

template <typename T> __global__ void residual_k(T *t, const T *def, int64_t n) {
  GRID_STRIDE(i, n) t[i] = def[i] - t[i];
}

template <typename T> __global__ void jacobi_k(T *z, const T *invd, const T *r, int64_t n) {
  GRID_STRIDE(i, n) z[i] = invd[i] * r[i];
}

template <typename T> __global__ void xpay_k(T *p, const T *z, T beta, int64_t n) {
  GRID_STRIDE(i, n) p[i] = z[i] + beta * p[i];
}

template <typename T> __global__ void axpy_k(T *y, const T *x, T alpha, int64_t n) {
  GRID_STRIDE(i, n) y[i] += alpha * x[i];
}

// block partial sums of a*b (or of the CG update's new r*r), FP64 accumulation
template <typename T>
__device__ __forceinline__ void block_reduce_store(double v, double *partials) {
  __shared__ double red[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = (threadIdx.x < kBlock / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = w;
  }
}

template <typename T>
__global__ void dot_partial_k(const T *a, const T *b, int64_t n, double *partials) {
  double v = 0.0;
  GRID_STRIDE(i, n) v += (double)a[i] * (double)b[i];
  block_reduce_store<T>(v, partials);
}

template <typename T>
__global__ void cg_update_k(T *x, T *r, const T *p, const T *v, T alpha, int64_t n, double *partials) {
  double acc = 0.0;
  GRID_STRIDE(i, n) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * v[i];
    r[i] = ri;
    acc += (double)ri * (double)ri;
  }
  block_reduce_store<T>(acc, partials);
}

// r = b - Ax and partial sums of r*r
template <typename T>
__global__ void residual_dot_k(T *r, const T *b, const T *Ax, int64_t n, double *partials) {
  double acc = 0.0;
  GRID_STRIDE(i, n) {
    const T ri = b[i] - Ax[i];
    r[i] = ri;
    acc += (double)ri * (double)ri;
  }
  block_reduce_store<T>(acc, partials);
}

// z = invd * r and partial sums of r*z
template <typename T>
__global__ void jacobi_dot_k(T *z, const T *invd, const T *r, int64_t n, double *partials) {
  double acc = 0.0;
  GRID_STRIDE(i, n) {
    const T zi = invd[i] * r[i];
    z[i] = zi;
    acc += (double)r[i] * (double)zi;
  }
  block_reduce_store<T>(acc, partials);
}

__global__ void finalize_k(const double *partials, int n_partials, double *out) {
  // fixed-order tree over at most kMaxPartials values: deterministic
  __shared__ double s[kMaxPartials];
  for (int i = threadIdx.x; i < kMaxPartials; i += blockDim.x) s[i] = (i < n_partials) ? partials[i] : 0.0;
  __syncthreads();
  for (int w = kMaxPartials / 2; w > 0; w >>= 1) {
    for (int i = threadIdx.x; i < w; i += blockDim.x) s[i] += s[i + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

struct Workspace {
  DeviceBuffer partials;
  DeviceBuffer results; // 64 doubles
  double *host = nullptr; // pinned, 64 doubles
};

Workspace &workspace() {
  static std::mutex mu;
  static Workspace ws[64];
  int dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  Workspace &w = ws[dev & 63];
  if (!w.partials.get()) {
    w.partials.allocate(sizeof(double) * kMaxPartials * 4);
    w.results.allocate(sizeof(double) * 64);
    PMG_CUDA(cudaMallocHost(&w.host, sizeof(double) * 64));
  }
  return w;
}

inline int reduce_grid(int64_t n) { return (int)std::min<int64_t>(kMaxPartials, std::max<int64_t>(1, (n + kBlock - 1) / kBlock)); }

double finish(Workspace &w, int grid, int slot, cudaStream_t s) {
  finalize_k<<<1, 1024, 0, s>>>(w.partials.as<double>(), grid, w.results.as<double>() + slot);
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaMemcpyAsync(w.host + slot, w.results.as<double>() + slot, sizeof(double),
                           cudaMemcpyDeviceToHost, s));
  PMG_CUDA(cudaStreamSynchronize(s));
  return w.host[slot];
}

} // namespace

#define DISPATCH(dtype, ...)                                                                  \
  do {                                                                                        \
    if ((dtype) == PMG_F64) {                                                                 \
      using T = double;                                                                       \
      __VA_ARGS__;                                                                            \
    } else {                                                                                  \
      using T = float;                                                                        \
      __VA_ARGS__;                                                                            \
    }                                                                                         \
  } while (0)

void fill_mod11(void *x, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  // mean of (i mod 11) over i < n, exactly
  const int64_t full = n / 11, rem = n % 11;
  const double sum = double(full) * 55.0 + double(rem * (rem - 1) / 2);
  const double mean = n > 0 ? sum / double(n) : 0.0;
  DISPATCH(dtype, fill_mod11_k<T><<<grid_for(n), kBlock, 0, s>>>(static_cast<T *>(x), n, mean));
  PMG_LAUNCH_CHECK();
}

void convert(void *dst, int dt_dst, const void *src, int dt_src, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  if (dt_dst == dt_src) {
    PMG_CUDA(cudaMemcpyAsync(dst, src, dtype_size(dt_dst) * n, cudaMemcpyDeviceToDevice, s));
    return;
  }
  if (dt_dst == PMG_F32)
    convert_k<float, double><<<grid_for(n), kBlock, 0, s>>>(static_cast<float *>(dst), static_cast<const double *>(src), n);
  else
    convert_k<double, float><<<grid_for(n), kBlock, 0, s>>>(static_cast<double *>(dst), static_cast<const float *>(src), n);
  PMG_LAUNCH_CHECK();
}

void cheb_init(void *dst, void *xo, const void *src, const void *invd, double scale, int dtype,
               int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, cheb_init_k<T><<<grid_for(n), kBlock, 0, s>>>(static_cast<T *>(dst), static_cast<T *>(xo),
                                                                 static_cast<const T *>(src), static_cast<const T *>(invd), (T)scale, n));
  PMG_LAUNCH_CHECK();
}

void cheb_first_step(void *dst, void *xo, const void *src, const void *Ax, const void *invd,
                     double scale, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, cheb_first_step_k<T><<<grid_for(n), kBlock, 0, s>>>(
                      static_cast<T *>(dst), static_cast<T *>(xo), static_cast<const T *>(src),
                      static_cast<const T *>(Ax), static_cast<const T *>(invd), (T)scale, n));
  PMG_LAUNCH_CHECK();
}

void cheb_first_step_into(void *out, const void *x0, const void *src, const void *Ax, const void *invd,
                          double scale, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, cheb_first_step_into_k<T><<<grid_for(n), kBlock, 0, s>>>(
                      static_cast<T *>(out), static_cast<const T *>(x0), static_cast<const T *>(src),
                      static_cast<const T *>(Ax), static_cast<const T *>(invd), (T)scale, n));
  PMG_LAUNCH_CHECK();
}

void cheb_update_into(void *out, const void *cur, const void *prev, const void *src, const void *Ax,
                      const void *invd, double f1, double f2, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, cheb_update_into_k<T><<<grid_for(n), kBlock, 0, s>>>(
                      static_cast<T *>(out), static_cast<const T *>(cur), static_cast<const T *>(prev),
                      static_cast<const T *>(src), static_cast<const T *>(Ax), static_cast<const T *>(invd),
                      (T)f1, (T)f2, n));
  PMG_LAUNCH_CHECK();
}

void residual(void *t, const void *def, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, residual_k<T><<<grid_for(n), kBlock, 0, s>>>(static_cast<T *>(t), static_cast<const T *>(def), n));
  PMG_LAUNCH_CHECK();
}

void jacobi(void *z, const void *invd, const void *r, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, jacobi_k<T><<<grid_for(n), kBlock, 0, s>>>(static_cast<T *>(z), static_cast<const T *>(invd),
                                                              static_cast<const T *>(r), n));
  PMG_LAUNCH_CHECK();
}

void xpay(void *p, const void *z, double beta, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, xpay_k<T><<<grid_for(n), kBlock, 0, s>>>(static_cast<T *>(p), static_cast<const T *>(z), (T)beta, n));
  PMG_LAUNCH_CHECK();
}

void axpy(void *y, const void *x, double alpha, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_update", s);
  DISPATCH(dtype, axpy_k<T><<<grid_for(n), kBlock, 0, s>>>(static_cast<T *>(y), static_cast<const T *>(x), (T)alpha, n));
  PMG_LAUNCH_CHECK();
}

double dot(const void *a, const void *b, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_reduce", s);
  Workspace &w = workspace();
  const int grid = reduce_grid(n);
  DISPATCH(dtype, dot_partial_k<T><<<grid, kBlock, 0, s>>>(static_cast<const T *>(a), static_cast<const T *>(b), n,
                                                            w.partials.as<double>()));
  PMG_LAUNCH_CHECK();
  return finish(w, grid, 0, s);
}

double cg_update(void *x, void *r, const void *p, const void *v, double alpha, int dtype, int64_t n,
                 cudaStream_t s) {
  prof::Scope scope_("vector_reduce", s);
  Workspace &w = workspace();
  const int grid = reduce_grid(n);
  DISPATCH(dtype, cg_update_k<T><<<grid, kBlock, 0, s>>>(static_cast<T *>(x), static_cast<T *>(r),
                                                          static_cast<const T *>(p), static_cast<const T *>(v),
                                                          (T)alpha, n, w.partials.as<double>()));
  PMG_LAUNCH_CHECK();
  return finish(w, grid, 1, s);
}

double residual_dot(void *r, const void *b, const void *Ax, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_reduce", s);
  Workspace &w = workspace();
  const int grid = reduce_grid(n);
  DISPATCH(dtype, residual_dot_k<T><<<grid, kBlock, 0, s>>>(static_cast<T *>(r), static_cast<const T *>(b),
                                                             static_cast<const T *>(Ax), n, w.partials.as<double>()));
  PMG_LAUNCH_CHECK();
  return finish(w, grid, 3, s);
}

double jacobi_dot(void *z, const void *invd, const void *r, int dtype, int64_t n, cudaStream_t s) {
  prof::Scope scope_("vector_reduce", s);
  Workspace &w = workspace();
  const int grid = reduce_grid(n);
  DISPATCH(dtype, jacobi_dot_k<T><<<grid, kBlock, 0, s>>>(static_cast<T *>(z), static_cast<const T *>(invd),
                                                           static_cast<const T *>(r), n, w.partials.as<double>()));
  PMG_LAUNCH_CHECK();
  return finish(w, grid, 2, s);
}

} // namespace vec
} // namespace pmg
