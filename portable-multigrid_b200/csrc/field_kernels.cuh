// Slab kernels of the adjoint path: the FE mass matrix, its diagonal, and the density of the
// Laplace form at every quadrature point.  None of them exists in the reference; they use the
// layouts and the warp/slab scheme of the Laplace kernels (laplace_kernels.cuh): a warp owns
// CPW = floor(32/N) consecutive cells, lane s of a cell holds the Y-slab y = s while gathering
// and scattering and the Z-slab z = s while working at the quadrature points, with one
// warp-local exchange through shared memory per switch.
//
//   mass:    v = Sz Sy Sx u at the Gauss points, times |det J| w_q, back by the transposes.
//   qp form: grad_ref u and grad_ref v at the Gauss points as in the Laplace kernel's first
//            half (w = Sz Sx u, wz = SDz Sx u, wx = Sz SDx u, then Sy / SDy), and
//            e_q = alpha * grad u^T G_q grad v, written lexicographically per cell.
#pragma once

#include "laplace_kernels.cuh"

namespace pmg {
namespace kern {

// MG 1: affine cell without a weight field, |det J| = geo[cell][6];
// MG 0: per-point weights |det J| w_q (times a coefficient) in wts = [group][N^2][LANES]
// (row-major point index y*N + x, lane = e*N + z).
template <int N, typename T, int MG>
__global__ void __launch_bounds__(128, 1) mass_slab_kernel(const __grid_constant__ Tab<N, T> tab,
                                                        const T *__restrict__ src, T *__restrict__ dst,
                                                        const uint32_t *__restrict__ idx,
                                                        const T *__restrict__ geo,
                                                        const T *__restrict__ wts, int64_t n_groups) {
  using Lo = Layout<N>;
  constexpr int CPW = Lo::CPW, LANES = Lo::LANES, N2 = Lo::N2;
  constexpr int CS = Stride<N>::CELL;
  constexpr unsigned MASK = Lo::MASK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= LANES) return;
  const int e = lane / N;
  const int s = lane - e * N;
  T *buf = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (CPW * CS) + e * CS;
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const uint64_t pol_first = policy_evict_first(), pol_last = policy_evict_last();
  // fully unrolled except FP64 degree 6, where the unrolled form exceeds the register file
  constexpr int UNR = (sizeof(T) == 8 && N >= 7) ? 1 : N;
  T wr = tab.W[0];
#pragma unroll
  for (int r = 1; r < N; ++r)
    if (s == r) wr = tab.W[r];

  for (int64_t g = warp0; g < n_groups; g += nwarps) {
    const uint32_t *ig = idx + g * (N2 * LANES) + lane;
    // Y-slab y = s: gather, x and z interpolation -> buf (z, y = s, x)
    {
      T u[N][N];
#pragma unroll
      for (int k = 0; k < N; ++k)
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const uint32_t id = ld_stream(ig + (k * N + i) * LANES, pol_first);
          u[k][i] = (id != kInvalidIdx) ? ld_keep(src + id, pol_last) : T(0);
        }
#pragma unroll UNR
      for (int p = 0; p < N; ++p) {
        T t[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
          T a = T(0);
#pragma unroll
          for (int i = 0; i < N; ++i) a = fma(tab.S[i * N + p], u[k][i], a);
          t[k] = a;
        }
#pragma unroll
        for (int r = 0; r < N; ++r) {
          T w = T(0);
#pragma unroll
          for (int k = 0; k < N; ++k) w = fma(tab.S[k * N + r], t[k], w);
          buf[(r * N + s) * N + p] = w;
        }
      }
    }
    __syncwarp(MASK);
    // Z-slab z = s: y interpolation, weights, and the transposed x and y contractions
    {
      const T vol = MG == 1 ? __ldg(geo + (g * CPW + e) * 8 + 6) * wr : T(1);
      T a[N][N];
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i) a[j][i] = T(0);
#pragma unroll UNR
      for (int p = 0; p < N; ++p) {
        T Wc[N];
#pragma unroll
        for (int j = 0; j < N; ++j) Wc[j] = buf[(s * N + j) * N + p];
        T f[N];
#pragma unroll
        for (int q = 0; q < N; ++q) {
          T v = T(0);
#pragma unroll
          for (int j = 0; j < N; ++j) v = fma(tab.S[j * N + q], Wc[j], v);
          const T wq = MG == 1 ? vol * tab.W[q] * tab.W[p]
                               : ld_stream(wts + g * (N2 * LANES) + (q * N + p) * LANES + lane, pol_first);
          f[q] = wq * v;
        }
#pragma unroll
        for (int j = 0; j < N; ++j) {
          T y = T(0);
#pragma unroll
          for (int q = 0; q < N; ++q) y = fma(tab.S[j * N + q], f[q], y);
#pragma unroll
          for (int i = 0; i < N; ++i) a[j][i] = fma(tab.S[i * N + p], y, a[j][i]);
        }
      }
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i) buf[(s * N + j) * N + i] = a[j][i];
    }
    __syncwarp(MASK);
    // Y-slab y = s: transposed z contraction and scatter
#pragma unroll UNR
    for (int i = 0; i < N; ++i) {
      T A[N];
#pragma unroll
      for (int r = 0; r < N; ++r) A[r] = buf[(r * N + s) * N + i];
#pragma unroll
      for (int k = 0; k < N; ++k) {
        T v = T(0);
#pragma unroll
        for (int r = 0; r < N; ++r) v = fma(tab.S[k * N + r], A[r], v);
        const uint32_t id = ld_stream(ig + (k * N + i) * LANES, pol_first);
        if (id != kInvalidIdx) red_keep(dst + id, v, pol_last);
      }
    }
    __syncwarp(MASK);
  }
}

// diag(M)(i,j,k) = sum_{p,q,r} S2[i,p] S2[j,q] S2[k,r] w(p,q,r), S2 = S*S elementwise.
template <int N, typename T, int MG>
__global__ void __launch_bounds__(128) mass_diag_slab_kernel(const __grid_constant__ Tab2<N, T> tab,
                                                             T *__restrict__ diag,
                                                             const uint32_t *__restrict__ idx,
                                                             const T *__restrict__ geo,
                                                             const T *__restrict__ wts, int64_t n_groups) {
  using Lo = Layout<N>;
  constexpr int CPW = Lo::CPW, LANES = Lo::LANES, N2 = Lo::N2;
  constexpr int CS = Stride<N>::CELL;
  constexpr unsigned MASK = Lo::MASK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= LANES) return;
  const int e = lane / N;
  const int s = lane - e * N;
  T *buf = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (CPW * CS) + e * CS;
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  T wr = tab.W[0];
#pragma unroll
  for (int r = 1; r < N; ++r)
    if (s == r) wr = tab.W[r];
  for (int64_t g = warp0; g < n_groups; g += nwarps) {
    const T vol = MG == 1 ? __ldg(geo + (g * CPW + e) * 8 + 6) * wr : T(1);
    T w[N][N]; // [q][p] on the Z-slab z = s
#pragma unroll
    for (int q = 0; q < N; ++q)
#pragma unroll
      for (int p = 0; p < N; ++p)
        w[q][p] = MG == 1 ? vol * tab.W[q] * tab.W[p] : __ldg(wts + g * (N2 * LANES) + (q * N + p) * LANES + lane);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      T x[N];
#pragma unroll
      for (int q = 0; q < N; ++q) {
        T a = T(0);
#pragma unroll
        for (int p = 0; p < N; ++p) a = fma(tab.S2[i * N + p], w[q][p], a);
        x[q] = a;
      }
#pragma unroll
      for (int j = 0; j < N; ++j) {
        T b = T(0);
#pragma unroll
        for (int q = 0; q < N; ++q) b = fma(tab.S2[j * N + q], x[q], b);
        buf[(s * N + j) * N + i] = b;
      }
    }
    __syncwarp(MASK);
    const uint32_t *ig = idx + g * (N2 * LANES) + lane;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        T v = T(0);
#pragma unroll
        for (int r = 0; r < N; ++r) v = fma(tab.S2[k * N + r], buf[(r * N + s) * N + i], v);
        const uint32_t id = __ldg(ig + (k * N + i) * LANES);
        if (id != kInvalidIdx) atomic_add(diag + id, v);
      }
    __syncwarp(MASK);
  }
}

// e_q = alpha * grad_ref(u)^T G_q grad_ref(v) at every Gauss point, written as
// out[cell][(z*N + y)*N + x] (FP64).  G_q is the operator's stored geometry (GEOM as in
// vmult_slab_kernel: 0 full, 1 affine, 2 affine times the per-point coefficient), so the
// coefficient is included: e summed over the points of all cells is a(u, v).
// Shared memory per warp: six exchange buffers (w, wz, wx of u and of v).
template <int N, typename T, int GEOM>
__global__ void __launch_bounds__(64, 1) qp_form_slab_kernel(const __grid_constant__ Tab<N, T> tab,
                                                          const T *__restrict__ u, const T *__restrict__ v,
                                                          double *__restrict__ out,
                                                          const uint32_t *__restrict__ idx,
                                                          const T *__restrict__ geo,
                                                          const T *__restrict__ coef, int64_t n_groups,
                                                          int64_t n_cells, double alpha) {
  using Lo = Layout<N>;
  constexpr int CPW = Lo::CPW, LANES = Lo::LANES, N2 = Lo::N2, N3 = Lo::N3;
  constexpr int CS = Stride<N>::CELL;
  constexpr unsigned MASK = Lo::MASK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= LANES) return;
  const int e = lane / N;
  const int s = lane - e * N;
  constexpr int UNR = (sizeof(T) == 8 && N >= 6) ? 1 : N;
  T *wbase = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (6 * CPW * CS);
  T *const B0 = wbase + e * CS; // buffer b of this cell: B0 + b * CPW * CS
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const uint64_t pol_first = policy_evict_first(), pol_last = policy_evict_last();
  T wr = tab.W[0];
#pragma unroll
  for (int r = 1; r < N; ++r)
    if (s == r) wr = tab.W[r];

  for (int64_t g = warp0; g < n_groups; g += nwarps) {
    const uint32_t *ig = idx + g * (N2 * LANES) + lane;
    // Y-slab y = s, for u (buffers 0..2) and v (buffers 3..5)
#pragma unroll 1
    for (int vec = 0; vec < 2; ++vec) {
      const T *src = vec == 0 ? u : v;
      T *bW = B0 + (3 * vec) * (CPW * CS), *bZ = bW + CPW * CS, *bX = bZ + CPW * CS;
      T x[N][N];
#pragma unroll
      for (int k = 0; k < N; ++k)
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const uint32_t id = ld_stream(ig + (k * N + i) * LANES, pol_first);
          x[k][i] = (id != kInvalidIdx) ? ld_keep(src + id, pol_last) : T(0);
        }
#pragma unroll UNR
      for (int p = 0; p < N; ++p) {
        T t[N], tx[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
          T a = T(0), b = T(0);
#pragma unroll
          for (int i = 0; i < N; ++i) {
            a = fma(tab.S[i * N + p], x[k][i], a);
            b = fma(tab.SD[i * N + p], x[k][i], b);
          }
          t[k] = a;
          tx[k] = b;
        }
#pragma unroll
        for (int r = 0; r < N; ++r) {
          T w = T(0), wz = T(0), wx = T(0);
#pragma unroll
          for (int k = 0; k < N; ++k) {
            w = fma(tab.S[k * N + r], t[k], w);
            wz = fma(tab.SD[k * N + r], t[k], wz);
            wx = fma(tab.S[k * N + r], tx[k], wx);
          }
          const int o = (r * N + s) * N + p;
          bW[o] = w;
          bZ[o] = wz;
          bX[o] = wx;
        }
      }
    }
    __syncwarp(MASK);
    // Z-slab z = s: gradients at the points (., ., s), the form, into buffer 0 in place
#pragma unroll 1
    for (int p = 0; p < N; ++p) {
      T c[6][N];
#pragma unroll
      for (int b = 0; b < 6; ++b)
#pragma unroll
        for (int j = 0; j < N; ++j) c[b][j] = B0[b * (CPW * CS) + (s * N + j) * N + p];
#pragma unroll
      for (int q = 0; q < N; ++q) {
        T du[3] = {T(0), T(0), T(0)}, dv[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int j = 0; j < N; ++j) {
          du[0] = fma(tab.S[j * N + q], c[2][j], du[0]);
          du[1] = fma(tab.SD[j * N + q], c[0][j], du[1]);
          du[2] = fma(tab.S[j * N + q], c[1][j], du[2]);
          dv[0] = fma(tab.S[j * N + q], c[5][j], dv[0]);
          dv[1] = fma(tab.SD[j * N + q], c[3][j], dv[1]);
          dv[2] = fma(tab.S[j * N + q], c[4][j], dv[2]);
        }
        T gc[6];
        load_g6<N, T, GEOM, false>(geo, nullptr, coef, tab, g, lane, e, q, p, wr, pol_first, gc);
        const T g0 = gc[0] * dv[0] + gc[1] * dv[1] + gc[2] * dv[2];
        const T g1 = gc[1] * dv[0] + gc[3] * dv[1] + gc[4] * dv[2];
        const T g2 = gc[2] * dv[0] + gc[4] * dv[1] + gc[5] * dv[2];
        B0[(s * N + q) * N + p] = du[0] * g0 + du[1] * g1 + du[2] * g2;
      }
    }
    __syncwarp(MASK);
    // the group's cells are consecutive: one contiguous, coalesced run of CPW*N^3 values
    const int64_t c0 = g * CPW;
    for (int t = lane; t < CPW * N3; t += LANES) {
      const int ec = t / N3, r = t - ec * N3;
      if (c0 + ec < n_cells) out[c0 * N3 + t] = alpha * double(wbase[ec * CS + r]);
    }
    __syncwarp(MASK);
  }
}

} // namespace kern
} // namespace pmg
