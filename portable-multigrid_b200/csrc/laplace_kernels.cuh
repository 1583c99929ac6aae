// Sum-factorized cell kernels of the continuous Q_p Laplace operator for sm_100a.
//
// What they compute is the BK3 cell operator of the reference
// (include/kernels/bk3_kokkos_kernel.h:25-746): per cell gather the nodal values (Dirichlet
// entries read as 0), interpolate to the Gauss points, take collocation gradients, apply
// the symmetric geometry tensor G, integrate against the gradients and scatter-add.  How
// they compute it is laid out for the B200:
//
//  * A warp owns a group of CPW = floor(32/N) consecutive cells (N = p+1 nodes per
//    direction), N lanes per cell.  Lane s of a cell holds a whole slab of the cell in
//    registers: the plane y = s ("Y-slab") while gathering, contracting along x and z and
//    scattering, and the plane z = s ("Z-slab") while contracting along x and y and
//    applying G.  Contractions along the held plane never leave the registers; switching
//    slabs is one warp-local exchange through shared memory.  The operator is factored so
//    that only two such switches (two arrays each) are needed per cell:
//        Y-slab:  w = Sz Sx u,   wz = SDz Sx u                    (SD = S*D)
//        Z-slab:  uq = Sy w, dy = SDy w, dz = Sy wz, dx = Dx uq;   f = G grad u
//                 a = Sy^T SDx^T fx + SDy^T Sx^T fy,   c = Sy^T Sx^T fz
//        Y-slab:  out = Sz^T a + SDz^T c
//    No block-wide barrier is used; warps are independent.
//  * The index map and G are stored lane-contiguous per group ([group][point][lane]), so
//    every load of them is a fully coalesced warp access, and each warp bulk-prefetches the
//    next group's G into L2 (cp.async.bulk.prefetch.L2) while it computes the current one.
//  * Scatter with native FP64/FP32 atomic adds (red.global.add) into L2.
//  * The 1D tables are kernel parameters (constant bank), indexed at compile time.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pmg {
namespace kern {

constexpr uint32_t kInvalidIdx = 0xFFFFFFFFu;

template <int N, typename T> struct Tab {
  T S[N * N];  // S[i*N+q]  = phi_i(g_q)
  T SD[N * N]; // SD[i*N+q] = phi_i'(g_q)
  T D[N * N];  // D[n*N+q]  = l_n'(g_q) on the Gauss points
  T W[N];      // Gauss weights
};

// squared tables for the diagonal: S2 = S*S, SS = S*SD, D2 = SD*SD (elementwise)
template <int N, typename T> struct Tab2 {
  T S2[N * N];
  T SS[N * N];
  T D2[N * N];
  T W[N];
};

template <int N> struct Layout {
  static constexpr int CPW = 32 / N;
  static constexpr int LANES = CPW * N;
  static constexpr unsigned MASK = LANES == 32 ? 0xffffffffu : ((1u << LANES) - 1u);
  static constexpr int N2 = N * N;
  static constexpr int N3 = N * N * N;
};

__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }

// GEOM 0: full G per quadrature point, geo = [group][N^2 (q,p)][6][LANES]
// GEOM 1: affine, geo = [cell][8] (6 used) multiplied by the tensor Gauss weight
// GEOM 2: affine as 1, times coef = [group][N^2][LANES] per quadrature point
template <int N, typename T, int GEOM>
__global__ void __launch_bounds__(128) vmult_slab_kernel(const Tab<N, T> tab,
                                                         const T *__restrict__ src,
                                                         T *__restrict__ dst,
                                                         const uint32_t *__restrict__ idx,
                                                         const T *__restrict__ geo,
                                                         const T *__restrict__ coef,
                                                         int64_t n_groups) {
  using Lo = Layout<N>;
  constexpr int CPW = Lo::CPW, LANES = Lo::LANES, N2 = Lo::N2, N3 = Lo::N3;
  constexpr unsigned MASK = Lo::MASK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= LANES) return;
  const int e = lane / N;
  const int s = lane - e * N;
  T *bufA = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (2 * CPW * N3) + e * N3;
  T *bufB = bufA + CPW * N3;
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;

  for (int64_t g = warp0; g < n_groups; g += nwarps) {
    if (GEOM == 0 && lane == 0 && g + nwarps < n_groups)
      prefetch_l2(geo + (g + nwarps) * (N2 * 6 * LANES), N2 * 6 * LANES * sizeof(T));

    // ---- gather, Y-slab (y = s): u[k][i] = src at node (i, s, k) ----
    const uint32_t *ig = idx + g * (N2 * LANES) + lane;
    T t[N][N];
    {
      T u[N][N];
#pragma unroll
      for (int k = 0; k < N; ++k)
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const uint32_t id = __ldg(ig + (k * N + i) * LANES);
          u[k][i] = (id != kInvalidIdx) ? __ldg(src + id) : T(0);
        }
      // x: nodes -> Gauss points
#pragma unroll
      for (int k = 0; k < N; ++k)
#pragma unroll
        for (int p = 0; p < N; ++p) {
          T a = T(0);
#pragma unroll
          for (int i = 0; i < N; ++i) a = fma(tab.S[i * N + p], u[k][i], a);
          t[k][p] = a;
        }
    }
    // z: nodes -> Gauss values (w) and Gauss derivatives (wz), to shared (r, y=s, p)
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int p = 0; p < N; ++p) {
        T a = T(0), b = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          a = fma(tab.S[k * N + r], t[k][p], a);
          b = fma(tab.SD[k * N + r], t[k][p], b);
        }
        bufA[(r * N + s) * N + p] = a;
        bufB[(r * N + s) * N + p] = b;
      }
    __syncwarp(MASK);

    // ---- Z-slab (z = s) ----
    T fx[N][N], fy[N][N], fz[N][N]; // [q][p]
    {
      T W[N][N], WZ[N][N];
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int p = 0; p < N; ++p) {
          W[j][p] = bufA[(s * N + j) * N + p];
          WZ[j][p] = bufB[(s * N + j) * N + p];
        }
      T uq[N][N];
#pragma unroll
      for (int p = 0; p < N; ++p)
#pragma unroll
        for (int q = 0; q < N; ++q) {
          T a = T(0), b = T(0), c = T(0);
#pragma unroll
          for (int j = 0; j < N; ++j) {
            a = fma(tab.S[j * N + q], W[j][p], a);
            b = fma(tab.SD[j * N + q], W[j][p], b);
            c = fma(tab.S[j * N + q], WZ[j][p], c);
          }
          uq[q][p] = a;
          fy[q][p] = b; // dy
          fz[q][p] = c; // dz
        }
#pragma unroll
      for (int q = 0; q < N; ++q)
#pragma unroll
        for (int p = 0; p < N; ++p) {
          T a = T(0);
#pragma unroll
          for (int m = 0; m < N; ++m) a = fma(tab.D[m * N + p], uq[q][m], a);
          fx[q][p] = a; // dx
        }
    }
    // geometry: f = G grad u at the N^2 points of this slab
    if (GEOM == 0) {
      const T *gg = geo + g * (N2 * 6 * LANES) + lane;
#pragma unroll
      for (int q = 0; q < N; ++q)
#pragma unroll
        for (int p = 0; p < N; ++p) {
          const T *gp = gg + (q * N + p) * 6 * LANES;
          const T g0 = __ldg(gp), g1 = __ldg(gp + LANES), g2 = __ldg(gp + 2 * LANES),
                  g3 = __ldg(gp + 3 * LANES), g4 = __ldg(gp + 4 * LANES),
                  g5 = __ldg(gp + 5 * LANES);
          const T dx = fx[q][p], dy = fy[q][p], dz = fz[q][p];
          fx[q][p] = g0 * dx + g1 * dy + g2 * dz;
          fy[q][p] = g1 * dx + g3 * dy + g4 * dz;
          fz[q][p] = g2 * dx + g4 * dy + g5 * dz;
        }
    } else {
      const T *cg = geo + (g * CPW + e) * 8;
      const T c0 = __ldg(cg), c1 = __ldg(cg + 1), c2 = __ldg(cg + 2), c3 = __ldg(cg + 3),
              c4 = __ldg(cg + 4), c5 = __ldg(cg + 5);
      T wr = tab.W[0]; // Gauss weight of this slab's z coordinate
#pragma unroll
      for (int r = 1; r < N; ++r)
        if (s == r) wr = tab.W[r];
#pragma unroll
      for (int q = 0; q < N; ++q)
#pragma unroll
        for (int p = 0; p < N; ++p) {
          T w = wr * tab.W[q] * tab.W[p];
          if (GEOM == 2) w *= __ldg(coef + g * (N2 * LANES) + (q * N + p) * LANES + lane);
          const T dx = fx[q][p], dy = fy[q][p], dz = fz[q][p];
          fx[q][p] = w * (c0 * dx + c1 * dy + c2 * dz);
          fy[q][p] = w * (c1 * dx + c3 * dy + c4 * dz);
          fz[q][p] = w * (c2 * dx + c4 * dy + c5 * dz);
        }
    }
    // integrate: X1 = SDx^T fx, X2 = Sx^T fy, X3 = Sx^T fz  (in place, row by row)
#pragma unroll
    for (int q = 0; q < N; ++q) {
      T x1[N], x2[N], x3[N];
#pragma unroll
      for (int i = 0; i < N; ++i) {
        T a = T(0), b = T(0), c = T(0);
#pragma unroll
        for (int p = 0; p < N; ++p) {
          a = fma(tab.SD[i * N + p], fx[q][p], a);
          b = fma(tab.S[i * N + p], fy[q][p], b);
          c = fma(tab.S[i * N + p], fz[q][p], c);
        }
        x1[i] = a;
        x2[i] = b;
        x3[i] = c;
      }
#pragma unroll
      for (int i = 0; i < N; ++i) {
        fx[q][i] = x1[i];
        fy[q][i] = x2[i];
        fz[q][i] = x3[i];
      }
    }
    __syncwarp(MASK); // every lane has read the first exchange
    // a = Sy^T X1 + SDy^T X2, c = Sy^T X3, to shared (z=s, j, i)
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        T a = T(0), c = T(0);
#pragma unroll
        for (int q = 0; q < N; ++q) {
          a = fma(tab.S[j * N + q], fx[q][i], a);
          a = fma(tab.SD[j * N + q], fy[q][i], a);
          c = fma(tab.S[j * N + q], fz[q][i], c);
        }
        bufA[(s * N + j) * N + i] = a;
        bufB[(s * N + j) * N + i] = c;
      }
    __syncwarp(MASK);

    // ---- Y-slab (y = s): out = Sz^T a + SDz^T c, scatter ----
    {
      T A[N][N], Cc[N][N];
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int i = 0; i < N; ++i) {
          A[r][i] = bufA[(r * N + s) * N + i];
          Cc[r][i] = bufB[(r * N + s) * N + i];
        }
#pragma unroll
      for (int k = 0; k < N; ++k)
#pragma unroll
        for (int i = 0; i < N; ++i) {
          T a = T(0);
#pragma unroll
          for (int r = 0; r < N; ++r) {
            a = fma(tab.S[k * N + r], A[r][i], a);
            a = fma(tab.SD[k * N + r], Cc[r][i], a);
          }
          const uint32_t id = __ldg(ig + (k * N + i) * LANES);
          if (id != kInvalidIdx) atomic_add(dst + id, a);
        }
    }
    __syncwarp(MASK); // shared buffers are reused by the next group
  }
}

// Diagonal of the cell operator summed into diag (atomic), same layout and slab scheme:
// diag(i,j,k) = sum_q sum_{d1,d2} G_{d1 d2}(q) d_{d1}phi_ijk(q) d_{d2}phi_ijk(q), factored
// by the z-factor of each component pair (S^2 for xx, xy, yy; S*SD for xz, yz; SD^2 for zz).
template <int N, typename T, int GEOM>
__global__ void __launch_bounds__(128) diag_slab_kernel(const Tab2<N, T> tab,
                                                        T *__restrict__ diag,
                                                        const uint32_t *__restrict__ idx,
                                                        const T *__restrict__ geo,
                                                        const T *__restrict__ coef,
                                                        int64_t n_groups) {
  using Lo = Layout<N>;
  constexpr int CPW = Lo::CPW, LANES = Lo::LANES, N2 = Lo::N2, N3 = Lo::N3;
  constexpr unsigned MASK = Lo::MASK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= LANES) return;
  const int e = lane / N;
  const int s = lane - e * N;
  T *b0 = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * (3 * CPW * N3) + e * N3;
  T *b1 = b0 + CPW * N3;
  T *b2 = b1 + CPW * N3;
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const T *S2 = tab.S2, *SS = tab.SS, *D2 = tab.D2;
  T wr = tab.W[0];
#pragma unroll
  for (int r = 1; r < N; ++r)
    if (s == r) wr = tab.W[r];
  for (int64_t g = warp0; g < n_groups; g += nwarps) {
    // Z-slab (z = s): G at the points of the slab
    T gxx[N][N], gxy[N][N], gyy[N][N], gxz[N][N], gyz[N][N], gzz[N][N];
#pragma unroll
    for (int q = 0; q < N; ++q)
#pragma unroll
      for (int p = 0; p < N; ++p) {
        T c[6];
        if (GEOM == 0) {
          const T *gp = geo + g * (N2 * 6 * LANES) + (q * N + p) * 6 * LANES + lane;
#pragma unroll
          for (int m = 0; m < 6; ++m) c[m] = __ldg(gp + m * LANES);
        } else {
          const T *cg = geo + (g * CPW + e) * 8;
          T w = wr * tab.W[q] * tab.W[p];
          if (GEOM == 2) w *= __ldg(coef + g * (N2 * LANES) + (q * N + p) * LANES + lane);
#pragma unroll
          for (int m = 0; m < 6; ++m) c[m] = w * __ldg(cg + m);
        }
        gxx[q][p] = c[0];
        gxy[q][p] = T(2) * c[1];
        gxz[q][p] = T(2) * c[2];
        gyy[q][p] = c[3];
        gyz[q][p] = T(2) * c[4];
        gzz[q][p] = c[5];
      }
    // x then y contractions, grouped by the z factor
#pragma unroll
    for (int i = 0; i < N; ++i) {
      T ua[N], ub[N], uc[N], va[N], vb[N], wc[N]; // per q
#pragma unroll
      for (int q = 0; q < N; ++q) {
        T a = 0, b = 0, c = 0, d = 0, f = 0, h = 0;
#pragma unroll
        for (int p = 0; p < N; ++p) {
          a = fma(D2[i * N + p], gxx[q][p], a);
          b = fma(SS[i * N + p], gxy[q][p], b);
          c = fma(S2[i * N + p], gyy[q][p], c);
          d = fma(SS[i * N + p], gxz[q][p], d);
          f = fma(S2[i * N + p], gyz[q][p], f);
          h = fma(S2[i * N + p], gzz[q][p], h);
        }
        ua[q] = a; ub[q] = b; uc[q] = c; va[q] = d; vb[q] = f; wc[q] = h;
      }
#pragma unroll
      for (int j = 0; j < N; ++j) {
        T A = 0, B = 0, Cz = 0;
#pragma unroll
        for (int q = 0; q < N; ++q) {
          A = fma(S2[j * N + q], ua[q], A);
          A = fma(SS[j * N + q], ub[q], A);
          A = fma(D2[j * N + q], uc[q], A);
          B = fma(S2[j * N + q], va[q], B);
          B = fma(SS[j * N + q], vb[q], B);
          Cz = fma(S2[j * N + q], wc[q], Cz);
        }
        b0[(s * N + j) * N + i] = A;
        b1[(s * N + j) * N + i] = B;
        b2[(s * N + j) * N + i] = Cz;
      }
    }
    __syncwarp(MASK);
    // Y-slab (y = s): z contraction and scatter
    const uint32_t *ig = idx + g * (N2 * LANES) + lane;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        T v = 0;
#pragma unroll
        for (int r = 0; r < N; ++r) {
          v = fma(S2[k * N + r], b0[(r * N + s) * N + i], v);
          v = fma(SS[k * N + r], b1[(r * N + s) * N + i], v);
          v = fma(D2[k * N + r], b2[(r * N + s) * N + i], v);
        }
        const uint32_t id = __ldg(ig + (k * N + i) * LANES);
        if (id != kInvalidIdx) atomic_add(diag + id, v);
      }
    __syncwarp(MASK);
  }
}

} // namespace kern

// host-side launchers, one translation unit per degree (laplace_p<degree>.cu)
struct SlabLaunch {
  const void *src;
  void *dst;
  const uint32_t *idx;
  const void *geo;
  const void *coef;
  int64_t n_groups;
  int geom; // 0 full, 1 affine, 2 affine + coefficient
  int dtype;
  int grid;
  cudaStream_t stream;
  const double *S, *SD, *D, *W; // host tables (double), converted to the kernel type
};
void launch_vmult_p1(const SlabLaunch &);
void launch_vmult_p2(const SlabLaunch &);
void launch_vmult_p3(const SlabLaunch &);
void launch_vmult_p4(const SlabLaunch &);
void launch_vmult_p5(const SlabLaunch &);
void launch_vmult_p6(const SlabLaunch &);
void launch_diag_p1(const SlabLaunch &);
void launch_diag_p2(const SlabLaunch &);
void launch_diag_p3(const SlabLaunch &);
void launch_diag_p4(const SlabLaunch &);
void launch_diag_p5(const SlabLaunch &);
void launch_diag_p6(const SlabLaunch &);
int occupancy_vmult_p1(int dtype, int geom);
int occupancy_vmult_p2(int dtype, int geom);
int occupancy_vmult_p3(int dtype, int geom);
int occupancy_vmult_p4(int dtype, int geom);
int occupancy_vmult_p5(int dtype, int geom);
int occupancy_vmult_p6(int dtype, int geom);
int occupancy_diag_p1(int dtype, int geom);
int occupancy_diag_p2(int dtype, int geom);
int occupancy_diag_p3(int dtype, int geom);
int occupancy_diag_p4(int dtype, int geom);
int occupancy_diag_p5(int dtype, int geom);
int occupancy_diag_p6(int dtype, int geom);

} // namespace pmg
