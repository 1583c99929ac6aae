// Sum-factorized cell kernels of the continuous Q_p Laplace operator for sm_100a.
//
// What they compute is the BK3 cell operator of the reference
// (include/kernels/bk3_kokkos_kernel.h:25-746): per cell gather the nodal values (Dirichlet
// entries read as 0), interpolate to the Gauss points, take collocation gradients, apply
// the symmetric geometry tensor G, integrate against the gradients and scatter-add.  How
// they compute it is laid out for the B200:
//
//  * A warp owns a group of CPW = floor(32/N) consecutive cells (N = p+1 nodes per
//    direction), N lanes per cell.  Lane s of a cell works on a slab of the cell: the
//    plane y = s ("Y-slab") while gathering, contracting along x and z and scattering,
//    and the plane z = s ("Z-slab") while contracting along x and y and applying G.
//    Contractions along the slab stay in registers; switching slabs is one warp-local
//    exchange through shared memory.  The operator is factored (SD = S*D, the derivative of
//    the nodal basis at the Gauss points) so that only two switches are needed per cell:
//        Y-slab:  w = Sz Sx u,  wz = SDz Sx u,  wx = Sz SDx u
//        Z-slab:  dx = Sy wx, dy = SDy w, dz = Sy wz;  f = G grad u;
//                 a = Sy^T SDx^T fx + SDy^T Sx^T fy,  c = Sy^T Sx^T fz
//        Y-slab:  out = Sz^T a + SDz^T c
//    No block-wide barrier is used; warps are independent.
//  * The index map and G are stored lane-contiguous per group ([group][point][lane]), so
//    every load of them is a fully coalesced warp access; G is column-major per group (one
//    contiguous chunk per x point). The ring variant streams the columns of the current
//    group through a two-slot shared-memory ring filled by TMA bulk copies one column ahead;
//    the direct-load variant bulk-prefetches the next group's G into L2
//    (cp.async.bulk.prefetch.L2) instead.
//  * Scatter with native FP64/FP32 atomic adds (red.global.add) into L2.
//  * The 1D tables are kernel parameters (constant bank), indexed at compile time.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pmg {
namespace kern {

constexpr uint32_t kInvalidIdx = 0xFFFFFFFFu;

// Even/odd form of a 1D apply out_q = sum_i M(i, q) in_i for a matrix with the mirror
// symmetry M(N-1-i, N-1-q) = SIG M(i, q) (SIG = +1: S and its transpose; -1: SD and its
// transpose, from the symmetric GLL nodes and Gauss points): with e_i = in_i + in_{N-1-i},
// o_i = in_i - in_{N-1-i} (i < H = N/2) and E_q = sum_i A(i,q) e_i + C(q) in_H (odd N),
// O_q = sum_i B(i,q) o_i, out_q = E_q + O_q and out_{N-1-q} = SIG (E_q - O_q): about half
// the multiply-adds of the plain product.  A = (M(i,q) + M(N-1-i,q))/2, B = (M(i,q) -
// M(N-1-i,q))/2, C(q) = M(H,q), for q < Q = (N+1)/2.
template <int N, typename T> struct EvenOdd {
  static constexpr int H = N / 2, Q = (N + 1) / 2;
  T A[H * Q > 0 ? H * Q : 1], B[H * Q > 0 ? H * Q : 1], C[Q];
};

template <int N, typename T> struct Tab {
  T S[N * N];  // S[i*N+q]  = phi_i(g_q)
  T SD[N * N]; // SD[i*N+q] = phi_i'(g_q)
  T D[N * N];  // D[n*N+q]  = l_n'(g_q) on the Gauss points
  T W[N];      // Gauss weights
  EvenOdd<N, T> eS, eSD;   // S and SD (input node i, output point q)
  EvenOdd<N, T> eST, eSDT; // their transposes (input point q, output node i)
};

// fill the even/odd tables of `tab` from the row-major N x N tables S and SD (host)
template <int N, typename T> inline void fill_even_odd(Tab<N, T> &tab, const double *S, const double *SD) {
  constexpr int H = N / 2, Q = (N + 1) / 2;
  auto fill = [&](EvenOdd<N, T> &e, auto M) {
    for (int i = 0; i < H; ++i)
      for (int q = 0; q < Q; ++q) {
        e.A[i * Q + q] = (T)(0.5 * (M(i, q) + M(N - 1 - i, q)));
        e.B[i * Q + q] = (T)(0.5 * (M(i, q) - M(N - 1 - i, q)));
      }
    for (int q = 0; q < Q; ++q) e.C[q] = (N & 1) ? (T)M(H, q) : T(0);
  };
  fill(tab.eS, [&](int i, int q) { return S[i * N + q]; });
  fill(tab.eSD, [&](int i, int q) { return SD[i * N + q]; });
  fill(tab.eST, [&](int r, int k) { return S[k * N + r]; });
  fill(tab.eSDT, [&](int r, int k) { return SD[k * N + r]; });
}

// out_q = sum_i M(i, q) in_i by the even/odd form; f(q, out_q) is called once for every q
template <int N, typename T, int SIG, typename F>
__device__ __forceinline__ void eo_apply(const EvenOdd<N, T> &m, const T (&in)[N], F &&f) {
  constexpr int H = N / 2, Q = (N + 1) / 2;
  T e[H > 0 ? H : 1], o[H > 0 ? H : 1];
#pragma unroll
  for (int i = 0; i < H; ++i) {
    e[i] = in[i] + in[N - 1 - i];
    o[i] = in[i] - in[N - 1 - i];
  }
#pragma unroll
  for (int q = 0; q < H; ++q) {
    T E = (N & 1) ? m.C[q] * in[H] : T(0), O = T(0);
#pragma unroll
    for (int i = 0; i < H; ++i) {
      E = fma(m.A[i * Q + q], e[i], E);
      O = fma(m.B[i * Q + q], o[i], O);
    }
    f(q, E + O);
    f(N - 1 - q, SIG > 0 ? E - O : O - E);
  }
  if (N & 1) {
    T v = T(0);
    if (SIG > 0) {
      v = m.C[H] * in[H];
#pragma unroll
      for (int i = 0; i < H; ++i) v = fma(m.A[i * Q + H], e[i], v);
    } else {
#pragma unroll
      for (int i = 0; i < H; ++i) v = fma(m.B[i * Q + H], o[i], v);
    }
    f(H, v);
  }
}

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

// L2 eviction policies: the geometry and index streams are read once and should not push
// the reused src/dst lines out of L2; src gathers and dst atomics should stay.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint64_t policy_evict_normal() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes, uint64_t pol) {
  asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(p), "r"(bytes),
               "l"(pol)
               : "memory");
}

// read-only loads with an L2 policy, not allocated in L1
__device__ __forceinline__ double ld_stream(const double *p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream(const float *p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
// the same loads as volatile asm: issued where they stand in the program, not sunk towards
// their first use (the register pipeline of vmult_slab_kernel issues them a phase early)
__device__ __forceinline__ uint32_t ld_stream_early(const uint32_t *p, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_keep_early(const double *p, uint64_t pol) {
  double v;
  asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_keep_early(const float *p, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
// gathered loads that are reused by neighbouring cells
__device__ __forceinline__ double ld_keep(const double *p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_keep(const float *p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void red_keep(double *p, double v, uint64_t pol) {
  asm volatile("red.global.add.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void red_keep(float *p, float v, uint64_t pol) {
  asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

// ---- bulk copies into shared memory completed on an mbarrier (sm_90+ async proxy) ----
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src, uint32_t bytes,
                                          uint64_t *bar, uint64_t pol) {
  // order earlier generic-proxy reads of the destination before the async-proxy write
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
               " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst_smem)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}
// bounded wait: gives up after `limit` polls, records the event in *err and returns false
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  unsigned int *err, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicOr(err, 1u);
  return false;
}

// ---- per-thread asynchronous copies into shared memory (cp.async, completion per thread) ----
__device__ __forceinline__ void cp_async(void *dst_smem, const void *src, int bytes, int src_bytes,
                                         uint64_t pol) {
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2, %3;" ::"r"(smem_u32(dst_smem)),
                 "l"(src), "r"(src_bytes), "l"(pol)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2, %3;" ::"r"(smem_u32(dst_smem)),
                 "l"(src), "r"(src_bytes), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

// GEOM 0: full G per quadrature point, geo = [group][N (x point p)][N (y point q)][6][LANES]
// GEOM 1: affine, geo = [cell][8] (6 used) multiplied by the tensor Gauss weight; affine cells
//         are axis-aligned boxes, so only rr, ss, tt are nonzero (the vmult uses those three)
// GEOM 2: affine as 1, times coef = [group][N^2][LANES] per quadrature point
//
// Register budget: every phase streams over one index so that at most ~2 N^2 values are
// live per lane (the accumulators of the back-contraction plus one column):
//   phase 1 (Y-slab y=s), per x point p:   t = Sx u, tx = SDx u along k, then
//            w = Sz t, wz = SDz t, wx = Sz tx  -> shared (z, y=s, p)
//   phase 2 (Z-slab z=s), per x point p:   dx = Sy wx, dy = SDy w, dz = Sy wz at (., p),
//            f = G grad u, a += SDx(.,p)^T (Sy^T fx) + Sx(.,p)^T (SDy^T fy);  fz -> shared
//            (in place over the consumed column of wx), then c = Sy^T Sx^T fz
//   phase 3 (Y-slab), per x node i:        out = Sz^T a + SDz^T c, scatter
// Each lane overwrites only its own slab's region of the buffers between the two
// exchanges, so only the two exchanges (and the end of a group) need a __syncwarp.
// compile-time overrides of the tuned choices in vmult_slab_kernel (-1: the tuned default,
// 0: off, 1: on): even/odd phase-2 contractions (EO2), rolled deferred passes and phase 3
// (TUNR), phase 2 without accumulators (DEFER), paired-point x contractions (EO1X)
#ifndef PMG_VMULT_EO_PHASE2
#define PMG_VMULT_EO_PHASE2 -1
#endif
#ifndef PMG_VMULT_ROLL_TAIL
#define PMG_VMULT_ROLL_TAIL -1
#endif
#ifndef PMG_VMULT_DEFER
#define PMG_VMULT_DEFER -1
#endif
#ifndef PMG_VMULT_EO_PHASE1X
#define PMG_VMULT_EO_PHASE1X -1
#endif
// L2 prefetch of the next group's geometry (full and inverse-Jacobian layouts): -1 the tuned
// default, 1 evict-first, 0 none, 2 evict-normal.  The default prefetches (evict-first) for the
// direct-load variants only: the ring variant streams each column through its TMA ring
// already, and the extra prefetch only added L2 traffic (deformed cube on B200, FP64 128^3:
// Q4 3914-3968 -> 3721-3737 us, Q5 at 64^3 1188 -> 1157 us, Q3 unchanged without it; FP32
// ring variants Q3 972 -> 914 us, Q2 398 -> 381 us; FP32 Q4 with direct loads 2156 ->
// 2430-2497 us without it)
#ifndef PMG_VMULT_PREFETCH
#define PMG_VMULT_PREFETCH -1
#endif
template <int N> struct Stride {
  // per-cell stride of the exchange buffers, padded where that lowers bank conflicts of
  // the two exchange patterns (offsets N*s and N*N*s within a cell)
  static constexpr int CELL = N * N * N + ((N == 3 || N == 5) ? 0 : 1);
};

// Inverse-Jacobian formulation (geo = [group][x point p][y point q][10][LANES]: J^{-1} row by
// row, then JxW): the physical gradient J^{-T} grad_ref, times JxW, and back with J^{-1}
// (include/kernels/portable_local_laplace_operator.h:329-347).
template <int N, typename T>
__device__ __forceinline__ void invjac_flux(const T *__restrict__ geo, int64_t g, int lane, int q, int p,
                                            uint64_t pol, T dx, T dy, T dz, T (&f)[3]) {
  constexpr int LANES = Layout<N>::LANES, N2 = Layout<N>::N2;
  const T *gp = geo + g * (N2 * 10 * LANES) + (p * N + q) * 10 * LANES + lane;
  T iv[9];
#pragma unroll
  for (int m = 0; m < 9; ++m) iv[m] = ld_stream(gp + m * LANES, pol);
  const T jw = ld_stream(gp + 9 * LANES, pol);
  T gx[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gx[k] = jw * (iv[k] * dx + iv[3 + k] * dy + iv[6 + k] * dz);
#pragma unroll
  for (int d = 0; d < 3; ++d) f[d] = iv[3 * d] * gx[0] + iv[3 * d + 1] * gx[1] + iv[3 * d + 2] * gx[2];
}

template <int N, typename T, int GEOM, bool SMEM_G>
__device__ __forceinline__ void load_g6(const T *__restrict__ geo, const T *gs,
                                        const T *__restrict__ coef, const Tab<N, T> &tab,
                                        int64_t g, int lane, int e, int q, int p, T wr,
                                        uint64_t pol, T (&c)[6]) {
  using Lo = Layout<N>;
  constexpr int LANES = Lo::LANES, N2 = Lo::N2, CPW = Lo::CPW;
  if (GEOM == 0 && SMEM_G) {
    const T *gp = gs + q * 6 * LANES + lane; // the staged x column p
#pragma unroll
    for (int m = 0; m < 6; ++m) c[m] = gp[m * LANES];
  } else if (GEOM == 0) {
    const T *gp = geo + g * (N2 * 6 * LANES) + (p * N + q) * 6 * LANES + lane;
#pragma unroll
    for (int m = 0; m < 6; ++m) c[m] = ld_stream(gp + m * LANES, pol);
  } else {
    const T *cg = geo + (g * CPW + e) * 8;
    T w = wr * tab.W[q] * tab.W[p];
    if (GEOM == 2) w *= ld_stream(coef + g * (N2 * LANES) + (q * N + p) * LANES + lane, pol);
#pragma unroll
    for (int m = 0; m < 6; ++m) c[m] = w * __ldg(cg + m);
  }
}

// resident blocks of 128 threads per SM the register allocation is sized for; matches the
// shared-memory footprint (3 exchange buffers per warp) of each degree and type
// FP64 affine kernels at 3 <= N <= 5: 0 plain runtime loops, 1 with even/odd z contractions,
// 2 (default) unrolled with every even/odd form at up to 255 registers, which measured fastest
// on B200 despite some spills (64^3 / 48^3 with kappa: Q4 217 -> 174 us, Q3 205 -> 200 us,
// Q2 74 -> 67 us; mode 1: 210, 199, 72 us)
// (at N = 6 and 7 the unrolled FP64 form spills 0.5-1.4 KB and measured 1.6-2.1x slower)
#ifndef PMG_VMULT_F64_AFFINE_NMAX
#define PMG_VMULT_F64_AFFINE_NMAX 5
#endif
#ifndef PMG_VMULT_F64_AFFINE_MODE
#define PMG_VMULT_F64_AFFINE_MODE 2
#endif
template <int N, typename T, int GEOM> constexpr int f64_affine_mode_v =
    (sizeof(T) == 8 && N <= PMG_VMULT_F64_AFFINE_NMAX && N >= 3 && (GEOM == 1 || GEOM == 2)) ? PMG_VMULT_F64_AFFINE_MODE : 0;
template <int N, typename T, int GEOM = 1> struct MinBlocks {
  static constexpr int value =
      f64_affine_mode_v<N, T, GEOM> == 2
          ? 2
          : (sizeof(T) == 8 ? (N >= 6 ? 2 : 3) : ((N == 7 && (GEOM == 0 || GEOM == 3)) ? 3 : 2));
};
// outer streaming loops: runtime loops for FP64 (bounded live registers), unrolled for FP32
// (registers are cheap at 4 bytes and unrolling keeps the tables as immediate operands),
// except FP32 Q6 with full geometry, where runtime loops at 170 registers (12 warps/SM)
// measured 1.4x faster on B200 than the unrolled form at 255
// (FP32 Q6 affine in runtime loops at 142 registers, 12 warps/SM, measured no faster than the
// unrolled form at 8 warps/SM)
template <int N, typename T, int GEOM = 1> struct Unroll {
  static constexpr int value = f64_affine_mode_v<N, T, GEOM> == 2
                                   ? N
                                   : ((sizeof(T) == 8 || (N == 7 && (GEOM == 0 || GEOM == 3))) ? 1 : N);
};

// Shared memory per warp of vmult_slab_kernel: 3 exchange buffers, plus (SMEM_G) the
// geometry column ring and its two mbarriers, plus the gather pipeline (PIPE): 1 = one
// group's index block, 2 = one group's gathered src values and two index blocks, 3 (the
// register pipeline) nothing.
template <int N, typename T, bool SMEM_G, int PIPE = 0> struct SlabSmem {
  static constexpr size_t XCHG = size_t(3) * Layout<N>::CPW * Stride<N>::CELL * sizeof(T);
  static constexpr size_t CHUNK = size_t(N) * 6 * Layout<N>::LANES * sizeof(T); // one x column
  static constexpr size_t GEO = SMEM_G ? 2 * CHUNK : 0;                         // two-slot ring
  static constexpr size_t IDXB = size_t(Layout<N>::N2) * Layout<N>::LANES * 4;   // one index block
  static constexpr size_t SRC = PIPE == 2 ? size_t(Layout<N>::N2) * Layout<N>::LANES * sizeof(T) : 0;
  static constexpr size_t IDX = (PIPE == 0 || PIPE == 3) ? 0 : (PIPE == 1 ? 1 : 2) * IDXB;
  static constexpr size_t OFF_SRC = ((GEO + XCHG + 15) / 16) * 16;
  static constexpr size_t OFF_IDX = OFF_SRC + ((SRC + 15) / 16) * 16;
  static constexpr size_t PER_WARP = OFF_IDX + ((IDX + 15) / 16) * 16 + (SMEM_G ? 16 : 0);
};

// SMEM_G: the x columns of each group's geometry (contiguous chunks) stream through a
// two-slot shared-memory ring; the copy of the next column (or of the next group's first
// column) is issued when a column starts, so it overlaps with that column's work.
// Warps share nothing (each has its own ring, barriers and buffers): any warps per block.
// PIPE: the dependent index -> src gather is taken off the critical path by per-thread
// cp.async copies one group ahead (each lane copies exactly the entries it later reads, so
// cp.async.wait_group alone orders them):
//   1: the next group's index block is copied once the current gather has read its own;
//   2: the next group's src values are copied (zero-filled at Dirichlet entries) right after
//      the current group's first phase, from an index block copied a group earlier still;
//      the scatter reads its indices from shared memory as well;
//   3: a register pipeline without shared memory: the next group's index block is loaded
//      into registers when phase 2 starts (it lands during phase 2) and its src values when
//      phase 3 starts (they land during the scatter); phase 1 then starts with the gathered
//      values in registers.  It costs N^2 index registers through phase 2 and N^2 values
//      through phase 3, which the shared-memory-bound ring variant has to spare.
template <int N, typename T, int GEOM, bool SMEM_G, int PIPE = 0>
__global__ void __launch_bounds__(SMEM_G ? 256 : 128, (SMEM_G ? 1 : MinBlocks<N, T, GEOM>::value))
    vmult_slab_kernel(const __grid_constant__ Tab<N, T> tab, const T *__restrict__ src, T *__restrict__ dst,
                      const uint32_t *__restrict__ idx, const T *__restrict__ geo,
                      const T *__restrict__ coef, int64_t n_groups, unsigned int *err) {
  using Lo = Layout<N>;
  constexpr int CPW = Lo::CPW, LANES = Lo::LANES, N2 = Lo::N2;
  constexpr int CS = Stride<N>::CELL;
  constexpr unsigned MASK = Lo::MASK;
  constexpr int UNR = SMEM_G ? N : Unroll<N, T, GEOM>::value;
  // even/odd contractions where they measured faster on B200 (the FP64 runtime-loop
  // variants spill with the extra live values; N = 2 gains nothing):
  //  EO   z contractions of phases 1 and 3: the ring variants, the FP32 direct variants
  //       other than N = 6 and N = 7 full geometry, and the FP64 affine kernels at N <= 5
  //  EO2  phase 2 (the y contractions of the columns, the x contraction of fz): the ring
  //       variants, FP32 N <= 5, every N = 7 variant and the unrolled FP64 affine kernels
  //  EO1X x contractions of phase 1 by mirrored pairs of points (the point loop unrolled):
  //       with EO except at N = 6
  //  DEFER (below) phase 2 without register accumulators, at N = 7
  constexpr bool EO =
      N >= 3 && (SMEM_G || (sizeof(T) == 4 && N != 6 && !(N == 7 && (GEOM == 0 || GEOM == 3))) ||
                 f64_affine_mode_v<N, T, GEOM> >= 1);
  constexpr bool EO2 =
      PMG_VMULT_EO_PHASE2 >= 0
          ? (PMG_VMULT_EO_PHASE2 == 1 && N >= 3)
          : N >= 3 && (SMEM_G || (sizeof(T) == 4 && N <= 5) || N == 7 || f64_affine_mode_v<N, T, GEOM> == 2);
  // DEFER: phase 2 keeps no accumulators; y1, y2 and x3 are parked in the lane's own plane and
  // contracted along x (and y) afterwards in even/odd form (N = 7: 8-35 % faster on B200,
  // the runtime-loop FP64 variants lose their spills; slower at N <= 6)
  constexpr bool DEFER = EO2 && (PMG_VMULT_DEFER >= 0 ? PMG_VMULT_DEFER == 1 : N == 7);
  // the deferred passes and phase 3 index the tables by their inner loops only, so their
  // outer loops can stay rolled (smaller code) at no table-load cost: FP32 Q4 affine falls
  // from ~205 to 128 registers and runs 21 % faster on B200; every other variant measured
  // 1-15 % slower rolled
  constexpr int TUNR = PMG_VMULT_ROLL_TAIL >= 0 ? (PMG_VMULT_ROLL_TAIL == 1 ? 1 : UNR)
                                                : ((sizeof(T) == 4 && N == 5 && (GEOM == 1 || GEOM == 2)) ? 1 : UNR);
  constexpr bool EO1X = PMG_VMULT_EO_PHASE1X >= 0 ? (PMG_VMULT_EO_PHASE1X == 1 && EO && UNR == N)
                                                  : (EO && UNR == N && N != 6);
  using SM = SlabSmem<N, T, SMEM_G, PIPE>;
  static_assert(!(SMEM_G && PIPE == 2), "src staging is not combined with the geometry ring");
  constexpr int NCOMP = GEOM == 3 ? 10 : 6; // geometry values per quadrature point
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  if (lane >= LANES) return;
  const int e = lane / N;
  const int s = lane - e * N;
  unsigned char *wsm = smem_raw + (threadIdx.x >> 5) * SM::PER_WARP;
  T *ring = reinterpret_cast<T *>(wsm);                     // geometry column ring (SMEM_G)
  T *bufW = reinterpret_cast<T *>(wsm + SM::GEO) + e * CS;  // exchange buffers
  T *bufZ = bufW + CPW * CS;
  T *bufX = bufZ + CPW * CS;
  uint64_t *bars = reinterpret_cast<uint64_t *>(wsm + SM::PER_WARP - 16);
  T *sbuf = reinterpret_cast<T *>(wsm + SM::OFF_SRC) + lane;               // [N2][LANES] (PIPE 2)
  uint32_t *ibuf = reinterpret_cast<uint32_t *>(wsm + SM::OFF_IDX) + lane; // [slot][N2][LANES]
  constexpr int CHUNK_ELEMS = N * 6 * LANES;
  uint32_t chunk = 0; // columns consumed so far; slot = chunk & 1, parity = (chunk >> 1) & 1
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const uint64_t pol_first = policy_evict_first(), pol_last = policy_evict_last();
  if (SMEM_G && GEOM == 0) {
    if (lane == 0) {
      mbar_init(&bars[0], 1);
      mbar_init(&bars[1], 1);
      if (warp0 < n_groups)
        bulk_load(ring, geo + warp0 * (N2 * 6 * LANES), CHUNK_ELEMS * sizeof(T), &bars[0], pol_first);
    }
    __syncwarp(MASK);
  }
  T wr = tab.W[0]; // Gauss weight of this lane's z point (affine geometry)
#pragma unroll
  for (int r = 1; r < N; ++r)
    if (s == r) wr = tab.W[r];

  // gather pipeline: copy the index block of group gg into slot `slot` / the src values
  // named by slot `slot` into sbuf; every call commits exactly one cp.async group
  auto issue_idx = [&](int64_t gg, int slot) {
    if (gg < n_groups) {
      const uint32_t *ip = idx + gg * (N2 * LANES) + lane;
#pragma unroll
      for (int a = 0; a < N2; ++a) cp_async(ibuf + (slot * N2 + a) * LANES, ip + a * LANES, 4, 4, pol_first);
    }
    cp_async_commit();
  };
  auto issue_src = [&](bool valid, int slot) {
    if (valid) {
#pragma unroll
      for (int a = 0; a < N2; ++a) {
        const uint32_t id = ibuf[(slot * N2 + a) * LANES];
        const bool ok = id != kInvalidIdx;
        cp_async(sbuf + a * LANES, ok ? src + id : src, (int)sizeof(T), ok ? (int)sizeof(T) : 0, pol_last);
      }
    }
    cp_async_commit();
  };
  int it = 0; // groups done by this warp (PIPE 2: index slot of group g = it & 1)
  // PIPE 3: the next group's index block and gathered src values, carried in registers
  constexpr int RP = PIPE == 3 ? N : 1;
  uint32_t nidx[RP][RP];
  T nsrc[RP][RP];
  auto load_next_idx = [&](int64_t gg) {
    if (PIPE == 3 && gg < n_groups) {
      const uint32_t *ip = idx + gg * (N2 * LANES) + lane;
#pragma unroll
      for (int k = 0; k < RP; ++k)
#pragma unroll
        for (int i = 0; i < RP; ++i) nidx[k][i] = ld_stream_early(ip + (k * N + i) * LANES, pol_first);
    }
  };
  auto load_next_src = [&](int64_t gg) {
    if (PIPE == 3 && gg < n_groups) {
#pragma unroll
      for (int k = 0; k < RP; ++k)
#pragma unroll
        for (int i = 0; i < RP; ++i)
          nsrc[k][i] = nidx[k][i] != kInvalidIdx ? ld_keep_early(src + nidx[k][i], pol_last) : T(0);
    }
  };
  if (PIPE == 3) {
    load_next_idx(warp0);
    load_next_src(warp0);
  }
  if (PIPE == 1) issue_idx(warp0, 0);
  if (PIPE == 2) {
    issue_idx(warp0, 0);
    cp_async_wait<0>();
    issue_src(warp0 < n_groups, 0);
    issue_idx(warp0 + nwarps, 1);
  }

  for (int64_t g = warp0; g < n_groups; g += nwarps, ++it) {
    constexpr bool PREFETCH = PMG_VMULT_PREFETCH == -1 ? !SMEM_G : PMG_VMULT_PREFETCH != 0;
    if ((GEOM == 0 || GEOM == 3) && PREFETCH && lane == 0 && g + nwarps < n_groups)
      prefetch_l2(geo + (g + nwarps) * (N2 * NCOMP * LANES), N2 * NCOMP * LANES * sizeof(T),
                  PMG_VMULT_PREFETCH == 2 ? policy_evict_normal() : pol_first);
    const uint32_t *ig = idx + g * (N2 * LANES) + lane;
    const int slot = it & 1;

    // ---- phase 1: gather the Y-slab y = s, u[k][i] = src at node (i, s, k) ----
    {
      T u[N][N];
      if (PIPE == 3) {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int i = 0; i < N; ++i) u[k][i] = nsrc[k < RP ? k : 0][i < RP ? i : 0];
      } else if (PIPE == 2) {
        cp_async_wait<1>(); // this group's src values (the next index block may be in flight)
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int i = 0; i < N; ++i) u[k][i] = sbuf[(k * N + i) * LANES];
      } else if (PIPE == 1) {
        cp_async_wait<0>(); // this group's index block
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int i = 0; i < N; ++i) {
            const uint32_t id = ibuf[(k * N + i) * LANES];
            u[k][i] = (id != kInvalidIdx) ? ld_keep(src + id, pol_last) : T(0);
          }
      } else {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int i = 0; i < N; ++i) {
            const uint32_t id = ld_stream(ig + (k * N + i) * LANES, pol_first);
            u[k][i] = (id != kInvalidIdx) ? ld_keep(src + id, pol_last) : T(0);
          }
      }
      if constexpr (EO1X) {
        // x contractions t = Sx u, tx = SDx u by mirrored pairs of points (p, N-1-p): the
        // sums and differences of mirrored nodes replace u in place (u[k][i] = e_i and
        // u[k][N-1-i] = o_i for i < H)
        constexpr int H = N / 2, Q = (N + 1) / 2;
        // z contraction of one x point p in even/odd form: w = Sz t, wz = SDz t, wx = Sz tx
        auto zstore = [&](int p, const T(&t)[N], const T(&tx)[N]) {
          eo_apply<N, T, 1>(tab.eS, t, [&](int r, T v) { bufW[(r * N + s) * N + p] = v; });
          eo_apply<N, T, -1>(tab.eSD, t, [&](int r, T v) { bufZ[(r * N + s) * N + p] = v; });
          eo_apply<N, T, 1>(tab.eS, tx, [&](int r, T v) { bufX[(r * N + s) * N + p] = v; });
        };
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int i = 0; i < H; ++i) {
            const T a = u[k][i], b = u[k][N - 1 - i];
            u[k][i] = a + b;
            u[k][N - 1 - i] = a - b;
          }
#pragma unroll
        for (int p = 0; p < H; ++p) {
          T tp[N], tm[N], xp[N], xm[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            T es = (N & 1) ? tab.eS.C[p] * u[k][H] : T(0), os = T(0);
            T ed = (N & 1) ? tab.eSD.C[p] * u[k][H] : T(0), od = T(0);
#pragma unroll
            for (int i = 0; i < H; ++i) {
              es = fma(tab.eS.A[i * Q + p], u[k][i], es);
              os = fma(tab.eS.B[i * Q + p], u[k][N - 1 - i], os);
              ed = fma(tab.eSD.A[i * Q + p], u[k][i], ed);
              od = fma(tab.eSD.B[i * Q + p], u[k][N - 1 - i], od);
            }
            tp[k] = es + os;
            tm[k] = es - os;
            xp[k] = ed + od;
            xm[k] = od - ed;
          }
          zstore(p, tp, xp);
          zstore(N - 1 - p, tm, xm);
        }
        if (N & 1) {
          T t[N], tx[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            T a = tab.eS.C[H] * u[k][H], b = T(0);
#pragma unroll
            for (int i = 0; i < H; ++i) {
              a = fma(tab.eS.A[i * Q + H], u[k][i], a);
              b = fma(tab.eSD.B[i * Q + H], u[k][N - 1 - i], b);
            }
            t[k] = a;
            tx[k] = b;
          }
          zstore(H, t, tx);
        }
      } else {
#pragma unroll UNR
        for (int p = 0; p < N; ++p) {
          T t[N], tx[N];
#pragma unroll
          for (int k = 0; k < N; ++k) {
            T a = T(0), b = T(0);
#pragma unroll
            for (int i = 0; i < N; ++i) {
              a = fma(tab.S[i * N + p], u[k][i], a);
              b = fma(tab.SD[i * N + p], u[k][i], b);
            }
            t[k] = a;
            tx[k] = b;
          }
          // z contraction: w = Sz t, wz = SDz t, wx = Sz tx at (z = r, y = s, x = p)
          if constexpr (EO) {
            eo_apply<N, T, 1>(tab.eS, t, [&](int r, T v) { bufW[(r * N + s) * N + p] = v; });
            eo_apply<N, T, -1>(tab.eSD, t, [&](int r, T v) { bufZ[(r * N + s) * N + p] = v; });
            eo_apply<N, T, 1>(tab.eS, tx, [&](int r, T v) { bufX[(r * N + s) * N + p] = v; });
          } else {
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
              bufW[o] = w;
              bufZ[o] = wz;
              bufX[o] = wx;
            }
          }
        }
      }
    }
    // the gather's shared-memory entries are consumed: refill them for the next group
    if (PIPE == 1) issue_idx(g + nwarps, 0);
    if (PIPE == 3) load_next_idx(g + nwarps); // lands during phase 2
    if (PIPE == 2) {
      cp_async_wait<0>(); // the next group's index block
      issue_src(g + nwarps < n_groups, slot ^ 1);
    }
    __syncwarp(MASK);

    // ---- phase 2: Z-slab z = s, streamed over the x point p ----
    T cd0 = T(0), cd3 = T(0), cd5 = T(0); // diagonal of the affine cell tensor
    if (GEOM == 1 || GEOM == 2) {
      const T *cg = geo + (g * CPW + e) * 8;
      cd0 = __ldg(cg);
      cd3 = __ldg(cg + 3);
      cd5 = __ldg(cg + 5);
    }
    {
      T a[N][N]; // [j][i]
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i) a[j][i] = T(0);
#pragma unroll UNR
      for (int p = 0; p < N; ++p) {
        const T *gcol = nullptr;
        if (SMEM_G && GEOM == 0) {
          // issue the next column (this group's p+1, or the next group's column 0) into the
          // other slot, whose previous column every lane finished with at the last syncwarp
          if (lane == 0) {
            const T *next = nullptr;
            if (p + 1 < N) next = geo + g * (N2 * 6 * LANES) + (p + 1) * CHUNK_ELEMS;
            else if (g + nwarps < n_groups) next = geo + (g + nwarps) * (N2 * 6 * LANES);
            if (next)
              bulk_load(ring + ((chunk + 1) & 1) * CHUNK_ELEMS, next, CHUNK_ELEMS * sizeof(T),
                        &bars[(chunk + 1) & 1], pol_first);
          }
          if (!mbar_wait_bounded(&bars[chunk & 1], (chunk >> 1) & 1, err, 1u << 24)) {
            if (lane == 0) mbar_wait_bounded(&bars[(chunk + 1) & 1], ((chunk + 1) >> 1) & 1, err, 1u << 24);
            if (PIPE == 1 || PIPE == 2) cp_async_wait<0>();
            return; // the error flag is set; let copies in flight land before leaving
          }
          gcol = ring + (chunk & 1) * CHUNK_ELEMS;
        }
        T Wc[N], Zc[N], Xc[N];
#pragma unroll
        for (int j = 0; j < N; ++j) {
          const int o = (s * N + j) * N + p;
          Wc[j] = bufW[o];
          Zc[j] = bufZ[o];
          Xc[j] = bufX[o];
        }
        T fx[N], fy[N];
        if constexpr (EO2) {
          // f = G grad u at the point (p, q) of this slab: fx, fy kept, fz -> own bufX region
          auto point = [&](int q, T dx, T dy, T dz) {
            if (GEOM == 0) {
              T gc[6];
              load_g6<N, T, GEOM, SMEM_G>(geo, gcol, coef, tab, g, lane, e, q, p, wr, pol_first, gc);
              fx[q] = gc[0] * dx + gc[1] * dy + gc[2] * dz;
              fy[q] = gc[1] * dx + gc[3] * dy + gc[4] * dz;
              bufX[(s * N + q) * N + p] = gc[2] * dx + gc[4] * dy + gc[5] * dz; // fz
            } else if (GEOM == 3) {
              T f3[3];
              invjac_flux<N, T>(geo, g, lane, q, p, pol_first, dx, dy, dz, f3);
              fx[q] = f3[0];
              fy[q] = f3[1];
              bufX[(s * N + q) * N + p] = f3[2]; // fz
            } else {
              // affine cells are axis-aligned boxes: the cell tensor is diagonal (rr, ss, tt)
              T w = wr * tab.W[q] * tab.W[p];
              if (GEOM == 2) w *= ld_stream(coef + g * (N2 * LANES) + (q * N + p) * LANES + lane, pol_first);
              fx[q] = (w * cd0) * dx;
              fy[q] = (w * cd3) * dy;
              bufX[(s * N + q) * N + p] = (w * cd5) * dz; // fz
            }
          };
          // dx = Sy wx, dy = SDy w, dz = Sy wz along the column; y1 = Sy^T fx, y2 = SDy^T fy
          T dxv[N], dyv[N], dzv[N], y1v[N], y2v[N];
          eo_apply<N, T, 1>(tab.eS, Xc, [&](int q, T v) { dxv[q] = v; });
          eo_apply<N, T, -1>(tab.eSD, Wc, [&](int q, T v) { dyv[q] = v; });
          eo_apply<N, T, 1>(tab.eS, Zc, [&](int q, T v) { dzv[q] = v; });
#pragma unroll
          for (int q = 0; q < N; ++q) point(q, dxv[q], dyv[q], dzv[q]);
          eo_apply<N, T, 1>(tab.eST, fx, [&](int j, T v) { y1v[j] = v; });
          eo_apply<N, T, -1>(tab.eSDT, fy, [&](int j, T v) { y2v[j] = v; });
          if constexpr (DEFER) {
            // park y1, y2 over the consumed column p of this lane's plane (bufW, bufZ)
#pragma unroll
            for (int j = 0; j < N; ++j) {
              bufW[(s * N + j) * N + p] = y1v[j];
              bufZ[(s * N + j) * N + p] = y2v[j];
            }
          } else {
#pragma unroll
            for (int j = 0; j < N; ++j)
#pragma unroll
              for (int i = 0; i < N; ++i) {
                a[j][i] = fma(tab.SD[i * N + p], y1v[j], a[j][i]);
                a[j][i] = fma(tab.S[i * N + p], y2v[j], a[j][i]);
              }
          }
        } else {
#pragma unroll
          for (int q = 0; q < N; ++q) {
            T dx = T(0), dy = T(0), dz = T(0);
#pragma unroll
            for (int j = 0; j < N; ++j) {
              dx = fma(tab.S[j * N + q], Xc[j], dx);
              dy = fma(tab.SD[j * N + q], Wc[j], dy);
              dz = fma(tab.S[j * N + q], Zc[j], dz);
            }
            // f = G grad u at the point (p, q) of this slab: fx, fy kept, fz -> own bufX region
            if (GEOM == 0) {
              T gc[6];
              load_g6<N, T, GEOM, SMEM_G>(geo, gcol, coef, tab, g, lane, e, q, p, wr, pol_first, gc);
              fx[q] = gc[0] * dx + gc[1] * dy + gc[2] * dz;
              fy[q] = gc[1] * dx + gc[3] * dy + gc[4] * dz;
              bufX[(s * N + q) * N + p] = gc[2] * dx + gc[4] * dy + gc[5] * dz; // fz
            } else if (GEOM == 3) {
              T f3[3];
              invjac_flux<N, T>(geo, g, lane, q, p, pol_first, dx, dy, dz, f3);
              fx[q] = f3[0];
              fy[q] = f3[1];
              bufX[(s * N + q) * N + p] = f3[2]; // fz
            } else {
              T w = wr * tab.W[q] * tab.W[p];
              if (GEOM == 2) w *= ld_stream(coef + g * (N2 * LANES) + (q * N + p) * LANES + lane, pol_first);
              fx[q] = (w * cd0) * dx;
              fy[q] = (w * cd3) * dy;
              bufX[(s * N + q) * N + p] = (w * cd5) * dz; // fz
            }
          }
#pragma unroll
          for (int j = 0; j < N; ++j) {
            T y1 = T(0), y2 = T(0);
#pragma unroll
            for (int q = 0; q < N; ++q) {
              y1 = fma(tab.S[j * N + q], fx[q], y1);
              y2 = fma(tab.SD[j * N + q], fy[q], y2);
            }
#pragma unroll
            for (int i = 0; i < N; ++i) {
              a[j][i] = fma(tab.SD[i * N + p], y1, a[j][i]);
              a[j][i] = fma(tab.S[i * N + p], y2, a[j][i]);
            }
          }
        }
        if (SMEM_G && GEOM == 0) {
          __syncwarp(MASK); // this slot may be refilled from the next column on
          ++chunk;
        }
      }
      if constexpr (DEFER) {
        // a(j, .) = SDx^T y1(j, .) + Sx^T y2(j, .), row by row in place over y1 (bufW)
#pragma unroll TUNR
        for (int j = 0; j < N; ++j) {
          T y1[N], y2[N], v[N];
#pragma unroll
          for (int p = 0; p < N; ++p) {
            y1[p] = bufW[(s * N + j) * N + p];
            y2[p] = bufZ[(s * N + j) * N + p];
          }
          eo_apply<N, T, -1>(tab.eSDT, y1, [&](int i, T x) { v[i] = x; });
          eo_apply<N, T, 1>(tab.eST, y2, [&](int i, T x) { v[i] += x; });
#pragma unroll
          for (int i = 0; i < N; ++i) bufW[(s * N + j) * N + i] = v[i];
        }
      } else {
        // a -> own slab region of bufW (all of this lane's reads of it are done)
#pragma unroll
        for (int j = 0; j < N; ++j)
#pragma unroll
          for (int i = 0; i < N; ++i) bufW[(s * N + j) * N + i] = a[j][i];
      }
    }
    if constexpr (DEFER) {
      // c = Sy^T Sx^T fz: x3 = Sx^T fz row by row in place (bufX), then Sy^T by columns into
      // this lane's region of bufZ (whose y2 values the pass above consumed)
#pragma unroll TUNR
      for (int q = 0; q < N; ++q) {
        T fz[N];
#pragma unroll
        for (int p = 0; p < N; ++p) fz[p] = bufX[(s * N + q) * N + p];
        eo_apply<N, T, 1>(tab.eST, fz, [&](int i, T x) { bufX[(s * N + q) * N + i] = x; });
      }
#pragma unroll TUNR
      for (int i = 0; i < N; ++i) {
        T x3[N];
#pragma unroll
        for (int q = 0; q < N; ++q) x3[q] = bufX[(s * N + q) * N + i];
        eo_apply<N, T, 1>(tab.eST, x3, [&](int j, T x) { bufZ[(s * N + j) * N + i] = x; });
      }
    } else {
      // c = Sy^T Sx^T fz from this lane's fz region, into its own region of bufZ
      T c[N][N];
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i) c[j][i] = T(0);
#pragma unroll UNR
      for (int q = 0; q < N; ++q) {
        T fz[N];
#pragma unroll
        for (int p = 0; p < N; ++p) fz[p] = bufX[(s * N + q) * N + p];
        if constexpr (EO2) {
          T x3v[N]; // x3 = Sx^T fz along this row
          eo_apply<N, T, 1>(tab.eST, fz, [&](int i, T v) { x3v[i] = v; });
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) c[j][i] = fma(tab.S[j * N + q], x3v[i], c[j][i]);
        } else {
#pragma unroll
          for (int i = 0; i < N; ++i) {
            T x3 = T(0);
#pragma unroll
            for (int p = 0; p < N; ++p) x3 = fma(tab.S[i * N + p], fz[p], x3);
#pragma unroll
            for (int j = 0; j < N; ++j) c[j][i] = fma(tab.S[j * N + q], x3, c[j][i]);
          }
        }
      }
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i) bufZ[(s * N + j) * N + i] = c[j][i];
    }
    __syncwarp(MASK);

    if (PIPE == 3) load_next_src(g + nwarps); // lands during the scatter

    // ---- phase 3: Y-slab y = s, out = Sz^T a + SDz^T c, scatter ----
#pragma unroll TUNR
    for (int i = 0; i < N; ++i) {
      T A[N], Cc[N];
#pragma unroll
      for (int r = 0; r < N; ++r) {
        A[r] = bufW[(r * N + s) * N + i];
        Cc[r] = bufZ[(r * N + s) * N + i];
      }
      // out = Sz^T a + SDz^T c
      T v[N];
      if constexpr (EO) {
        eo_apply<N, T, 1>(tab.eST, A, [&](int k, T x) { v[k] = x; });
        eo_apply<N, T, -1>(tab.eSDT, Cc, [&](int k, T x) { v[k] += x; });
      } else {
#pragma unroll
        for (int k = 0; k < N; ++k) {
          v[k] = T(0);
#pragma unroll
          for (int r = 0; r < N; ++r) {
            v[k] = fma(tab.S[k * N + r], A[r], v[k]);
            v[k] = fma(tab.SD[k * N + r], Cc[r], v[k]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const uint32_t id = PIPE == 2 ? ibuf[(slot * N2 + k * N + i) * LANES]
                                      : ld_stream(ig + (k * N + i) * LANES, pol_first);
        if (id != kInvalidIdx) red_keep(dst + id, v[k], pol_last);
      }
    }
    if (PIPE == 2) issue_idx(g + 2 * nwarps, slot); // this group's index slot is free
    __syncwarp(MASK); // buffers are rewritten by the next group
  }
  if (PIPE == 1 || PIPE == 2) cp_async_wait<0>(); // no copy may land after the warp has left
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
          const T *gp = geo + g * (N2 * 6 * LANES) + (p * N + q) * 6 * LANES + lane;
#pragma unroll
          for (int m = 0; m < 6; ++m) c[m] = __ldg(gp + m * LANES);
        } else if (GEOM == 3) {
          // G = JxW J^{-1} J^{-T} from the inverse-Jacobian layout, in the order of G
          const T *gp = geo + g * (N2 * 10 * LANES) + (p * N + q) * 10 * LANES + lane;
          T iv[9];
#pragma unroll
          for (int m = 0; m < 9; ++m) iv[m] = __ldg(gp + m * LANES);
          const T jw = __ldg(gp + 9 * LANES);
          int m = 0;
#pragma unroll
          for (int d1 = 0; d1 < 3; ++d1)
#pragma unroll
            for (int d2 = d1; d2 < 3; ++d2)
              c[m++] = jw * (iv[3 * d1] * iv[3 * d2] + iv[3 * d1 + 1] * iv[3 * d2 + 1] + iv[3 * d1 + 2] * iv[3 * d2 + 2]);
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
  int64_t resident_warps;      // warps of the kernel resident on the whole device
  int64_t resident_warps_ring; // the same for the geometry-ring variant of vmult
  unsigned int *err; // device flag set when a bounded wait gives up
  cudaStream_t stream;
  const double *S, *SD, *D, *W; // host tables (double), converted to the kernel type
  int64_t *launched;            // if set: receives the number of warps the vmult launched
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
// resident warps per SM of the vmult / diagonal kernels
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
