// DG-SIPG face terms on axis-aligned boxes (the interior-penalty operator of
// include/operators/portable_laplace_operator_dg.h with the fluxes of
// include/kernels/laplace_dg_kokkos_kernels.h:833-2026 and
// source/plain_laplace_solver_dg/program.cc:128-217).
//
// The cell stiffness term comes from the continuous slab kernel run on the discontinuous
// numbering (dof = cell * N^3 + l).  This file adds the face terms with one fused kernel.
// Where the box is refined at least twice (every 64 consecutive cells form a 4x4x4 cube) a
// block takes such a tile into shared memory and evaluates each face between two of its
// cells once, for both cells; the faces on the tile surface take the neighbour's trace from
// L2.  Elsewhere a block takes a batch of cells, and for each of the six faces of each cell
// it forms its own trace (the node layer on the face and the reference normal derivative)
// and the neighbour's trace, recomputed from the neighbour's DoFs straight from L2, so each
// face is evaluated from both sides.  The reference instead writes every trace to global
// face buffers and reads them back in three more launches.  In both forms every block
// writes only its own cells' DoFs: no global atomics and no face buffers.
//
// On GLL nodes with the (p+1)-point Gauss face rule the face integrals of products of
// basis functions are exact, so the face quadrature is applied as the 1D GLL mass matrix
// M1 = S diag(w) S^T in each tangential direction.
#include <algorithm>
#include <map>
#include <mutex>
#include <cstdlib>
#include <vector>

#include "dg.hpp"
#include "pmg_internal.hpp"

namespace pmg {
namespace {

template <int N, typename T> struct DGTab {
  T M1[N * N];  // 1D mass matrix of the GLL Lagrange basis
  T K1[N * N];  // 1D stiffness matrix (reference interval), for the fused cell term
  T dphi0[N];   // phi_i'(0)
  T dphi1[N];   // phi_i'(1)
};

// copy of the 1D tables in shared memory, for the accesses whose index differs between the
// lanes of a warp (a constant-bank load with divergent addresses is replayed per address)
template <int N, typename T> __device__ __forceinline__ void load_tab_shared(DGTab<N, T> &st, const DGTab<N, T> &tab) {
  constexpr int n = (int)(sizeof(DGTab<N, T>) / sizeof(T));
  const T *from = reinterpret_cast<const T *>(&tab);
  T *to = reinterpret_cast<T *>(&st);
  for (int e = threadIdx.x; e < n; e += blockDim.x) to[e] = from[e];
}

struct DGGeo {
  double h[3];   // cell extents
  double c_pen;  // sigma = c_pen / h_normal
  int dirichlet; // face mask (x-, x+, y-, y+, z-, z+)
};

// local index of the node with coordinate `layer` along d and tangential (a, b)
template <int N> __device__ __forceinline__ int face_node(int d, int layer, int a, int b) {
  // tangential directions in increasing axis order: d=0 -> (y, z); d=1 -> (x, z); d=2 -> (x, y)
  const int i = d == 0 ? layer : a;
  const int j = d == 1 ? layer : (d == 0 ? a : b);
  const int k = d == 2 ? layer : b;
  return (k * N + j) * N + i;
}

// flux values of face F (compile time, so the node indexing folds to constants) at face point
// (a, bb) of cell c: f1 = sigma [u] - {d_n u}, f2 = -[u]/2 (Dirichlet: mirror u+ = -u-)
// the N values of cell u along the normal of face direction d at face point (a, b): for d = 0
// they are contiguous and, with VEC (src 16-byte aligned, N * sizeof(T) a multiple of 16), read
// as 16-byte vectors
template <int N, typename T, int d, bool VEC>
__device__ __forceinline__ void normal_line(const T *__restrict__ u, int a, int bb, T (&line)[N]) {
  if constexpr (d == 0 && VEC) {
    const float4 *p = reinterpret_cast<const float4 *>(u + face_node<N>(0, 0, a, bb));
#pragma unroll
    for (int v = 0; v < N * (int)sizeof(T) / 16; ++v) {
      const float4 w = __ldg(p + v);
      memcpy(line + v * (16 / (int)sizeof(T)), &w, 16);
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) line[i] = __ldg(u + face_node<N>(d, i, a, bb));
  }
}

template <int N, typename T, int F, bool VEC>
__device__ __forceinline__ void face_flux(const DGTab<N, T> &tab, const DGGeo &geo, const T *__restrict__ src,
                                          const int32_t *__restrict__ nbr, int64_t c, int a, int bb, T sgn_h,
                                          T sigma, T &f1, T &f2) {
  constexpr int N3 = N * N * N, d = F >> 1, sd = F & 1;
  constexpr int own_layer = sd ? N - 1 : 0, nb_layer = sd ? 0 : N - 1;
  const T *dphi_own = sd ? tab.dphi1 : tab.dphi0;
  const T *dphi_nb = sd ? tab.dphi0 : tab.dphi1;
  const T *uo = src + c * N3;
  // the N values along the normal: the face value is one of them
  T line[N];
  normal_line<N, T, d, VEC>(uo, a, bb, line);
  const T vo = line[own_layer];
  T dn = T(0);
#pragma unroll
  for (int i = 0; i < N; ++i) dn += dphi_own[i] * line[i];
  dn *= sgn_h;
  const int32_t nb = __ldg(nbr + c * 6 + F);
  if (nb >= 0) {
    const T *un = src + int64_t(nb) * N3;
    normal_line<N, T, d, VEC>(un, a, bb, line);
    const T vn = line[nb_layer];
    T dnn = T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) dnn += dphi_nb[i] * line[i];
    dnn *= sgn_h;
    const T jump = vo - vn;
    f1 = sigma * jump - T(0.5) * (dn + dnn);
    f2 = T(-0.5) * jump;
  } else if ((geo.dirichlet >> F) & 1) {
    f1 = sigma * T(2) * vo - dn;
    f2 = -vo;
  }
}

// cells per block: six faces x N^2 face points per cell, about 384 threads per block
template <int N> constexpr int dg_batch() { return (384 / (6 * N * N)) > 0 ? 384 / (6 * N * N) : 1; }
template <int N> constexpr int dg_threads() { return ((6 * dg_batch<N>() * N * N + 31) / 32) * 32; }

// One block per batch of B cells; all six faces of the batch are evaluated at once, one
// thread per (face, cell, face point):
//   1. per face point the flux values f1 = sigma [u] - {d_n u}, f2 = -[u]/2 from the own
//      and the neighbour's traces (read through L1 / L2; every value is read by a few face
//      points of the batch);
//   2./3. the face mass matrix M1 x M1 applied along the two tangential directions, giving
//      the value-test and normal-derivative-test coefficients of every face point;
//   4. one thread per cell node sums what the six faces give it: the value test where the
//      node lies on the face layer, and the normal-derivative test on every layer.
// Phases 1-3 exchange data only among the N^2 threads of one face of one cell; where N^2
// divides 32 (N = 2, 4) those threads lie in one warp and a warp barrier orders them, so a
// batch takes two block barriers instead of four.  No shared-memory atomics.
template <int N, typename T, bool VEC>
__global__ void __launch_bounds__(dg_threads<N>(), 4) dg_face_kernel(const __grid_constant__ DGTab<N, T> tab,
                                                                  const __grid_constant__ DGGeo geo,
                                                                  const T *__restrict__ src,
                                                                  T *__restrict__ dst,
                                                                  const int32_t *__restrict__ nbr,
                                                                  int64_t n_cells) {
  constexpr int N2 = N * N, N3 = N2 * N, B = dg_batch<N>(), FP = 6 * B * N2;
  __shared__ T F1[6][B][N2], F2[6][B][N2], G1[6][B][N2], G2[6][B][N2];
  __shared__ DGTab<N, T> st;
  load_tab_shared(st, tab);
  __syncthreads();
  const int t = threadIdx.x;
  // this thread's face point (phases 2-4)
  const int f = t / (B * N2), rem = t - f * (B * N2), b = rem / N2, ab = rem - b * N2, a = ab % N, bb = ab / N;
  const int d = f >> 1, sd = f & 1;
  const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
  const T sgn_h = t < FP ? (sd ? T(1) : T(-1)) / (T)geo.h[d] : T(0); // n . grad = sgn_h d/dxi_d
  const T area = t < FP ? (T)(geo.h[ta] * geo.h[tb]) : T(0);
  const T sigma = t < FP ? (T)(geo.c_pen / geo.h[d]) : T(0);
  // a face's N^2 threads share a warp when N^2 divides 32 (blockDim is a multiple of 32)
  auto face_sync = [] {
    if constexpr (32 % (N * N) == 0) __syncwarp();
    else __syncthreads();
  };
  for (int64_t base = int64_t(blockIdx.x) * B; base < n_cells; base += int64_t(gridDim.x) * B) {
    if (t < FP) {
      const int64_t c = base + b;
      T f1 = T(0), f2 = T(0);
      if (c < n_cells) {
        // f is uniform over a warp where B * N^2 is a multiple of 32 (N = 2, 4); elsewhere a
        // warp can span two faces and takes both branches
        switch (f) {
        case 0: face_flux<N, T, 0, VEC>(tab, geo, src, nbr, c, a, bb, sgn_h, sigma, f1, f2); break;
        case 1: face_flux<N, T, 1, VEC>(tab, geo, src, nbr, c, a, bb, sgn_h, sigma, f1, f2); break;
        case 2: face_flux<N, T, 2, VEC>(tab, geo, src, nbr, c, a, bb, sgn_h, sigma, f1, f2); break;
        case 3: face_flux<N, T, 3, VEC>(tab, geo, src, nbr, c, a, bb, sgn_h, sigma, f1, f2); break;
        case 4: face_flux<N, T, 4, VEC>(tab, geo, src, nbr, c, a, bb, sgn_h, sigma, f1, f2); break;
        default: face_flux<N, T, 5, VEC>(tab, geo, src, nbr, c, a, bb, sgn_h, sigma, f1, f2); break;
        }
      }
      F1[f][b][ab] = f1 * area;
      F2[f][b][ab] = f2 * area;
    }
    face_sync();
    if (t < FP) { // face mass along a
      T g1 = T(0), g2 = T(0);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        g1 += st.M1[a * N + k] * F1[f][b][bb * N + k];
        g2 += st.M1[a * N + k] * F2[f][b][bb * N + k];
      }
      G1[f][b][ab] = g1;
      G2[f][b][ab] = g2;
    }
    face_sync();
    if (t < FP) { // along b: value-test and normal-test coefficients (F1/F2 reused)
      T tv = T(0), tn = T(0);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        tv += st.M1[bb * N + k] * G1[f][b][k * N + a];
        tn += st.M1[bb * N + k] * G2[f][b][k * N + a];
      }
      F1[f][b][ab] = tv;
      F2[f][b][ab] = tn * sgn_h;
    }
    __syncthreads();
    for (int e = t; e < B * N3; e += blockDim.x) {
      const int cb = e / N3, l = e - cb * N3;
      const int64_t c = base + cb;
      if (c >= n_cells) continue;
      const int idx[3] = {l % N, (l / N) % N, l / N2};
      T v = T(0);
#pragma unroll
      for (int ff = 0; ff < 6; ++ff) {
        const int dd = ff >> 1, ss = ff & 1;
        const int pa = dd == 0 ? idx[1] : idx[0], pb = dd == 2 ? idx[1] : idx[2];
        const int pab = pb * N + pa;
        const T *dphi = ss ? st.dphi1 : st.dphi0;
        v += F2[ff][cb][pab] * dphi[idx[dd]];
        if (idx[dd] == (ss ? N - 1 : 0)) v += F1[ff][cb][pab];
      }
      dst[c * N3 + l] += v;
    }
    __syncthreads();
  }
}

// The six faces one after another (three block barriers per face, 128 threads for a batch of
// 128 / N^2 cells): kept as the comparison form of dg_face_kernel (PMG_DG_FACE=0).
template <int N> constexpr int dg_batch_seq() { return (128 / (N * N)) > 0 ? 128 / (N * N) : 1; }

template <int N, typename T>
__global__ void __launch_bounds__(128) dg_face_seq_kernel(const __grid_constant__ DGTab<N, T> tab,
                                                          const __grid_constant__ DGGeo geo,
                                                      const T *__restrict__ src,
                                                      T *__restrict__ dst,
                                                      const int32_t *__restrict__ nbr,
                                                      int64_t n_cells) {
  constexpr int N2 = N * N, N3 = N2 * N, B = dg_batch_seq<N>();
  __shared__ T own[B][N3];
  __shared__ T out[B][N3];
  __shared__ T F1[B][N2], F2[B][N2], G1[B][N2], G2[B][N2];
  const int t = threadIdx.x;
  for (int64_t base = int64_t(blockIdx.x) * B; base < n_cells; base += int64_t(gridDim.x) * B) {
    for (int e = t; e < B * N3; e += blockDim.x) {
      const int b = e / N3, l = e - b * N3;
      const int64_t c = base + b;
      own[b][l] = c < n_cells ? src[c * N3 + l] : T(0);
      out[b][l] = T(0);
    }
    __syncthreads();
    for (int f = 0; f < 6; ++f) {
      const int d = f >> 1, s = f & 1;
      const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
      const T hd = (T)geo.h[d];
      const T sgn_h = (s ? T(1) : T(-1)) / hd; // n . grad = sgn_h * d/dxi_d
      const T area = (T)(geo.h[ta] * geo.h[tb]);
      const T sigma = (T)(geo.c_pen / geo.h[d]);
      const T *dphi_own = s ? tab.dphi1 : tab.dphi0;
      const T *dphi_nb = s ? tab.dphi0 : tab.dphi1;
      const int own_layer = s ? N - 1 : 0, nb_layer = s ? 0 : N - 1;
      const bool bc_dirichlet = (geo.dirichlet >> f) & 1;
      if (t < B * N2) {
        const int b = t / N2, ab = t - b * N2, a = ab % N, bb = ab / N;
        const int64_t c = base + b;
        T f1 = T(0), f2 = T(0);
        if (c < n_cells) {
          T vo = own[b][face_node<N>(d, own_layer, a, bb)], dn = T(0);
#pragma unroll
          for (int i = 0; i < N; ++i) dn += dphi_own[i] * own[b][face_node<N>(d, i, a, bb)];
          dn *= sgn_h;
          const int32_t nb = nbr[c * 6 + f];
          if (nb >= 0) {
            const T *un = src + int64_t(nb) * N3;
            const T vn = un[face_node<N>(d, nb_layer, a, bb)];
            T dnn = T(0);
#pragma unroll
            for (int i = 0; i < N; ++i) dnn += dphi_nb[i] * un[face_node<N>(d, i, a, bb)];
            dnn *= sgn_h;
            const T jump = vo - vn;
            f1 = sigma * jump - T(0.5) * (dn + dnn);
            f2 = T(-0.5) * jump;
          } else if (bc_dirichlet) { // mirror: u+ = -u-, d_n u+ = d_n u-
            f1 = sigma * T(2) * vo - dn;
            f2 = -vo;
          }
        }
        F1[b][ab] = f1 * area;
        F2[b][ab] = f2 * area;
      }
      __syncthreads();
      // face mass along a, then along b
      if (t < B * N2) {
        const int b = t / N2, ab = t - b * N2, a = ab % N, bb = ab / N;
        T g1 = T(0), g2 = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          g1 += tab.M1[a * N + k] * F1[b][bb * N + k];
          g2 += tab.M1[a * N + k] * F2[b][bb * N + k];
        }
        G1[b][ab] = g1;
        G2[b][ab] = g2;
      }
      __syncthreads();
      if (t < B * N2) {
        const int b = t / N2, ab = t - b * N2, a = ab % N, bb = ab / N;
        T tv = T(0), tn = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          tv += tab.M1[bb * N + k] * G1[b][k * N + a];
          tn += tab.M1[bb * N + k] * G2[b][k * N + a];
        }
        // value test on the face layer, normal-derivative test on every layer along d
        out[b][face_node<N>(d, own_layer, a, bb)] += tv;
        tn *= sgn_h;
#pragma unroll
        for (int i = 0; i < N; ++i) out[b][face_node<N>(d, i, a, bb)] += tn * dphi_own[i];
      }
      __syncthreads();
    }
    for (int e = t; e < B * N3; e += blockDim.x) {
      const int b = e / N3, l = e - b * N3;
      const int64_t c = base + b;
      if (c < n_cells) dst[c * N3 + l] += out[b][l];
    }
    __syncthreads();
  }
}

// face self terms of the diagonal: a node on the face layer of face (d, s) with
// g = phi'(s) (+-1)/h gets m (sigma - g) (inner) or m (2 sigma - 2 g) (Dirichlet),
// m = h_a h_b M1[a][a] M1[b][b]
template <int N, typename T>
__global__ void dg_face_diag_kernel(const DGTab<N, T> tab, const DGGeo geo, T *__restrict__ diag,
                                    const int32_t *__restrict__ nbr, int64_t n_cells) {
  constexpr int N3 = N * N * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_cells * N3;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / N3;
    const int l = int(e - c * N3);
    const int idx[3] = {l % N, (l / N) % N, l / (N * N)};
    T add = T(0);
    for (int f = 0; f < 6; ++f) {
      const int d = f >> 1, s = f & 1;
      if (idx[d] != (s ? N - 1 : 0)) continue;
      const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
      const int32_t nb = nbr[c * 6 + f];
      const bool dir = (geo.dirichlet >> f) & 1;
      if (nb < 0 && !dir) continue;
      const T sigma = (T)(geo.c_pen / geo.h[d]);
      const T g = (s ? tab.dphi1[N - 1] : -tab.dphi0[0]) / (T)geo.h[d];
      const T m = (T)(geo.h[ta] * geo.h[tb]) * tab.M1[idx[ta] * N + idx[ta]] * tab.M1[idx[tb] * N + idx[tb]];
      add += nb >= 0 ? m * (sigma - g) : T(2) * m * (sigma - g);
    }
    diag[e] += add;
  }
}

template <typename T> __global__ void add_kernel(T *__restrict__ dst, const double *__restrict__ src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] += (T)src[i];
}

// ---- each face once: 4x4x4 tiles of cells ----
// With the box refined at least twice, every 64 consecutive cells (Morton order inside a
// coarse cell) form a 4x4x4 cube.  A block loads such a tile into shared memory (one
// coalesced read), evaluates every face between two tile cells once (144 faces: the flux
// from the lower cell's side, its face mass, then the value and normal-derivative tests of
// both cells, the upper cell's with the signs of its own outward normal) and every face on
// the tile's surface from the inside (96 faces: the neighbour's normal line from global
// memory, or the Dirichlet mirror).  Then one thread per tile node sums what its six faces
// give it, in a fixed order (no atomics, so the result does not depend on scheduling), and
// adds that to dst in one coalesced pass.  The faces of the tile surface are still met from
// both sides.
//
// Faces are numbered by direction d: 80 d + f, f < 48 inside the tile (f = 16 x along + the
// tangential position), 48 <= f < 64 on the lower and 64 <= f < 80 on the upper surface.  A
// face point is (a, b), a along the first and b along the second tangential axis; the flux
// of face point t = (80 d + f) N^2 + b N + a is evaluated with d known at compile time.
// Where a face's N^2 points divide a warp (N = 2, 4) they lie in one warp, and the face mass
// M1 x M1 is applied with shuffles, without shared memory or block barriers.
constexpr int kTileFaces = 240;
constexpr int kDirFaces = 80;
template <int N> constexpr int tile_cell_stride() { return N * N * N + 1; } // padded: fewer bank conflicts
template <int N> constexpr bool tile_shuffles() { return 32 % (N * N) == 0; }
template <int N, typename T> constexpr size_t dg_tile_region() {
  // the tile's values; without shuffles also the face-mass arrays G1, G2 over them
  return tile_shuffles<N>() || size_t(64) * tile_cell_stride<N>() > size_t(2) * kTileFaces * N * N
             ? size_t(64) * tile_cell_stride<N>()
             : size_t(2) * kTileFaces * N * N;
}
// shared memory of the tile kernel: the node-face table (64 x 6 ints), the face-point arrays
// F1, F2, then the tile region
template <int N, typename T> constexpr size_t dg_tile_smem() {
  return sizeof(int) * 384 + sizeof(T) * (size_t(2) * kTileFaces * N * N + dg_tile_region<N, T>());
}

__device__ __forceinline__ int tile_index(int x, int y, int z) {
  return (x & 1) | ((y & 1) << 1) | ((z & 1) << 2) | ((x >> 1) << 3) | ((y >> 1) << 4) | ((z >> 1) << 5);
}

// flux values (times the face area) of face f of direction D at face point (a, bb): f1 =
// sigma [u] - {d_n u}, f2 = -[u]/2 with the normal +D inside the tile, the inside cell's
// outward normal on the surface (Dirichlet: mirror u+ = -u-, d_n u+ = d_n u-)
// face_node in a tile layout whose z planes are PZ entries apart
template <int N, int PZ> __device__ __forceinline__ int face_node_t(int d, int layer, int a, int b) {
  const int i = d == 0 ? layer : a;
  const int j = d == 1 ? layer : (d == 0 ? a : b);
  const int k = d == 2 ? layer : b;
  return k * PZ + j * N + i;
}

// (the tile in shared memory: cell stride CS, z planes PZ apart; src in memory: N^3 per cell)
template <int N, typename T, int D, int CS = tile_cell_stride<N>(), int PZ = N * N>
__device__ __forceinline__ void tile_flux(const DGTab<N, T> &tab, const DGGeo &geo, const T *__restrict__ U,
                                          const T *__restrict__ src, const int32_t *__restrict__ nbr,
                                          int64_t base, int f, int a, int bb, T &f1, T &f2) {
  constexpr int N3 = N * N * N;
  constexpr int ta = D == 0 ? 1 : 0, tb = D == 2 ? 1 : 2;
  const T h = (T)geo.h[D], area = (T)(geo.h[ta] * geo.h[tb]), sigma = (T)(geo.c_pen / geo.h[D]);
  int c[3];
  f1 = T(0);
  f2 = T(0);
  if (f < 48) {
    const int along = f >> 4, tan = f & 15;
    c[D] = along;
    c[ta] = tan & 3;
    c[tb] = tan >> 2;
    const T *ul = U + tile_index(c[0], c[1], c[2]) * CS;
    c[D] = along + 1;
    const T *uu = U + tile_index(c[0], c[1], c[2]) * CS;
    T dn = T(0), dnn = T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const int l = face_node_t<N, PZ>(D, i, a, bb);
      dn += tab.dphi1[i] * ul[l];
      dnn += tab.dphi0[i] * uu[l];
    }
    const T jump = ul[face_node_t<N, PZ>(D, N - 1, a, bb)] - uu[face_node_t<N, PZ>(D, 0, a, bb)];
    f1 = sigma * jump - T(0.5) * (dn + dnn) / h;
    f2 = T(-0.5) * jump;
  } else {
    const int sd = (f - 48) >> 4, tan = (f - 48) & 15, F = 2 * D + sd;
    c[D] = sd ? 3 : 0;
    c[ta] = tan & 3;
    c[tb] = tan >> 2;
    const int in = tile_index(c[0], c[1], c[2]);
    const T *uo = U + in * CS;
    const T sgn_h = (sd ? T(1) : T(-1)) / h;
    T dn = T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) dn += (sd ? tab.dphi1[i] : tab.dphi0[i]) * uo[face_node_t<N, PZ>(D, i, a, bb)];
    dn *= sgn_h;
    const T vo = sd ? uo[face_node_t<N, PZ>(D, N - 1, a, bb)] : uo[face_node_t<N, PZ>(D, 0, a, bb)];
    const int32_t nb = __ldg(nbr + (base + in) * 6 + F);
    if (nb >= 0) {
      const T *un = src + int64_t(nb) * N3;
      T dnn = T(0);
#pragma unroll
      for (int i = 0; i < N; ++i) dnn += (sd ? tab.dphi0[i] : tab.dphi1[i]) * __ldg(un + face_node<N>(D, i, a, bb));
      dnn *= sgn_h;
      const T vn = sd ? __ldg(un + face_node<N>(D, 0, a, bb)) : __ldg(un + face_node<N>(D, N - 1, a, bb));
      const T jump = vo - vn;
      f1 = sigma * jump - T(0.5) * (dn + dnn);
      f2 = T(-0.5) * jump;
    } else if ((geo.dirichlet >> F) & 1) {
      f1 = sigma * T(2) * vo - dn;
      f2 = -vo;
    }
  }
  f1 *= area;
  f2 *= area;
}

// node-face table: face f of direction d seen from tile cell ct as its upper (+d) face (ct
// the lower cell of an inside face), its lower face (ct the upper cell) or a surface face;
// entry 2 x (first face point) + 1 for the upper cell of an inside face
template <int N, int TT> __device__ __forceinline__ void fill_node_faces(int *NF) {
  constexpr int N2 = N * N;
  for (int e = threadIdx.x; e < 384; e += TT) {
    const int ct = e / 6, F = e - ct * 6, d = F >> 1, sd = F & 1;
    const int cc[3] = {(ct & 1) | (((ct >> 3) & 1) << 1), ((ct >> 1) & 1) | (((ct >> 4) & 1) << 1),
                       ((ct >> 2) & 1) | (((ct >> 5) & 1) << 1)};
    const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
    const int tan = cc[ta] + 4 * cc[tb];
    int f, up = 0;
    if (sd && cc[d] < 3) {
      f = 16 * cc[d] + tan;
    } else if (!sd && cc[d] > 0) {
      f = 16 * (cc[d] - 1) + tan;
      up = 1;
    } else {
      f = 48 + 16 * sd + tan;
    }
    NF[e] = 2 * ((kDirFaces * d + f) * N2) + up;
  }
}

// phase 1 of the tile kernels with the face mass on shuffles (N^2 divides 32): the fluxes of
// face point t, then M1 x M1 over the face's N^2 lanes; F1 = the value-test coefficient, F2 =
// the normal-derivative-test coefficient divided by h (on the lower surface times -1)
template <int N, typename T, int CS = tile_cell_stride<N>(), int PZ = N * N>
__device__ __forceinline__ void tile_face_point_shfl(const DGTab<N, T> &tab, const DGTab<N, T> &st, const DGGeo &geo,
                                                     const T *__restrict__ U, const T *__restrict__ src,
                                                     const int32_t *__restrict__ nbr, int64_t base, int t, T *F1,
                                                     T *F2) {
  constexpr int N2 = N * N, DP = kDirFaces * N2;
  const int d = t / DP, r = t - d * DP, f = r / N2, ab = r - f * N2, a = ab % N, bb = ab / N;
  T f1, f2;
  if (d == 0) tile_flux<N, T, 0, CS, PZ>(tab, geo, U, src, nbr, base, f, a, bb, f1, f2);
  else if (d == 1) tile_flux<N, T, 1, CS, PZ>(tab, geo, U, src, nbr, base, f, a, bb, f1, f2);
  else tile_flux<N, T, 2, CS, PZ>(tab, geo, U, src, nbr, base, f, a, bb, f1, f2);
  const int lane0 = (threadIdx.x & 31) - ab; // the face's first lane
  T g1 = T(0), g2 = T(0);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const T x1 = __shfl_sync(0xffffffffu, f1, lane0 + bb * N + k);
    const T x2 = __shfl_sync(0xffffffffu, f2, lane0 + bb * N + k);
    g1 += st.M1[a * N + k] * x1;
    g2 += st.M1[a * N + k] * x2;
  }
  T tv = T(0), tn = T(0);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const T y1 = __shfl_sync(0xffffffffu, g1, lane0 + k * N + a);
    const T y2 = __shfl_sync(0xffffffffu, g2, lane0 + k * N + a);
    tv += st.M1[bb * N + k] * y1;
    tn += st.M1[bb * N + k] * y2;
  }
  const T sg = (f >= 48 && f < 64) ? T(-1) : T(1);
  F1[t] = tv;
  F2[t] = tn * sg / (T)geo.h[d];
}

// phase 4 of the tile kernels for node e of the tile: the sum of its six faces' tests in a
// fixed order (the value test on the face layer, minus for the upper cell of an inside face,
// and the normal-derivative test on every layer)
template <int N, typename T>
__device__ __forceinline__ T tile_node_faces(const DGTab<N, T> &st, const int *__restrict__ NF, const T *F1,
                                             const T *F2, int ct, int l) {
  constexpr int N2 = N * N;
  const int idx[3] = {l % N, (l / N) % N, l / N2};
  const int *nf = NF + ct * 6;
  T v = T(0);
#pragma unroll
  for (int F = 0; F < 6; ++F) {
    const int d = F >> 1, sd = F & 1;
    const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
    const int x = nf[F];
    const int pab = (x >> 1) + idx[tb] * N + idx[ta];
    v += F2[pab] * (sd ? st.dphi1[idx[d]] : st.dphi0[idx[d]]);
    if (idx[d] == (sd ? N - 1 : 0)) v += (x & 1) ? -F1[pab] : F1[pab];
  }
  return v;
}

template <int N, typename T, int TT>
__global__ void __launch_bounds__(TT, 1024 / TT) dg_face_tile_kernel(const __grid_constant__ DGTab<N, T> tab,
                                                                    const __grid_constant__ DGGeo geo,
                                                                    const T *__restrict__ src, T *__restrict__ dst,
                                                                    const int32_t *__restrict__ nbr, int64_t n_tiles) {
  constexpr int N2 = N * N, N3 = N2 * N, CS = tile_cell_stride<N>(), NP = kTileFaces * N2, DP = kDirFaces * N2;
  constexpr bool SHFL = tile_shuffles<N>();
  extern __shared__ __align__(16) unsigned char dg_tile_raw[];
  int *NF = reinterpret_cast<int *>(dg_tile_raw); // [tile cell][face]: 2 x first face point + upper
  T *F1 = reinterpret_cast<T *>(dg_tile_raw + sizeof(int) * 384), *F2 = F1 + NP;
  T *U = F2 + NP;                  // the tile's values, cell stride CS
  T *G1 = U, *G2 = G1 + NP;        // over them from phase 2 on (without shuffles)
  __shared__ DGTab<N, T> st;
  load_tab_shared(st, tab);
  fill_node_faces<N, TT>(NF);
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t base = tile * 64;
    const T *ts = src + base * N3;
    for (int e = threadIdx.x; e < 64 * N3; e += TT) {
      const int ct = e / N3;
      U[ct * CS + (e - ct * N3)] = ts[e];
    }
    __syncthreads();
    // 1. fluxes at every face point; with shuffles also the face mass (2., 3.): a face's N^2
    //    points are N^2 consecutive lanes of one warp (NP is a multiple of 32, so every lane
    //    of a warp takes part)
    for (int t = threadIdx.x; t < NP; t += TT) {
      if constexpr (SHFL) {
        tile_face_point_shfl<N, T>(tab, st, geo, U, src, nbr, base, t, F1, F2);
      } else {
        const int d = t / DP, r = t - d * DP, f = r / N2, ab = r - f * N2, a = ab % N, bb = ab / N;
        T f1, f2;
        if (d == 0) tile_flux<N, T, 0>(tab, geo, U, src, nbr, base, f, a, bb, f1, f2);
        else if (d == 1) tile_flux<N, T, 1>(tab, geo, U, src, nbr, base, f, a, bb, f1, f2);
        else tile_flux<N, T, 2>(tab, geo, U, src, nbr, base, f, a, bb, f1, f2);
        F1[t] = f1;
        F2[t] = f2;
      }
    }
    __syncthreads();
    if constexpr (!SHFL) {
      // 2. face mass along a
      for (int t = threadIdx.x; t < NP; t += TT) {
        const int fi = t / N2, ab = t - fi * N2, a = ab % N, bb = ab / N;
        const T *f1 = F1 + fi * N2 + bb * N, *f2 = F2 + fi * N2 + bb * N;
        T g1 = T(0), g2 = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          g1 += st.M1[a * N + k] * f1[k];
          g2 += st.M1[a * N + k] * f2[k];
        }
        G1[t] = g1;
        G2[t] = g2;
      }
      __syncthreads();
      // 3. face mass along b: the value-test coefficient (F1) and the normal-derivative-test
      //    coefficient (F2, divided by h; on the lower surface times -1)
      for (int t = threadIdx.x; t < NP; t += TT) {
        const int fi = t / N2, ab = t - fi * N2, a = ab % N, bb = ab / N;
        const T *g1 = G1 + fi * N2 + a, *g2 = G2 + fi * N2 + a;
        T tv = T(0), tn = T(0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          tv += st.M1[bb * N + k] * g1[k * N];
          tn += st.M1[bb * N + k] * g2[k * N];
        }
        const int d = fi / kDirFaces, f = fi - d * kDirFaces;
        const T sg = (f >= 48 && f < 64) ? T(-1) : T(1);
        F1[t] = tv;
        F2[t] = tn * sg / (T)geo.h[d];
      }
      __syncthreads();
    }
    // 4. one thread per tile node sums its six faces in a fixed order (deterministic): the
    //    value test on the face layer (minus for the upper cell of an inside face, whose
    //    outward normal is opposite to the one the face was evaluated with) and the
    //    normal-derivative test on every layer, then adds the sum to dst
    T *td = dst + base * N3;
    for (int e = threadIdx.x; e < 64 * N3; e += TT) {
      const int ct = e / N3, l = e - ct * N3;
      const T v = tile_node_faces<N, T>(st, NF, F1, F2, ct, l);
      td[e] += v;
    }
    __syncthreads();
  }
}

// The whole DG vmult on a tile (N = 2, 4: the face mass on shuffles): the cell stiffness term
// of axis-aligned cells, A_K u = cx (K1 x M1 x M1) u + (M1 x (cy K1 x M1 + cz M1 x K1)) u with
// cx = hy hz / hx, cy = hx hz / hy, cz = hx hy / hz (K1, M1 the 1D stiffness and mass
// matrices on the reference interval, x acting on the first index), by three passes over the
// tile in shared memory (z by lines into A and B, y by lines in place, x by nodes into the tile
// array once the faces have read it), and the face terms as in dg_face_tile_kernel; phase 4
// stores cell plus face terms: src is read once, dst written once, no index map, no zeroing.
// Shared-memory layout of a cell in the fused kernel: node (i, j, k) at k PZ + j N + i, cell
// stride CS.  At N = 4 each z plane is padded to 20 entries and the cell to 80: in FP32 the two
// cells a warp covers in a line pass then fall on the two halves of the 32 banks, and in both
// types the 16 lines of a y pass (planes 20 apart) on distinct banks.  At N = 2 planes of
// N^2 and a cell stride of N^3 + 1.
template <int N, typename T> struct FusedLayout {
  static constexpr bool PAD = N == 4;
  static constexpr int PZ = PAD ? N * N + 4 : N * N;
  static constexpr int CS = PAD ? N * PZ : N * N * N + 1;
};
template <int N, typename T> constexpr size_t dg_fused_smem() {
  return sizeof(int) * 384 + sizeof(T) * (size_t(2) * kTileFaces * N * N + size_t(3) * 64 * FusedLayout<N, T>::CS);
}

// the fluxes of face f of direction D at this thread's face point, whose node offsets within
// a cell are fb + i * stride(D) in the tile's layout (cell stride CS, z planes PZ apart) and
// fbg + i * stride(D) in memory (fb, fbg = the point's node on layer 0); as tile_flux
template <int N, typename T, int D, int CS, int PZ>
__device__ __forceinline__ void tile_flux_at(const DGTab<N, T> &tab, const DGGeo &geo, const T *__restrict__ U,
                                             const T *__restrict__ src, const int32_t *__restrict__ nbr, int64_t base,
                                             int f, int tan_f, int fb, int fbg, T &f1, T &f2) {
  constexpr int N3 = N * N * N, SD = D == 0 ? 1 : (D == 1 ? N : PZ), SG = D == 0 ? 1 : (D == 1 ? N : N * N);
  // tile cell (x, y, z) -> index: bit interleaving (tile_index); `tan_f` is the face's
  // tangential cell position (c_ta + 4 c_tb) and f its along position / surface side
  constexpr int ta = D == 0 ? 1 : 0, tb = D == 2 ? 1 : 2;
  const T h = (T)geo.h[D], area = (T)(geo.h[ta] * geo.h[tb]), sigma = (T)(geo.c_pen / geo.h[D]);
  int c[3];
  c[ta] = tan_f & 3;
  c[tb] = tan_f >> 2;
  f1 = T(0);
  f2 = T(0);
  if (f < 48) {
    c[D] = f >> 4;
    const T *ul = U + tile_index(c[0], c[1], c[2]) * CS + fb;
    c[D] += 1;
    const T *uu = U + tile_index(c[0], c[1], c[2]) * CS + fb;
    T dn = T(0), dnn = T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      dn += tab.dphi1[i] * ul[i * SD];
      dnn += tab.dphi0[i] * uu[i * SD];
    }
    const T jump = ul[(N - 1) * SD] - uu[0];
    f1 = sigma * jump - T(0.5) * (dn + dnn) / h;
    f2 = T(-0.5) * jump;
  } else {
    const int sd = f >= 64, F = 2 * D + sd;
    c[D] = sd ? 3 : 0;
    const int in = tile_index(c[0], c[1], c[2]);
    const T *uo = U + in * CS + fb;
    const T sgn_h = (sd ? T(1) : T(-1)) / h;
    T dn = T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) dn += (sd ? tab.dphi1[i] : tab.dphi0[i]) * uo[i * SD];
    dn *= sgn_h;
    const T vo = sd ? uo[(N - 1) * SD] : uo[0];
    const int32_t nb = __ldg(nbr + (base + in) * 6 + F);
    if (nb >= 0) {
      const T *un = src + int64_t(nb) * N3 + fbg;
      T dnn = T(0), line[N];
#pragma unroll
      for (int i = 0; i < N; ++i) line[i] = __ldg(un + i * SG);
#pragma unroll
      for (int i = 0; i < N; ++i) dnn += (sd ? tab.dphi0[i] : tab.dphi1[i]) * line[i];
      dnn *= sgn_h;
      const T jump = vo - (sd ? line[0] : line[N - 1]);
      f1 = sigma * jump - T(0.5) * (dn + dnn);
      f2 = T(-0.5) * jump;
    } else if ((geo.dirichlet >> F) & 1) {
      f1 = sigma * T(2) * vo - dn;
      f2 = -vo;
    }
  }
  f1 *= area;
  f2 *= area;
}

// the Chebyshev step the fused kernel can apply in place of storing A x (CHEB):
// out = x + f1 (x - x_prev) + f2 D^{-1} (b - A x), x = src; prev null: x_prev = 0
template <typename T> struct ChebArgs {
  const T *prev, *b, *invd;
  T f1, f2;
};

template <int N, typename T, int TT, bool CHEB = false>
__global__ void __launch_bounds__(TT, 1024 / TT) dg_tile_fused_kernel(const __grid_constant__ DGTab<N, T> tab,
                                                                     const __grid_constant__ DGGeo geo,
                                                                     const T *__restrict__ src, T *__restrict__ dst,
                                                                     const int32_t *__restrict__ nbr, int64_t n_tiles,
                                                                     ChebArgs<T> cheb = ChebArgs<T>{}) {
  static_assert(tile_shuffles<N>(), "the fused tile kernel applies the face mass on shuffles");
  constexpr int N2 = N * N, N3 = N2 * N, NP = kTileFaces * N2;
  constexpr int CS = FusedLayout<N, T>::CS, PZ = FusedLayout<N, T>::PZ; // cell stride, z-plane stride
  // the block size is a multiple of N^3: every thread keeps one node position (l) in the node
  // passes and one line position (r) in the line passes, for cells ct0 + k * (TT / N^3) and
  // ct1 + k * (TT / N^2), so the index arithmetic and the table rows of its position are
  // computed once
  static_assert(TT % N3 == 0, "block size");
  constexpr int CN = TT / N3, CL = TT / N2;                  // cells per sweep of a pass
  constexpr int QN = (64 + CN - 1) / CN, QL = (64 + CL - 1) / CL; // sweeps (the last may be partial)
  // a warp's lanes take 32 / N^2 consecutive faces, and 240 is a multiple of that: the bound
  // of the face loop is the same for every lane of a warp, so its shuffles see full warps
  static_assert(kTileFaces % (32 / N2) == 0, "warp-uniform face loop");
  constexpr int QF = (kTileFaces + CL - 1) / CL;
  extern __shared__ __align__(16) unsigned char dg_tile_raw[];
  int *NF = reinterpret_cast<int *>(dg_tile_raw);
  T *F1 = reinterpret_cast<T *>(dg_tile_raw + sizeof(int) * 384), *F2 = F1 + NP;
  T *U = F2 + NP;       // the tile's values, then the cell term
  T *A = U + 64 * CS;   // z pass M1 u, then the y pass P = M1 M1 u
  T *B = A + 64 * CS;   // z pass K1 u, then the y pass S = cy K1 M1 u + cz M1 K1 u
  __shared__ DGTab<N, T> st;
  load_tab_shared(st, tab);
  fill_node_faces<N, TT>(NF);
  const T cx = (T)(geo.h[1] * geo.h[2] / geo.h[0]), cy = (T)(geo.h[0] * geo.h[2] / geo.h[1]),
          cz = (T)(geo.h[0] * geo.h[1] / geo.h[2]);
  // this thread's node position l = (iz N + iy) N + ix and line position r
  const int l = threadIdx.x % N3, ct0 = threadIdx.x / N3;
  const int r = threadIdx.x % N2, ct1 = threadIdx.x / N2;
  const int idx[3] = {l % N, (l / N) % N, l / N2};
  const int sl = idx[2] * PZ + idx[1] * N + idx[0]; // the node's place in the tile layout
  // this thread's face point (a, b) = (r mod N, r / N) in every face it evaluates: the
  // face's first lane and the layer-0 node of the point per direction
  const int fa = r % N, fbb = r / N, lane0 = (threadIdx.x & 31) - r;
  // layer-0 node of the face point: in memory (k N^2 + j N + i) and in the tile layout
  const int fg0 = face_node<N>(0, 0, fa, fbb), fg1 = face_node<N>(1, 0, fa, fbb), fg2 = face_node<N>(2, 0, fa, fbb);
  auto tile_off = [](int g) { return (g / (N * N)) * PZ + g % (N * N); };
  const int fb0 = tile_off(fg0), fb1 = tile_off(fg1), fb2 = tile_off(fg2);
  // the table rows of its positions (x-pass rows of K1 and M1, face-mass rows of a and b, the
  // node's normal-derivative tests) held in registers in FP32; in FP64 they would exceed
  // the 64 registers a thread has and are read from shared memory instead
  constexpr bool HOLD = sizeof(T) == 4;
  constexpr int HN = HOLD ? N : 1, H6 = HOLD ? 6 : 1;
  T kx[HN], mx[HN], ma[HN], mb[HN], dph[H6];
  int off[6];      // the node's face point within each of its six faces
  bool lay[6];     // the node lies on the face layer
#pragma unroll
  for (int F = 0; F < 6; ++F) {
    const int d = F >> 1, sd = F & 1;
    const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
    off[F] = idx[tb] * N + idx[ta];
    lay[F] = idx[d] == (sd ? N - 1 : 0);
  }
  if constexpr (HOLD) {
#pragma unroll
    for (int m = 0; m < N; ++m) {
      kx[m] = tab.K1[idx[0] * N + m];
      mx[m] = tab.M1[idx[0] * N + m];
      ma[m] = tab.M1[fa * N + m];
      mb[m] = tab.M1[fbb * N + m];
    }
#pragma unroll
    for (int F = 0; F < 6; ++F) {
      const int d = F >> 1;
      dph[F] = (F & 1) ? tab.dphi1[idx[d]] : tab.dphi0[idx[d]];
    }
  }
  auto KX = [&](int m) { if constexpr (HOLD) return kx[m]; else return st.K1[idx[0] * N + m]; };
  auto MX = [&](int m) { if constexpr (HOLD) return mx[m]; else return st.M1[idx[0] * N + m]; };
  auto MA = [&](int m) { if constexpr (HOLD) return ma[m]; else return st.M1[fa * N + m]; };
  auto MB = [&](int m) { if constexpr (HOLD) return mb[m]; else return st.M1[fbb * N + m]; };
  auto DPH = [&](int F) {
    if constexpr (HOLD) return dph[F];
    else return (F & 1) ? st.dphi1[idx[F >> 1]] : st.dphi0[idx[F >> 1]];
  };
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t base = tile * 64;
    const T *ts = src + base * N3;
#pragma unroll
    for (int k = 0; k < QN; ++k) {
      const int ct = ct0 + k * CN;
      if (ct < 64) U[ct * CS + sl] = ts[ct * N3 + l];
    }
    __syncthreads();
    // cell term, z pass: line r = j N + i of each cell
#pragma unroll
    for (int q = 0; q < QL; ++q) {
      if (ct1 + q * CL >= 64) break;
      const int o = (ct1 + q * CL) * CS + r;
      T v[N];
#pragma unroll
      for (int k = 0; k < N; ++k) v[k] = U[o + k * PZ];
#pragma unroll
      for (int k = 0; k < N; ++k) {
        T sa = T(0), sb = T(0);
#pragma unroll
        for (int m = 0; m < N; ++m) {
          sa += tab.M1[k * N + m] * v[m];
          sb += tab.K1[k * N + m] * v[m];
        }
        A[o + k * PZ] = sa;
        B[o + k * PZ] = sb;
      }
    }
    // face fluxes and face mass (phases 1-3 of the tile kernel): faces ct1 + q * CL, each on
    // N^2 consecutive lanes of one warp; FP64 takes the generic loop (the unrolled one
    // exceeds its registers)
    if constexpr (!HOLD) {
      for (int t = threadIdx.x; t < NP; t += TT)
        tile_face_point_shfl<N, T, CS, PZ>(tab, st, geo, U, src, nbr, base, t, F1, F2);
    } else
#pragma unroll
    for (int q = 0; q < QF; ++q) {
      const int fi = ct1 + q * CL; // face 80 d + f
      if (fi >= kTileFaces) break; // warp-uniform
      T f1, f2;
      if (fi < kDirFaces) {
        tile_flux_at<N, T, 0, CS, PZ>(tab, geo, U, src, nbr, base, fi, fi < 48 ? fi & 15 : (fi - 48) & 15, fb0, fg0,
                                      f1, f2);
      } else if (fi < 2 * kDirFaces) {
        const int f = fi - kDirFaces;
        tile_flux_at<N, T, 1, CS, PZ>(tab, geo, U, src, nbr, base, f, f < 48 ? f & 15 : (f - 48) & 15, fb1, fg1, f1,
                                      f2);
      } else {
        const int f = fi - 2 * kDirFaces;
        tile_flux_at<N, T, 2, CS, PZ>(tab, geo, U, src, nbr, base, f, f < 48 ? f & 15 : (f - 48) & 15, fb2, fg2, f1,
                                      f2);
      }
      T g1 = T(0), g2 = T(0);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        g1 += MA(k) * __shfl_sync(0xffffffffu, f1, lane0 + fbb * N + k);
        g2 += MA(k) * __shfl_sync(0xffffffffu, f2, lane0 + fbb * N + k);
      }
      T tv = T(0), tn = T(0);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        tv += MB(k) * __shfl_sync(0xffffffffu, g1, lane0 + k * N + fa);
        tn += MB(k) * __shfl_sync(0xffffffffu, g2, lane0 + k * N + fa);
      }
      const int d = fi / kDirFaces, f = fi - d * kDirFaces;
      const T sg = (f >= 48 && f < 64) ? T(-1) : T(1);
      F1[fi * N2 + r] = tv;
      F2[fi * N2 + r] = tn * sg / (T)geo.h[d];
    }
    __syncthreads();
    // cell term, y pass in place: line r = k N + i of each cell
#pragma unroll
    for (int q = 0; q < QL; ++q) {
      if (ct1 + q * CL >= 64) break;
      const int o = (ct1 + q * CL) * CS + (r / N) * PZ + (r % N);
      T av[N], bv[N];
#pragma unroll
      for (int j = 0; j < N; ++j) {
        av[j] = A[o + j * N];
        bv[j] = B[o + j * N];
      }
#pragma unroll
      for (int j = 0; j < N; ++j) {
        T pp = T(0), qa = T(0), qb = T(0);
#pragma unroll
        for (int m = 0; m < N; ++m) {
          pp += tab.M1[j * N + m] * av[m];
          qa += tab.K1[j * N + m] * av[m];
          qb += tab.M1[j * N + m] * bv[m];
        }
        A[o + j * N] = pp;
        B[o + j * N] = cy * qa + cz * qb;
      }
    }
    __syncthreads();
    // cell term, x pass: this thread's node of each cell, into the tile array (read by now)
#pragma unroll
    for (int k = 0; k < QN; ++k) {
      if (ct0 + k * CN >= 64) break;
      const int row = (ct0 + k * CN) * CS + (sl - idx[0]);
      T c = T(0), d = T(0);
#pragma unroll
      for (int m = 0; m < N; ++m) {
        c += KX(m) * A[row + m];
        d += MX(m) * B[row + m];
      }
      U[row + idx[0]] = cx * c + d;
    }
    __syncthreads();
    // cell plus face terms into dst, the six faces in a fixed order
    T *td = dst + base * N3;
#pragma unroll
    for (int k = 0; k < QN; ++k) {
      const int ct = ct0 + k * CN;
      if (ct >= 64) break;
      const int *nf = NF + ct * 6;
      T v = U[ct * CS + sl];
#pragma unroll
      for (int F = 0; F < 6; ++F) {
        const int x = nf[F];
        const int pab = (x >> 1) + off[F];
        v += F2[pab] * DPH(F);
        if (lay[F]) v += (x & 1) ? -F1[pab] : F1[pab];
      }
      if constexpr (CHEB) {
        // the Chebyshev step of vector_ops (cheb_update_into) with A x from registers; out
        // (dst) may be prev, whose entry only this thread reads, never src, which the
        // neighbouring tiles read
        const int64_t gi = (base + ct) * N3 + l;
        const T xv = ts[ct * N3 + l];
        const T xo = cheb.prev ? cheb.prev[gi] : T(0);
        dst[gi] = xv + cheb.f1 * (xv - xo) + cheb.f2 * cheb.invd[gi] * (cheb.b[gi] - v);
      } else {
        td[ct * N3 + l] = v;
      }
    }
    __syncthreads();
  }
}

// the face form: PMG_DG_FACE=0 the face-by-face kernel, 1 the cell-batch kernel, 2 the tile
// kernel wherever the mesh allows it (comparison switches, read at every launch); unset: the
// tile kernel where the mesh allows it and the tiles fill the device at least twice, else the
// cell-batch kernel
int face_form() {
  const char *e = std::getenv("PMG_DG_FACE");
  if (e && (e[0] == '0' || e[0] == '1' || e[0] == '2') && e[1] == 0) return e[0] - '0';
  return -1;
}

// block size of a tile kernel on the current device: 256, 512 or 1024 threads, whichever keeps
// the most threads per SM resident (their shared memory allows few blocks per SM)
struct TileShape {
  int threads = 256, blocks_per_sm = 1;
};
template <int N, typename T, bool FUSED> TileShape tile_shape() {
  static std::mutex mu;
  static std::map<int, TileShape> cache; // device -> shape
  int dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  constexpr size_t smem = FUSED ? dg_fused_smem<N, T>() : dg_tile_smem<N, T>();
  TileShape best;
  int best_threads = 0;
  auto probe = [&](auto k, int tt) {
    PMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, tt, smem));
    if (nb * tt > best_threads) {
      best_threads = nb * tt;
      best.threads = tt;
      best.blocks_per_sm = std::max(1, nb);
    }
  };
  if constexpr (FUSED) {
    if constexpr (tile_shuffles<N>()) {
      probe(dg_tile_fused_kernel<N, T, 256>, 256);
      probe(dg_tile_fused_kernel<N, T, 512>, 512);
      probe(dg_tile_fused_kernel<N, T, 1024>, 1024);
      // the Chebyshev-step variants take the same shape; they need the same shared memory
      PMG_CUDA(cudaFuncSetAttribute(dg_tile_fused_kernel<N, T, 256, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PMG_CUDA(cudaFuncSetAttribute(dg_tile_fused_kernel<N, T, 512, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PMG_CUDA(cudaFuncSetAttribute(dg_tile_fused_kernel<N, T, 1024, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
  } else {
    probe(dg_face_tile_kernel<N, T, 256>, 256);
    probe(dg_face_tile_kernel<N, T, 512>, 512);
    probe(dg_face_tile_kernel<N, T, 1024>, 1024);
  }
  cache.emplace(dev, best);
  return best;
}

template <int N, typename T> DGTab<N, T> make_dg_tab(const DGHost &h) {
  DGTab<N, T> t;
  for (int a = 0; a < N * N; ++a) {
    t.M1[a] = (T)h.M1[a];
    t.K1[a] = (T)h.K1[a];
  }
  for (int a = 0; a < N; ++a) {
    t.dphi0[a] = (T)h.dphi0[a];
    t.dphi1[a] = (T)h.dphi1[a];
  }
  return t;
}

DGGeo make_geo(const DGHost &h) {
  DGGeo g;
  for (int d = 0; d < 3; ++d) g.h[d] = h.h[d];
  g.c_pen = h.c_pen;
  g.dirichlet = h.dirichlet;
  return g;
}

template <int N, typename T>
void face_launch(const DGHost &h, const void *src, void *dst, int64_t n_cells, int sms, cudaStream_t s,
                 bool diag, int64_t *units, int64_t *blocks) {
  if (diag) {
    const int grid = (int)std::min<int64_t>((n_cells * N * N * N + 255) / 256, (int64_t)sms * 16);
    dg_face_diag_kernel<N, T><<<std::max(grid, 1), 256, 0, s>>>(make_dg_tab<N, T>(h), make_geo(h),
                                                                  static_cast<T *>(dst), h.nbr.as<int32_t>(), n_cells);
  } else {
    constexpr size_t tile_smem = dg_tile_smem<N, T>();
    const int form = face_form();
    const int64_t n_tiles = n_cells / 64;
    bool tiles = (form == 2 || form < 0) && h.tiles64 && n_cells % 64 == 0 && tile_smem <= 200 * 1024;
    TileShape sh;
    if (tiles) {
      sh = tile_shape<N, T, false>();
      if (form < 0 && n_tiles < 2 * (int64_t)sh.blocks_per_sm * sms) tiles = false;
    }
    if (tiles) {
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, (int64_t)sh.blocks_per_sm * sms));
      if (units) *units = n_tiles;
      if (blocks) *blocks = grid;
      const auto tab = make_dg_tab<N, T>(h);
      const auto geo = make_geo(h);
      const T *sp = static_cast<const T *>(src);
      T *dp = static_cast<T *>(dst);
      const int32_t *nb = h.nbr.as<int32_t>();
      if (sh.threads == 1024)
        dg_face_tile_kernel<N, T, 1024><<<grid, 1024, tile_smem, s>>>(tab, geo, sp, dp, nb, n_tiles);
      else if (sh.threads == 512)
        dg_face_tile_kernel<N, T, 512><<<grid, 512, tile_smem, s>>>(tab, geo, sp, dp, nb, n_tiles);
      else
        dg_face_tile_kernel<N, T, 256><<<grid, 256, tile_smem, s>>>(tab, geo, sp, dp, nb, n_tiles);
    } else if (form == 0) {
      constexpr int B = dg_batch_seq<N>();
      const int grid = (int)std::min<int64_t>((n_cells + B - 1) / B, (int64_t)sms * 16);
      if (units) *units = (n_cells + B - 1) / B;
      if (blocks) *blocks = std::max(grid, 1);
      dg_face_seq_kernel<N, T><<<std::max(grid, 1), 128, 0, s>>>(make_dg_tab<N, T>(h), make_geo(h),
                                                                  static_cast<const T *>(src), static_cast<T *>(dst),
                                                                  h.nbr.as<int32_t>(), n_cells);
    } else {
      constexpr int B = dg_batch<N>();
      const int grid = (int)std::min<int64_t>((n_cells + B - 1) / B, (int64_t)sms * 8);
      if (units) *units = (n_cells + B - 1) / B;
      if (blocks) *blocks = std::max(grid, 1);
      // 16-byte loads of the x-normal lines where the rows allow them and src is aligned
      constexpr bool rows16 = (N * sizeof(T)) % 16 == 0;
      if (rows16 && reinterpret_cast<uintptr_t>(src) % 16 == 0)
        dg_face_kernel<N, T, rows16><<<std::max(grid, 1), dg_threads<N>(), 0, s>>>(
            make_dg_tab<N, T>(h), make_geo(h), static_cast<const T *>(src), static_cast<T *>(dst),
            h.nbr.as<int32_t>(), n_cells);
      else
        dg_face_kernel<N, T, false><<<std::max(grid, 1), dg_threads<N>(), 0, s>>>(
            make_dg_tab<N, T>(h), make_geo(h), static_cast<const T *>(src), static_cast<T *>(dst),
            h.nbr.as<int32_t>(), n_cells);
    }
  }
  PMG_LAUNCH_CHECK();
}

template <typename T>
void face_dispatch(int degree, const DGHost &h, const void *src, void *dst, int64_t n_cells, int sms,
                   cudaStream_t s, bool diag, int64_t *units = nullptr, int64_t *blocks = nullptr) {
  switch (degree) {
  case 1: face_launch<2, T>(h, src, dst, n_cells, sms, s, diag, units, blocks); break;
  case 2: face_launch<3, T>(h, src, dst, n_cells, sms, s, diag, units, blocks); break;
  case 3: face_launch<4, T>(h, src, dst, n_cells, sms, s, diag, units, blocks); break;
  case 4: face_launch<5, T>(h, src, dst, n_cells, sms, s, diag, units, blocks); break;
  case 5: face_launch<6, T>(h, src, dst, n_cells, sms, s, diag, units, blocks); break;
  case 6: face_launch<7, T>(h, src, dst, n_cells, sms, s, diag, units, blocks); break;
  default: fail(PMG_EINVAL, "DG degree must be in [1,6]");
  }
}

// PMG_DG_FUSE=0 turns the fused tile kernel off (a comparison switch, read at every launch)
bool fuse_allowed() {
  const char *e = std::getenv("PMG_DG_FUSE");
  return !(e && e[0] == '0' && e[1] == 0);
}

// cheb (optional): apply the Chebyshev step (dst = out) instead of storing A src
template <int N, typename T>
bool fused_launch(const DGHost &h, const void *src, void *dst, int64_t n_cells, int sms, cudaStream_t s,
                  int64_t *units, int64_t *blocks, const DGChebStep *cheb, bool launch = true) {
  if constexpr (!tile_shuffles<N>()) {
    return false;
  } else {
    constexpr size_t smem = dg_fused_smem<N, T>();
    const int form = face_form();
    if (!fuse_allowed() || !(form == 2 || form < 0) || !h.tiles64 || n_cells % 64 != 0 || smem > 200 * 1024)
      return false;
    const TileShape sh = tile_shape<N, T, true>();
    const int64_t n_tiles = n_cells / 64;
    if (form < 0 && n_tiles < 2 * (int64_t)sh.blocks_per_sm * sms) return false;
    if (!launch) return true;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, (int64_t)sh.blocks_per_sm * sms));
    if (units) *units = n_tiles;
    if (blocks) *blocks = grid;
    const auto tab = make_dg_tab<N, T>(h);
    const auto geo = make_geo(h);
    const T *sp = static_cast<const T *>(src);
    T *dp = static_cast<T *>(dst);
    const int32_t *nb = h.nbr.as<int32_t>();
    if (cheb) {
      const ChebArgs<T> ca{static_cast<const T *>(cheb->prev), static_cast<const T *>(cheb->b),
                           static_cast<const T *>(cheb->invd), (T)cheb->f1, (T)cheb->f2};
      if (sh.threads == 1024)
        dg_tile_fused_kernel<N, T, 1024, true><<<grid, 1024, smem, s>>>(tab, geo, sp, dp, nb, n_tiles, ca);
      else if (sh.threads == 512)
        dg_tile_fused_kernel<N, T, 512, true><<<grid, 512, smem, s>>>(tab, geo, sp, dp, nb, n_tiles, ca);
      else
        dg_tile_fused_kernel<N, T, 256, true><<<grid, 256, smem, s>>>(tab, geo, sp, dp, nb, n_tiles, ca);
    } else if (sh.threads == 1024) {
      dg_tile_fused_kernel<N, T, 1024><<<grid, 1024, smem, s>>>(tab, geo, sp, dp, nb, n_tiles);
    } else if (sh.threads == 512) {
      dg_tile_fused_kernel<N, T, 512><<<grid, 512, smem, s>>>(tab, geo, sp, dp, nb, n_tiles);
    } else {
      dg_tile_fused_kernel<N, T, 256><<<grid, 256, smem, s>>>(tab, geo, sp, dp, nb, n_tiles);
    }
    PMG_LAUNCH_CHECK();
    return true;
  }
}

template <typename T>
bool fused_dispatch(int degree, const DGHost &h, const void *src, void *dst, int64_t n_cells, int sms, cudaStream_t s,
                    int64_t *units, int64_t *blocks, const DGChebStep *cheb, bool launch = true) {
  switch (degree) {
  case 1: return fused_launch<2, T>(h, src, dst, n_cells, sms, s, units, blocks, cheb, launch);
  case 3: return fused_launch<4, T>(h, src, dst, n_cells, sms, s, units, blocks, cheb, launch);
  default: return false;
  }
}

} // namespace

bool dg_apply_fused(const DGHost &h, int degree, int dtype, const void *src, void *dst, int64_t n_cells, int sms,
                    cudaStream_t s, int64_t *units, int64_t *blocks, const DGChebStep *cheb) {
  return dtype == PMG_F64 ? fused_dispatch<double>(degree, h, src, dst, n_cells, sms, s, units, blocks, cheb)
                          : fused_dispatch<float>(degree, h, src, dst, n_cells, sms, s, units, blocks, cheb);
}

bool dg_fused_applies(const DGHost &h, int degree, int dtype, int64_t n_cells, int sms) {
  return dtype == PMG_F64
             ? fused_dispatch<double>(degree, h, nullptr, nullptr, n_cells, sms, nullptr, nullptr, nullptr, nullptr, false)
             : fused_dispatch<float>(degree, h, nullptr, nullptr, n_cells, sms, nullptr, nullptr, nullptr, nullptr, false);
}

void dg_setup(DGHost &h, const BoxMesh &mesh, int degree, double c_pen) {
  const int N = degree + 1;
  const Tables1D t = make_tables(degree, N);
  h.M1.assign(N * N, 0.0);
  h.K1.assign(N * N, 0.0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0, k = 0;
      for (int q = 0; q < N; ++q) {
        s += t.S[i * N + q] * t.S[j * N + q] * t.W[q];
        k += t.SD[i * N + q] * t.SD[j * N + q] * t.W[q];
      }
      h.M1[i * N + j] = s;
      h.K1[i * N + j] = k;
    }
  h.dphi0 = lagrange_derivative_at(degree, 0.0);
  h.dphi1 = lagrange_derivative_at(degree, 1.0);
  for (int d = 0; d < 3; ++d) h.h[d] = (mesh.box.hi[d] - mesh.box.lo[d]) / double(mesh.n[d]);
  h.c_pen = c_pen > 0 ? c_pen : degree * (degree + 1.0);
  h.dirichlet = mesh.box.dirichlet_mask;
  h.tiles64 = mesh.box.refine >= 2;
  // neighbour table [cell][2 d + s], -1 on the boundary
  const int64_t C = mesh.n_cells, nx = mesh.n[0], ny = mesh.n[1];
  std::vector<int32_t> lut(C);
  for (int64_t c = 0; c < C; ++c) {
    const int64_t x = mesh.cell_xyz[3 * c], y = mesh.cell_xyz[3 * c + 1], z = mesh.cell_xyz[3 * c + 2];
    lut[(z * ny + y) * nx + x] = (int32_t)c;
  }
  std::vector<int32_t> nb(C * 6);
  for (int64_t c = 0; c < C; ++c) {
    const int64_t xyz[3] = {mesh.cell_xyz[3 * c], mesh.cell_xyz[3 * c + 1], mesh.cell_xyz[3 * c + 2]};
    for (int f = 0; f < 6; ++f) {
      int64_t q[3] = {xyz[0], xyz[1], xyz[2]};
      const int d = f >> 1;
      q[d] += (f & 1) ? 1 : -1;
      nb[c * 6 + f] = (q[d] < 0 || q[d] >= mesh.n[d]) ? -1 : lut[(q[2] * ny + q[1]) * nx + q[0]];
    }
  }
  h.nbr = upload(nb);
}

void dg_apply_faces(const DGHost &h, int degree, int dtype, const void *src, void *dst, int64_t n_cells,
                    int sms, cudaStream_t s, int64_t *units, int64_t *blocks) {
  if (dtype == PMG_F64) face_dispatch<double>(degree, h, src, dst, n_cells, sms, s, false, units, blocks);
  else face_dispatch<float>(degree, h, src, dst, n_cells, sms, s, false, units, blocks);
}

void dg_add_face_diagonal(const DGHost &h, int degree, int dtype, void *diag, int64_t n_cells, int sms,
                          cudaStream_t s) {
  if (dtype == PMG_F64) face_dispatch<double>(degree, h, nullptr, diag, n_cells, sms, s, true);
  else face_dispatch<float>(degree, h, nullptr, diag, n_cells, sms, s, true);
}

// weak Dirichlet data of u = exp(x) sin(pi y) cos(pi z): b_l += (g, 2 sigma phi_l - d_n phi_l)
// on Dirichlet faces, nq-point Gauss rule per tangential direction (host, setup only)
void dg_add_boundary_rhs(const DGHost &h, const BoxMesh &mesh, int degree, int nq, int dtype, void *b,
                         cudaStream_t s) {
  const int N = degree + 1, N3 = N * N * N;
  const Tables1D t = make_tables(degree, nq);
  const int64_t C = mesh.n_cells;
  std::vector<double> add(C * N3, 0.0);
  bool any = false;
  for (int64_t c = 0; c < C; ++c) {
    const int64_t xyz[3] = {mesh.cell_xyz[3 * c], mesh.cell_xyz[3 * c + 1], mesh.cell_xyz[3 * c + 2]};
    for (int f = 0; f < 6; ++f) {
      const int d = f >> 1, sd = f & 1;
      const bool outside = sd ? xyz[d] == mesh.n[d] - 1 : xyz[d] == 0;
      if (!outside || !((h.dirichlet >> f) & 1)) continue;
      any = true;
      const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
      const double sigma = h.c_pen / h.h[d], sgn_h = (sd ? 1.0 : -1.0) / h.h[d];
      for (int bb = 0; bb < N; ++bb)
        for (int a = 0; a < N; ++a) {
          double gab = 0.0; // (g, phi_a phi_b) over the face
          for (int qb = 0; qb < nq; ++qb)
            for (int qa = 0; qa < nq; ++qa) {
              double x[3];
              x[d] = mesh.box.lo[d] + (xyz[d] + (sd ? 1.0 : 0.0)) * h.h[d];
              x[ta] = mesh.box.lo[ta] + (xyz[ta] + t.xg[qa]) * h.h[ta];
              x[tb] = mesh.box.lo[tb] + (xyz[tb] + t.xg[qb]) * h.h[tb];
              const double g = std::exp(x[0]) * std::sin(M_PI * x[1]) * std::cos(M_PI * x[2]);
              gab += g * t.W[qa] * t.W[qb] * h.h[ta] * h.h[tb] * t.S[a * nq + qa] * t.S[bb * nq + qb];
            }
          for (int i = 0; i < N; ++i) {
            int idx[3];
            idx[d] = i;
            idx[ta] = a;
            idx[tb] = bb;
            const int l = (idx[2] * N + idx[1]) * N + idx[0];
            const double phi_face = (i == (sd ? N - 1 : 0)) ? 1.0 : 0.0;
            const double dphi = (sd ? h.dphi1[i] : h.dphi0[i]) * sgn_h;
            add[c * N3 + l] += gab * (2.0 * sigma * phi_face - dphi);
          }
        }
    }
  }
  if (!any) return;
  DeviceBuffer tmp = upload(add);
  int sms = 0, dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = (int)std::min<int64_t>((C * N3 + 255) / 256, (int64_t)sms * 16);
  if (dtype == PMG_F64) add_kernel<double><<<grid, 256, 0, s>>>(static_cast<double *>(b), tmp.as<double>(), C * N3);
  else add_kernel<float><<<grid, 256, 0, s>>>(static_cast<float *>(b), tmp.as<double>(), C * N3);
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaStreamSynchronize(s)); // tmp is freed on return
}

} // namespace pmg
