// Tensor-core variant of the affine (+ coefficient) FP32 cell operator: TF32 mma.sync.
//
// The operator is the one of vmult_slab_kernel with GEOM 1 / 2 (axis-aligned cells, the
// diagonal cell tensor rr, ss, tt times the Gauss weights and the coefficient per point), the
// BK3 cell operator of include/kernels/bk3_kokkos_kernel.h:25-746.  Here one warp applies a
// cell as twelve 1D contractions, each a product of the cell's 64 node lines (8 x 8, the
// nodes padded from N <= 8 to 8 with zeros) with an 8 x 8 1D matrix on the tensor cores
// (mma.sync.m16n8k8, TF32 inputs, FP32 accumulation: four 16-row tiles per contraction),
// staged through the warp's shared memory, which re-slices the cell between contractions:
//   forward   T = U Sx, TX = U SDx;  W = T Sz, WZ = T SDz, WX = TX Sz;
//             DX = WX Sy, DY = W SDy, DZ = WZ Sy;  F = (rr, ss, tt) w kappa D  (in registers)
//   backward  GX = FX Sy^T, GY = FY SDy^T, GZ = FZ Sy^T;  HX = GX Sz^T, HYZ = GY Sz^T + GZ SDz^T;
//             out = HX SDx^T + HYZ Sx^T  -> scatter (red.global.add) from the accumulators.
// SPLIT = 1 rounds each operand to TF32 once (10 mantissa bits); SPLIT = 3 writes each as
// hi + lo TF32 parts and sums hi*hi + hi*lo + lo*hi (three products), about FP32 accuracy.
#include <algorithm>
#include <map>
#include <mutex>

#include "pmg_internal.hpp"
#include "fields.hpp"
#include "vmult_tc.hpp"

namespace pmg {
namespace {

constexpr int kTcWarps = 4;   // warps per block, one cell per warp at a time
constexpr int kRS = 8;        // stride of the second index (rows of 8)
constexpr int kKS = 72;       // stride of the outer index (8 rows + 8 pad: conflict-free z slices)
constexpr int kArr = 8 * kKS; // one padded cell array, floats
constexpr int kArrays = 4;    // shared arrays per warp

// the 1D tables as TF32 B fragments: m[which][hi/lo][0/1] for the thread's (t, g) positions
struct TcTables {
  float S[8][8], SD[8][8]; // S[i][q] = phi_i(g_q), padded with zeros
  float W[8];              // Gauss weights, 0 beyond N
};

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// B fragment of an 8 x 8 matrix M (K index = contracted input, N index = output): b0 = M[t][g],
// b1 = M[t + 4][g]; TRANS reads M^T (the transposed 1D table); split into TF32 hi / lo parts
template <int SPLIT> struct BFrag {
  uint32_t hi[2], lo[2];
};
template <int SPLIT, bool TRANS>
__device__ __forceinline__ BFrag<SPLIT> bfrag(const float (&M)[8][8], int g, int t) {
  BFrag<SPLIT> f;
  const float v0 = TRANS ? M[g][t] : M[t][g], v1 = TRANS ? M[g][t + 4] : M[t + 4][g];
  f.hi[0] = to_tf32(v0);
  f.hi[1] = to_tf32(v1);
  if (SPLIT == 3) {
    f.lo[0] = to_tf32(v0 - __uint_as_float(f.hi[0]));
    f.lo[1] = to_tf32(v1 - __uint_as_float(f.hi[1]));
  }
  return f;
}

// shared-memory offset of (outer o, middle m, inner i) in a padded cell array
__device__ __forceinline__ int off3(int o, int m, int i) { return o * kKS + m * kRS + i; }

// Contraction along AXIS (0: the inner index, 1: the middle, 2: the outer) of array X for the
// 16 rows of tile `mt`: A fragment of X (row = the two other indices, column = the contracted
// index) -> D += A B for each given B.  Row r of the tile order: axis 0: (outer, middle) = (r>>3,
// r&7); axis 1: (outer, inner); axis 2: (middle, inner).
template <int AXIS> __device__ __forceinline__ int a_off(int r, int c) {
  if (AXIS == 0) return off3(r >> 3, r & 7, c);
  if (AXIS == 1) return off3(r >> 3, c, r & 7);
  return off3(c, r >> 3, r & 7);
}

template <int AXIS, int SPLIT> struct AFrag {
  uint32_t hi[4], lo[4];
};
template <int AXIS, int SPLIT>
__device__ __forceinline__ AFrag<AXIS, SPLIT> afrag(const float *X, int mt, int g, int t) {
  AFrag<AXIS, SPLIT> f;
  const int r0 = 16 * mt + g, r1 = r0 + 8;
  const float v[4] = {X[a_off<AXIS>(r0, t)], X[a_off<AXIS>(r1, t)], X[a_off<AXIS>(r0, t + 4)],
                      X[a_off<AXIS>(r1, t + 4)]};
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    f.hi[m] = to_tf32(v[m]);
    if (SPLIT == 3) f.lo[m] = to_tf32(v[m] - __uint_as_float(f.hi[m]));
  }
  return f;
}

template <int AXIS, int SPLIT>
__device__ __forceinline__ void mma_acc(float (&d)[4], const AFrag<AXIS, SPLIT> &a, const BFrag<SPLIT> &b) {
  mma_tf32(d, a.hi, b.hi);
  if (SPLIT == 3) {
    mma_tf32(d, a.hi, b.lo);
    mma_tf32(d, a.lo, b.hi);
  }
}

// D fragment (rows 16 mt + g (+8), columns 2t, 2t+1) written back to Y in the slicing of AXIS
template <int AXIS> __device__ __forceinline__ void store_d(float *Y, int mt, int g, int t, const float (&d)[4]) {
  const int r0 = 16 * mt + g, r1 = r0 + 8;
  Y[a_off<AXIS>(r0, 2 * t)] = d[0];
  Y[a_off<AXIS>(r0, 2 * t + 1)] = d[1];
  Y[a_off<AXIS>(r1, 2 * t)] = d[2];
  Y[a_off<AXIS>(r1, 2 * t + 1)] = d[3];
}

// Y_j = X B_j along AXIS for the matrices B_j (one A fragment per tile, shared by the products)
template <int AXIS, int SPLIT, int NB>
__device__ __forceinline__ void contract(const float *X, float *const (&Y)[NB], const BFrag<SPLIT> (&B)[NB], int g,
                                         int t) {
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const AFrag<AXIS, SPLIT> a = afrag<AXIS, SPLIT>(X, mt, g, t);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      mma_acc<AXIS, SPLIT>(d, a, B[j]);
      store_d<AXIS>(Y[j], mt, g, t, d);
    }
  }
}

template <int N, int SPLIT, int GEOM>
__global__ void __launch_bounds__(32 * kTcWarps) vmult_tc_kernel(const __grid_constant__ TcTables tab,
                                                                 const float *__restrict__ src, float *__restrict__ dst,
                                                                 const uint32_t *__restrict__ idx,
                                                                 const float *__restrict__ geo,
                                                                 const float *__restrict__ coef, int64_t n_cells) {
  constexpr int CPW = 32 / N, LANES = CPW * N, N2 = N * N, N3 = N2 * N;
  extern __shared__ __align__(16) float tc_smem[];
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float *const A0 = tc_smem + (threadIdx.x >> 5) * kArrays * kArr;
  float *const A1 = A0 + kArr, *const A2 = A1 + kArr, *const A3 = A2 + kArr;
  for (int e = lane; e < kArrays * kArr; e += 32) A0[e] = 0.f; // padding stays zero from here on
  __syncwarp();
  const BFrag<SPLIT> bS = bfrag<SPLIT, false>(tab.S, g, t), bSD = bfrag<SPLIT, false>(tab.SD, g, t);
  const BFrag<SPLIT> bST = bfrag<SPLIT, true>(tab.S, g, t), bSDT = bfrag<SPLIT, true>(tab.SD, g, t);
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t c = warp0; c < n_cells; c += nwarps) {
    const int64_t grp = c / CPW;
    const int e = (int)(c - grp * CPW);
    // gather U[k][j][i] (sentinel -> 0) from the slab index map [group][k*N+i][e*N+j]
    for (int l = lane; l < N3; l += 32) {
      const int i = l % N, j = (l / N) % N, k = l / N2;
      const uint32_t id = __ldg(idx + (grp * N2 + k * N + i) * LANES + e * N + j);
      A0[off3(k, j, i)] = id != 0xFFFFFFFFu ? __ldg(src + id) : 0.f;
    }
    __syncwarp();
    { // x: T = U Sx -> A1, TX = U SDx -> A2
      float *const Y[2] = {A1, A2};
      const BFrag<SPLIT> B[2] = {bS, bSD};
      contract<0, SPLIT, 2>(A0, Y, B, g, t);
    }
    __syncwarp();
    { // z: W = T Sz -> A0, WZ = T SDz -> A3
      float *const Y[2] = {A0, A3};
      const BFrag<SPLIT> B[2] = {bS, bSD};
      contract<2, SPLIT, 2>(A1, Y, B, g, t);
    }
    __syncwarp();
    { // z: WX = TX Sz -> A1 (T is consumed)
      float *const Y[1] = {A1};
      const BFrag<SPLIT> B[1] = {bS};
      contract<2, SPLIT, 1>(A2, Y, B, g, t);
    }
    __syncwarp();
    // y with the point factors in the epilogue: F = c_d w kappa D at (qx, qy, qz), written over
    // the array each product read (a tile's rows occupy their own slice of every array, so a
    // tile is stored once all lanes have loaded it): FX over WX (A1), FY over W (A0), FZ over
    // WZ (A3)
    const float *cg = geo + c * 8;
    const float c0 = __ldg(cg), c3 = __ldg(cg + 3), c5 = __ldg(cg + 5);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const AFrag<1, SPLIT> ax = afrag<1, SPLIT>(A1, mt, g, t); // WX: rows (qz, qx), column y node
      const AFrag<1, SPLIT> ay = afrag<1, SPLIT>(A0, mt, g, t); // W
      const AFrag<1, SPLIT> az = afrag<1, SPLIT>(A3, mt, g, t); // WZ
      float dx[4] = {0.f, 0.f, 0.f, 0.f}, dy[4] = {0.f, 0.f, 0.f, 0.f}, dz[4] = {0.f, 0.f, 0.f, 0.f};
      mma_acc<1, SPLIT>(dx, ax, bS);
      mma_acc<1, SPLIT>(dy, ay, bSD);
      mma_acc<1, SPLIT>(dz, az, bS);
      // point factors of the four accumulator entries: rows (qz, qx), columns qy
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int r = 16 * mt + g + (m >= 2 ? 8 : 0), qy = 2 * t + (m & 1);
        const int qz = r >> 3, qx = r & 7;
        float w = 0.f;
        if (qx < N && qy < N && qz < N) {
          w = tab.W[qx] * tab.W[qy] * tab.W[qz];
          if (GEOM == 2) w *= __ldg(coef + (grp * N2 + qy * N + qx) * LANES + e * N + qz);
        }
        dx[m] *= c0 * w;
        dy[m] *= c3 * w;
        dz[m] *= c5 * w;
      }
      __syncwarp(); // every lane has read this tile of WX, W, WZ before it is overwritten
      store_d<1>(A1, mt, g, t, dx); // FX over WX
      store_d<1>(A0, mt, g, t, dy); // FY over W
      store_d<1>(A3, mt, g, t, dz); // FZ over WZ
    }
    __syncwarp();
    { // y^T: GX = FX Sy^T -> A2, GY = FY SDy^T -> A1 ... in place after loading each tile
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const AFrag<1, SPLIT> ax = afrag<1, SPLIT>(A1, mt, g, t);
        const AFrag<1, SPLIT> ay = afrag<1, SPLIT>(A0, mt, g, t);
        const AFrag<1, SPLIT> az = afrag<1, SPLIT>(A3, mt, g, t);
        float gx[4] = {0.f, 0.f, 0.f, 0.f}, gy[4] = {0.f, 0.f, 0.f, 0.f}, gz[4] = {0.f, 0.f, 0.f, 0.f};
        mma_acc<1, SPLIT>(gx, ax, bST);
        mma_acc<1, SPLIT>(gy, ay, bSDT);
        mma_acc<1, SPLIT>(gz, az, bST);
        __syncwarp();
        store_d<1>(A1, mt, g, t, gx);
        store_d<1>(A0, mt, g, t, gy);
        store_d<1>(A3, mt, g, t, gz);
      }
    }
    __syncwarp();
    { // z^T: HX = GX Sz^T -> A2, HYZ = GY Sz^T + GZ SDz^T -> A1 ... rows (y node, qx), column qz
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const AFrag<2, SPLIT> ax = afrag<2, SPLIT>(A1, mt, g, t);
        const AFrag<2, SPLIT> ay = afrag<2, SPLIT>(A0, mt, g, t);
        const AFrag<2, SPLIT> az = afrag<2, SPLIT>(A3, mt, g, t);
        float hx[4] = {0.f, 0.f, 0.f, 0.f}, hyz[4] = {0.f, 0.f, 0.f, 0.f};
        mma_acc<2, SPLIT>(hx, ax, bST);
        mma_acc<2, SPLIT>(hyz, ay, bST);
        mma_acc<2, SPLIT>(hyz, az, bSDT);
        store_d<2>(A2, mt, g, t, hx);
        __syncwarp();
        store_d<2>(A1, mt, g, t, hyz);
      }
    }
    __syncwarp();
    // x^T: out = HX SDx^T + HYZ Sx^T: rows (z node, y node), columns the x node -> scatter
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
      const AFrag<0, SPLIT> ax = afrag<0, SPLIT>(A2, mt, g, t);
      const AFrag<0, SPLIT> ay = afrag<0, SPLIT>(A1, mt, g, t);
      float o[4] = {0.f, 0.f, 0.f, 0.f};
      mma_acc<0, SPLIT>(o, ax, bSDT);
      mma_acc<0, SPLIT>(o, ay, bST);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int r = 16 * mt + g + (m >= 2 ? 8 : 0), i = 2 * t + (m & 1);
        const int k = r >> 3, j = r & 7;
        if (i < N && j < N && k < N) {
          const uint32_t id = __ldg(idx + (grp * N2 + k * N + i) * LANES + e * N + j);
          if (id != 0xFFFFFFFFu) atomicAdd(dst + id, o[m]);
        }
      }
    }
    __syncwarp(); // the arrays are rewritten by the next cell
  }
}

template <int N, int SPLIT, int GEOM> void launch_n(const pmg_operator &op, const void *src, void *dst, cudaStream_t s) {
  auto k = vmult_tc_kernel<N, SPLIT, GEOM>;
  const size_t smem = sizeof(float) * kTcWarps * kArrays * kArr;
  static std::mutex mu;
  static std::map<int, int> per_sm;
  int blocks = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = per_sm.find(op.device);
    if (it == per_sm.end()) {
      PMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int nb = 0;
      PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * kTcWarps, smem));
      it = per_sm.emplace(op.device, std::max(1, nb)).first;
    }
    blocks = it->second;
  }
  const int64_t want = (op.n_cells + kTcWarps - 1) / kTcWarps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)blocks * op.sms));
  const Tables1D &t1 = cached_tables(op.degree);
  TcTables tab{};
  for (int i = 0; i < N; ++i)
    for (int q = 0; q < N; ++q) {
      tab.S[i][q] = (float)t1.S[i * N + q];
      tab.SD[i][q] = (float)t1.SD[i * N + q];
    }
  for (int q = 0; q < N; ++q) tab.W[q] = (float)t1.W[q];
  op.launch_units[PMG_KERNEL_VMULT_CELL] = op.n_cells;
  op.launch_par[PMG_KERNEL_VMULT_CELL] = (int64_t)grid * kTcWarps;
  k<<<grid, 32 * kTcWarps, smem, s>>>(tab, static_cast<const float *>(src), static_cast<float *>(dst),
                                      op.idx.as<uint32_t>(), op.geo.as<float>(), op.coef.as<float>(), op.n_cells);
  PMG_LAUNCH_CHECK();
}

template <int SPLIT, int GEOM> void launch_split(const pmg_operator &op, const void *src, void *dst, cudaStream_t s) {
  switch (op.nm) {
  case 2: launch_n<2, SPLIT, GEOM>(op, src, dst, s); break;
  case 3: launch_n<3, SPLIT, GEOM>(op, src, dst, s); break;
  case 4: launch_n<4, SPLIT, GEOM>(op, src, dst, s); break;
  case 5: launch_n<5, SPLIT, GEOM>(op, src, dst, s); break;
  case 6: launch_n<6, SPLIT, GEOM>(op, src, dst, s); break;
  case 7: launch_n<7, SPLIT, GEOM>(op, src, dst, s); break;
  default: fail(PMG_EINVAL, "tensor-core vmult: degree must be in [1,6]");
  }
}

} // namespace

void vmult_cells_tensor_cores(const pmg_operator &op, const void *src, void *dst, cudaStream_t s) {
  const bool coef = op.has_coeff_values;
  if (op.tensor_cores == 3) {
    if (coef) launch_split<3, 2>(op, src, dst, s);
    else launch_split<3, 1>(op, src, dst, s);
  } else {
    if (coef) launch_split<1, 2>(op, src, dst, s);
    else launch_split<1, 1>(op, src, dst, s);
  }
}

} // namespace pmg
