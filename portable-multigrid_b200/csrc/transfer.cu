// Multigrid transfers between levels: polynomial (same mesh, degree pc -> pf;
// include/multigrid/portable_polynomial_transfer.h + BK1 batched kernels
// include/kernels/bk1_kokkos_kernels.h:462-1051) and geometric (same degree, one global
// refinement; include/multigrid/portable_geometric_transfer.h).  Both are "patch"
// transfers: every patch (fine cell for p, coarse cell for h) maps its coarse DoFs
// (Dirichlet entries dropped) through the tensor product of a 1D matrix onto its fine
// DoFs, each fine entry scaled by 1/(number of patches holding it), 0 when constrained.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

#include "pmg_internal.hpp"
#include "transfer.hpp"

namespace pmg {
namespace {

template <typename T>
__global__ void transfer_kernel(int dir, int nc, int nf, int ppb, const T *__restrict__ P,
                                const T *__restrict__ src, T *__restrict__ dst,
                                const uint32_t *__restrict__ cidx,
                                const uint32_t *__restrict__ fidx, const T *__restrict__ w,
                                int64_t n_patches) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sP = reinterpret_cast<T *>(smem_raw);
  const int nf3 = nf * nf * nf, nc3 = nc * nc * nc;
  T *buf = sP + ((nc * nf + 3) & ~3);
  for (int i = threadIdx.x; i < nc * nf; i += blockDim.x) sP[i] = P[i];
  __syncthreads();
  const int a = dir == 0 ? nc : nf, b = dir == 0 ? nf : nc;
  const int a3 = a * a * a, b3 = b * b * b;
  const int bs = blockDim.x;
#define MAT(i, o) (dir == 0 ? sP[(i) * nf + (o)] : sP[(o) * nf + (i)])
  for (int64_t base = blockIdx.x * (int64_t)ppb; base < n_patches; base += (int64_t)gridDim.x * ppb) {
    const int np = (int)min((int64_t)ppb, n_patches - base);
    for (int t = threadIdx.x; t < np * a3; t += bs) {
      const int pi = t / a3, l = t - pi * a3;
      const int64_t patch = base + pi;
      T *in = buf + pi * 3 * nf3;
      if (dir == 0) {
        const uint32_t id = cidx[patch * nc3 + l];
        in[l] = (id != kInvalid) ? src[id] : T(0);
      } else {
        in[l] = w[patch * nf3 + l] * src[fidx[patch * nf3 + l]];
      }
    }
    __syncthreads();
    // x: t1[k][j][x] = sum_i M(i,x) in[k][j][i]
    for (int t = threadIdx.x; t < np * a * a * b; t += bs) {
      const int pi = t / (a * a * b), r = t - pi * (a * a * b);
      const int x = r % b, kj = r / b;
      const T *in = buf + pi * 3 * nf3 + kj * a;
      T s = 0;
      for (int i = 0; i < a; ++i) s += MAT(i, x) * in[i];
      buf[pi * 3 * nf3 + nf3 + kj * b + x] = s;
    }
    __syncthreads();
    // y: t2[k][y][x] = sum_j M(j,y) t1[k][j][x]
    for (int t = threadIdx.x; t < np * a * b * b; t += bs) {
      const int pi = t / (a * b * b), r = t - pi * (a * b * b);
      const int x = r % b, y = (r / b) % b, k = r / (b * b);
      const T *t1 = buf + pi * 3 * nf3 + nf3 + k * a * b;
      T s = 0;
      for (int j = 0; j < a; ++j) s += MAT(j, y) * t1[j * b + x];
      buf[pi * 3 * nf3 + 2 * nf3 + (k * b + y) * b + x] = s;
    }
    __syncthreads();
    // z and scatter
    for (int t = threadIdx.x; t < np * b3; t += bs) {
      const int pi = t / b3, l = t - pi * b3;
      const int yx = l % (b * b), z = l / (b * b);
      const T *t2 = buf + pi * 3 * nf3 + 2 * nf3 + yx;
      T s = 0;
      for (int k = 0; k < a; ++k) s += MAT(k, z) * t2[k * b * b];
      const int64_t patch = base + pi;
      if (dir == 0) {
        atomicAdd(dst + fidx[patch * nf3 + l], w[patch * nf3 + l] * s);
      } else {
        const uint32_t id = cidx[patch * nc3 + l];
        if (id != kInvalid) atomicAdd(dst + id, s);
      }
    }
    __syncthreads();
  }
#undef MAT
}

// Warp-per-patch form of transfer_kernel for NC, NF <= 7 (every p-transfer up to degree 6
// and the h-transfers up to degree 3): sizes known at compile time, the patch's three
// tensor sweeps run through per-warp shared-memory buffers with warp barriers only, the 1D
// matrix sits in shared memory (lanes read different entries).  Same index conventions
// and results as transfer_kernel.
template <int NC, int NF, typename T> struct TMat {
  T m[NC * NF]; // m[i_c * NF + j_f]
};

template <typename T, int NC, int NF, int DIR> struct PatchShape {
  static constexpr int A = DIR == 0 ? NC : NF, B = DIR == 0 ? NF : NC;
  static constexpr int A3 = A * A * A, B3 = B * B * B, T1 = A * A * B, T2 = A * B * B;
  static constexpr int PER_WARP = A3 + T1 + T2; // elements of T
};

constexpr int kPatchWarps = 8;

template <typename T, int NC, int NF, int DIR>
__global__ void __launch_bounds__(32 * kPatchWarps)
    transfer_patch_kernel(const __grid_constant__ TMat<NC, NF, T> P, const T *__restrict__ src,
                          T *__restrict__ dst, const uint32_t *__restrict__ cidx,
                          const uint32_t *__restrict__ fidx, const T *__restrict__ w, int64_t n_patches) {
  using Sh = PatchShape<T, NC, NF, DIR>;
  constexpr int A = Sh::A, B = Sh::B, NC3 = NC * NC * NC, NF3 = NF * NF * NF;
  __shared__ T sM[NC * NF];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for (int i = threadIdx.x; i < NC * NF; i += blockDim.x) sM[i] = P.m[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  T *in = reinterpret_cast<T *>(smem_raw) + (threadIdx.x >> 5) * Sh::PER_WARP;
  T *t1 = in + Sh::A3;
  T *t2 = t1 + Sh::T1;
  const int64_t warp0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  // M(i, o): input index i, output index o
  auto M = [&](int i, int o) -> T { return DIR == 0 ? sM[i * NF + o] : sM[o * NF + i]; };
  for (int64_t patch = warp0; patch < n_patches; patch += nwarps) {
    for (int l = lane; l < Sh::A3; l += 32) {
      if (DIR == 0) {
        const uint32_t id = __ldg(cidx + patch * NC3 + l);
        in[l] = (id != kInvalid) ? src[id] : T(0);
      } else {
        in[l] = __ldg(w + patch * NF3 + l) * src[__ldg(fidx + patch * NF3 + l)];
      }
    }
    __syncwarp();
    for (int t = lane; t < Sh::T1; t += 32) { // t1[k][j][x] = sum_i M(i, x) in[k][j][i]
      const int x = t % B, kj = t / B;
      T s = T(0);
#pragma unroll
      for (int i = 0; i < A; ++i) s = fma(M(i, x), in[kj * A + i], s);
      t1[kj * B + x] = s;
    }
    __syncwarp();
    for (int t = lane; t < Sh::T2; t += 32) { // t2[k][y][x] = sum_j M(j, y) t1[k][j][x]
      const int x = t % B, y = (t / B) % B, k = t / (B * B);
      T s = T(0);
#pragma unroll
      for (int j = 0; j < A; ++j) s = fma(M(j, y), t1[(k * A + j) * B + x], s);
      t2[(k * B + y) * B + x] = s;
    }
    __syncwarp();
    for (int t = lane; t < Sh::B3; t += 32) { // z sweep and scatter
      const int yx = t % (B * B), z = t / (B * B);
      T s = T(0);
#pragma unroll
      for (int k = 0; k < A; ++k) s = fma(M(k, z), t2[k * B * B + yx], s);
      if (DIR == 0) {
        atomicAdd(dst + __ldg(fidx + patch * NF3 + t), __ldg(w + patch * NF3 + t) * s);
      } else {
        const uint32_t id = __ldg(cidx + patch * NC3 + t);
        if (id != kInvalid) atomicAdd(dst + id, s);
      }
    }
    __syncwarp();
  }
}

// DG <-> CG at equal degree: the 1D matrix is the identity and every fine (DG) entry is
// listed once, so the transfer is an entry-wise gather / scatter-add.
template <typename T, int DIR>
__global__ void transfer_identity_kernel(const T *__restrict__ src, T *__restrict__ dst,
                                         const uint32_t *__restrict__ cidx, const uint32_t *__restrict__ fidx,
                                         const T *__restrict__ w, int64_t n_entries) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_entries;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t id = __ldg(cidx + e);
    if (DIR == 0) {
      const uint32_t f = __ldg(fidx + e);
      dst[f] += (id != kInvalid) ? __ldg(w + e) * src[id] : T(0);
    } else if (id != kInvalid) {
      atomicAdd(dst + id, __ldg(w + e) * src[__ldg(fidx + e)]);
    }
  }
}

template <typename T, int NC, int NF, int DIR>
void patch_launch(const pmg_transfer &t, void *dst, const void *src, cudaStream_t s) {
  using Sh = PatchShape<T, NC, NF, DIR>;
  auto k = transfer_patch_kernel<T, NC, NF, DIR>;
  const size_t smem = size_t(kPatchWarps) * Sh::PER_WARP * sizeof(T);
  TMat<NC, NF, T> P;
  for (int i = 0; i < NC * NF; ++i) P.m[i] = (T)t.P_host[i];
  static std::mutex mu;
  static std::map<int, int> per_sm; // device -> resident blocks per SM
  int blocks = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = per_sm.find(t.device);
    if (it == per_sm.end()) {
      PMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int nb = 0;
      PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * kPatchWarps, smem));
      it = per_sm.emplace(t.device, std::max(1, nb)).first;
    }
    blocks = it->second;
  }
  const int64_t want = (t.n_patches + kPatchWarps - 1) / kPatchWarps;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)blocks * t.sms));
  t.launch_units = t.n_patches;
  t.launch_par = (int64_t)grid * kPatchWarps;
  k<<<grid, 32 * kPatchWarps, smem, s>>>(P, static_cast<const T *>(src), static_cast<T *>(dst),
                                         t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                         t.weights.as<T>(), t.n_patches);
  PMG_LAUNCH_CHECK();
}

// runtime (nc, nf) -> compiled pair; false if the pair has no compiled form
template <typename T, int DIR, int NC, int NF> bool try_pair(const pmg_transfer &t, void *dst, const void *src,
                                                           cudaStream_t s) {
  if (t.nc != NC || t.nf != NF) return false;
  patch_launch<T, NC, NF, DIR>(t, dst, src, s);
  return true;
}
template <typename T, int DIR> bool patch_dispatch(const pmg_transfer &t, void *dst, const void *src, cudaStream_t s) {
  return try_pair<T, DIR, 2, 3>(t, dst, src, s) || try_pair<T, DIR, 2, 4>(t, dst, src, s) ||
         try_pair<T, DIR, 2, 5>(t, dst, src, s) || try_pair<T, DIR, 2, 6>(t, dst, src, s) ||
         try_pair<T, DIR, 2, 7>(t, dst, src, s) || try_pair<T, DIR, 3, 4>(t, dst, src, s) ||
         try_pair<T, DIR, 3, 5>(t, dst, src, s) || try_pair<T, DIR, 3, 6>(t, dst, src, s) ||
         try_pair<T, DIR, 3, 7>(t, dst, src, s) || try_pair<T, DIR, 4, 5>(t, dst, src, s) ||
         try_pair<T, DIR, 4, 6>(t, dst, src, s) || try_pair<T, DIR, 4, 7>(t, dst, src, s) ||
         try_pair<T, DIR, 5, 6>(t, dst, src, s) || try_pair<T, DIR, 5, 7>(t, dst, src, s) ||
         try_pair<T, DIR, 6, 7>(t, dst, src, s);
}

template <typename T> std::vector<T> cast(const std::vector<double> &v) {
  return std::vector<T>(v.begin(), v.end());
}

// PMG_TRANSFER_GENERIC=1 keeps every transfer on transfer_kernel (a comparison switch)
bool patch_kernels_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("PMG_TRANSFER_GENERIC");
    return !(e && e[0] == '1');
  }();
  return on;
}

bool same_box_geometry(const pmg_box &a, const pmg_box &b) {
  for (int d = 0; d < 3; ++d)
    if (a.coarse[d] != b.coarse[d] || a.lo[d] != b.lo[d] || a.hi[d] != b.hi[d]) return false;
  return a.deform == b.deform && a.amp == b.amp && a.dirichlet_mask == b.dirichlet_mask;
}

// weights (1 / multiplicity of the fine DoF over all patches, 0 when constrained, unless
// given), the 1D matrix and the maps on the device, launch parameters
void transfer_finish(pmg_transfer &t, const pmg_operator &fine, const std::vector<double> &P,
                     const std::vector<uint32_t> &cidx, const std::vector<uint32_t> &fidx,
                     const double *given_weights) {
  std::vector<double> w(fidx.size());
  if (given_weights) {
    std::copy(given_weights, given_weights + fidx.size(), w.begin());
  } else {
    std::vector<double> mult(t.n_fine, 0.0);
    for (uint32_t d : fidx) mult[d] += 1.0;
    for (int64_t i = 0; i < t.n_fine; ++i)
      mult[i] = (fine.num.constrained[i] || mult[i] == 0.0) ? 0.0 : 1.0 / mult[i];
    for (size_t e = 0; e < fidx.size(); ++e) w[e] = mult[fidx[e]];
  }
  t.P_host = P;
  if (t.dtype == PMG_F64) {
    t.P1d = upload(P);
    t.weights = upload(w);
  } else {
    t.P1d = upload(cast<float>(P));
    t.weights = upload(cast<float>(w));
  }
  t.coarse_idx = upload(cidx);
  t.fine_idx = upload(fidx);
  const size_t s = dtype_size(t.dtype);
  const int nf3 = t.nf * t.nf * t.nf;
  t.ppb = (int)std::max<size_t>(1, (32 * 1024) / (3 * nf3 * s));
  t.smem = s * (((t.nc * t.nf + 3) & ~3) + (size_t)t.ppb * 3 * nf3);
  int sms = 0;
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, t.device));
  t.sms = sms;
  t.patch_kernels = patch_kernels_enabled();
  t.grid = (int)std::max<int64_t>(1, std::min<int64_t>((t.n_patches + t.ppb - 1) / t.ppb, (int64_t)sms * 8));
  if (t.dtype == PMG_F64)
    PMG_CUDA(cudaFuncSetAttribute(transfer_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  else
    PMG_CUDA(cudaFuncSetAttribute(transfer_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
}

} // namespace

void transfer_setup_from_maps(pmg_transfer &t, const pmg_operator &coarse, const pmg_operator &fine,
                              const pmg_transfer_maps &m) {
  PMG_REQUIRE(coarse.dtype == fine.dtype, "transfer levels must have the same dtype");
  PMG_REQUIRE(coarse.device == fine.device, "transfer levels must live on one device");
  PMG_REQUIRE(m.n_patches >= 0, "negative patch count");
  PMG_REQUIRE(m.n_patches == 0 || (m.coarse_indices && m.fine_indices), "null index map");
  PMG_CUDA(cudaSetDevice(fine.device));
  t.device = fine.device;
  t.dtype = fine.dtype;
  t.n_coarse = coarse.n_dofs;
  t.n_fine = fine.n_dofs;
  t.n_patches = m.n_patches;
  const int pc = coarse.degree, pf = fine.degree;
  std::vector<double> P;
  if (m.kind == PMG_TRANSFER_POLYNOMIAL) {
    PMG_REQUIRE(pc < pf, "polynomial transfer needs degree_coarse < degree_fine");
    t.kind = 0;
    t.nc = pc + 1;
    t.nf = pf + 1;
    P = p_transfer_matrix(pc, pf);
  } else if (m.kind == PMG_TRANSFER_GEOMETRIC) {
    PMG_REQUIRE(pc == pf, "geometric transfer needs equal degrees");
    t.kind = 1;
    t.nc = pc + 1;
    t.nf = 2 * pc + 1;
    P = h_transfer_matrix(pc);
  } else if (m.kind == PMG_TRANSFER_DG_CG) {
    PMG_REQUIRE(pc == pf, "DG <-> CG transfer needs equal degrees");
    t.kind = 2;
    t.nc = t.nf = pc + 1;
    P.assign(t.nc * t.nf, 0.0);
    for (int i = 0; i < t.nc; ++i) P[i * t.nf + i] = 1.0;
  } else {
    fail(PMG_EINVAL, "kind must be PMG_TRANSFER_POLYNOMIAL, _GEOMETRIC or _DG_CG");
  }
  const size_t nc3 = (size_t)t.nc * t.nc * t.nc, nf3 = (size_t)t.nf * t.nf * t.nf;
  std::vector<uint32_t> cidx(m.coarse_indices, m.coarse_indices + m.n_patches * nc3);
  std::vector<uint32_t> fidx(m.fine_indices, m.fine_indices + m.n_patches * nf3);
  for (size_t e = 0; e < cidx.size(); ++e) {
    uint32_t &d = cidx[e];
    if (d == kInvalid) continue;
    if ((int64_t)d >= t.n_coarse)
      fail(PMG_EBOUNDS, "coarse_indices[" + std::to_string(e) + "] = " + std::to_string(d) + " >= " +
                            std::to_string(t.n_coarse));
    if (coarse.num.constrained[d]) d = kInvalid;
  }
  for (size_t e = 0; e < fidx.size(); ++e)
    if ((int64_t)fidx[e] >= t.n_fine)
      fail(PMG_EBOUNDS, "fine_indices[" + std::to_string(e) + "] = " + std::to_string(fidx[e]) + " >= " +
                            std::to_string(t.n_fine));
  transfer_finish(t, fine, P, cidx, fidx, m.weights);
}

void transfer_setup(pmg_transfer &t, const pmg_operator &coarse, const pmg_operator &fine) {
  PMG_REQUIRE(!coarse.from_maps && !fine.from_maps,
              "operators built from caller maps take their transfers from pmg_transfer_create_from_maps");
  PMG_REQUIRE(coarse.dtype == fine.dtype, "transfer levels must have the same dtype");
  PMG_REQUIRE(coarse.device == fine.device, "transfer levels must live on one device");
  PMG_REQUIRE(same_box_geometry(coarse.mesh.box, fine.mesh.box), "levels must discretise the same box");
  PMG_CUDA(cudaSetDevice(fine.device));
  t.device = fine.device;
  t.dtype = fine.dtype;
  t.n_coarse = coarse.n_dofs;
  t.n_fine = fine.n_dofs;
  const int pc = coarse.degree, pf = fine.degree;
  std::vector<double> P;
  std::vector<uint32_t> cidx, fidx;
  if (fine.kind == PMG_OP_DG_SIPG) {
    // DG <-> CG at equal degree (ContinuousTransfer): identity on every cell, unit weights
    PMG_REQUIRE(coarse.kind == PMG_OP_LAPLACE, "the coarse level of a DG transfer must be continuous");
    PMG_REQUIRE(pc == pf && coarse.mesh.box.refine == fine.mesh.box.refine,
                "DG <-> CG transfer needs equal degrees on the same mesh");
    t.kind = 2;
    t.nc = t.nf = pc + 1;
    t.n_patches = fine.n_cells;
    P.assign(t.nc * t.nf, 0.0);
    for (int i = 0; i < t.nc; ++i) P[i * t.nf + i] = 1.0;
    cidx.resize(coarse.num.plain.size());
    for (size_t e = 0; e < cidx.size(); ++e) {
      const uint32_t d = coarse.num.plain[e];
      cidx[e] = coarse.num.constrained[d] ? kInvalid : d;
    }
    fidx = fine.num.plain;
  } else if (coarse.mesh.box.refine == fine.mesh.box.refine) {
    PMG_REQUIRE(coarse.kind == PMG_OP_LAPLACE, "a DG level can only be the finest level of a transfer");
    PMG_REQUIRE(pc < pf, "polynomial transfer needs degree_coarse < degree_fine");
    t.kind = 0;
    t.nc = pc + 1;
    t.nf = pf + 1;
    t.n_patches = fine.n_cells;
    P = p_transfer_matrix(pc, pf);
    const int nc3 = t.nc * t.nc * t.nc;
    cidx.resize((size_t)t.n_patches * nc3);
    for (size_t e = 0; e < cidx.size(); ++e) {
      const uint32_t d = coarse.num.plain[e];
      cidx[e] = coarse.num.constrained[d] ? kInvalid : d;
    }
    fidx = fine.num.plain;
  } else {
    PMG_REQUIRE(fine.mesh.box.refine == coarse.mesh.box.refine + 1,
                "geometric transfer needs the fine mesh refined exactly once more");
    PMG_REQUIRE(pc == pf, "geometric transfer needs equal degrees");
    PMG_REQUIRE(!fine.num.lattice.empty(), "fine operator has no node lattice");
    const int p = pc;
    t.kind = 1;
    t.nc = p + 1;
    t.nf = 2 * p + 1;
    t.n_patches = coarse.n_cells;
    P = h_transfer_matrix(p);
    const int nc3 = t.nc * t.nc * t.nc, nf = t.nf, nf3 = nf * nf * nf;
    cidx.resize((size_t)t.n_patches * nc3);
    for (size_t e = 0; e < cidx.size(); ++e) {
      const uint32_t d = coarse.num.plain[e];
      cidx[e] = coarse.num.constrained[d] ? kInvalid : d;
    }
    fidx.resize((size_t)t.n_patches * nf3);
    const int64_t L0 = fine.num.L[0], L1 = fine.num.L[1];
    for (int64_t c = 0; c < t.n_patches; ++c) {
      const int64_t bx = 2LL * p * coarse.mesh.cell_xyz[3 * c], by = 2LL * p * coarse.mesh.cell_xyz[3 * c + 1],
                    bz = 2LL * p * coarse.mesh.cell_xyz[3 * c + 2];
      for (int k = 0; k < nf; ++k)
        for (int j = 0; j < nf; ++j)
          for (int i = 0; i < nf; ++i)
            fidx[c * nf3 + (k * nf + j) * nf + i] = fine.num.lattice[((bz + k) * L1 + (by + j)) * L0 + bx + i];
    }
  }
  transfer_finish(t, fine, P, cidx, fidx, nullptr);
}

void transfer_apply(const pmg_transfer &t, int dir, void *dst, const void *src, cudaStream_t s) {
  PMG_REQUIRE(dst && src, "null vector");
  if (t.n_patches == 0) return;
  prof::Scope scope(dir == 0 ? "transfer_prolongate" : "transfer_restrict", s);
  if (t.kind == 2) {
    const int64_t n = t.n_patches * t.nf * t.nf * t.nf;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)t.sms * 16));
    t.launch_units = n;
    t.launch_par = (int64_t)grid * 256;
    if (t.dtype == PMG_F64) {
      if (dir == 0)
        transfer_identity_kernel<double, 0><<<grid, 256, 0, s>>>(static_cast<const double *>(src), static_cast<double *>(dst),
                                                                 t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                                                 t.weights.as<double>(), n);
      else
        transfer_identity_kernel<double, 1><<<grid, 256, 0, s>>>(static_cast<const double *>(src), static_cast<double *>(dst),
                                                                 t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                                                 t.weights.as<double>(), n);
    } else {
      if (dir == 0)
        transfer_identity_kernel<float, 0><<<grid, 256, 0, s>>>(static_cast<const float *>(src), static_cast<float *>(dst),
                                                                t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                                                t.weights.as<float>(), n);
      else
        transfer_identity_kernel<float, 1><<<grid, 256, 0, s>>>(static_cast<const float *>(src), static_cast<float *>(dst),
                                                                t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                                                t.weights.as<float>(), n);
    }
    PMG_LAUNCH_CHECK();
    return;
  }
  if (t.patch_kernels) {
    bool done = false;
    if (t.dtype == PMG_F64) done = dir == 0 ? patch_dispatch<double, 0>(t, dst, src, s) : patch_dispatch<double, 1>(t, dst, src, s);
    else done = dir == 0 ? patch_dispatch<float, 0>(t, dst, src, s) : patch_dispatch<float, 1>(t, dst, src, s);
    if (done) return;
  }
  t.launch_units = (t.n_patches + t.ppb - 1) / t.ppb;
  t.launch_par = t.grid;
  if (t.dtype == PMG_F64)
    transfer_kernel<double><<<t.grid, 128, t.smem, s>>>(dir, t.nc, t.nf, t.ppb, t.P1d.as<double>(),
                                                        static_cast<const double *>(src), static_cast<double *>(dst),
                                                        t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                                        t.weights.as<double>(), t.n_patches);
  else
    transfer_kernel<float><<<t.grid, 128, t.smem, s>>>(dir, t.nc, t.nf, t.ppb, t.P1d.as<float>(),
                                                       static_cast<const float *>(src), static_cast<float *>(dst),
                                                       t.coarse_idx.as<uint32_t>(), t.fine_idx.as<uint32_t>(),
                                                       t.weights.as<float>(), t.n_patches);
  PMG_LAUNCH_CHECK();
}

} // namespace pmg
