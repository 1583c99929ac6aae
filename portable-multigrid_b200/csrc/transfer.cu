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

// ---- transfer maps and weights on the device (setup) ----
// out[e] = the sentinel where plain[e] is one or a constrained DoF, else plain[e]
__global__ void sentinel_map_kernel(const uint32_t *__restrict__ plain, const uint8_t *__restrict__ cons, int64_t n,
                                    uint32_t *__restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t d = plain[e];
    out[e] = (d == kInvalid || cons[d]) ? kInvalid : d;
  }
}

// h-transfer patch of coarse cell c: the (2p+1)^3 fine nodes from 2p * (cell coordinates) on
__global__ void h_patch_kernel(const int32_t *__restrict__ coarse_xyz, int64_t n_patches, int p,
                               const uint32_t *__restrict__ fine_lattice, int64_t L0, int64_t L1,
                               uint32_t *__restrict__ fidx) {
  const int nf = 2 * p + 1, nf3 = nf * nf * nf;
  const int64_t total = n_patches * nf3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / nf3;
    const int l = (int)(t - c * nf3);
    const int i = l % nf, j = (l / nf) % nf, k = l / (nf * nf);
    const int64_t x = 2LL * p * coarse_xyz[3 * c] + i, y = 2LL * p * coarse_xyz[3 * c + 1] + j,
                  z = 2LL * p * coarse_xyz[3 * c + 2] + k;
    fidx[t] = fine_lattice[(z * L1 + y) * L0 + x];
  }
}

__global__ void multiplicity_kernel(const uint32_t *__restrict__ fidx, int64_t n, uint32_t *__restrict__ cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + fidx[e], 1u);
}

// w[e] = 1 / (patches holding fine DoF fidx[e]), 0 on constrained fine DoFs
template <typename T>
__global__ void weights_kernel(const uint32_t *__restrict__ fidx, int64_t n, const uint32_t *__restrict__ cnt,
                               const uint8_t *__restrict__ cons, T *__restrict__ w) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t d = fidx[e];
    const uint32_t m = cnt[d];
    w[e] = (cons[d] || m == 0) ? T(0) : (T)(1.0 / (double)m);
  }
}

int setup_grid(int64_t n, int sms) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 32));
}

// the 1D matrix, the weights (1 / multiplicity of the fine DoF over all patches, 0 when
// constrained, unless given), launch parameters; t.coarse_idx and t.fine_idx are set
void transfer_finish(pmg_transfer &t, const pmg_operator &fine, const std::vector<double> &P,
                     const double *given_weights) {
  int sms = 0;
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, t.device));
  t.sms = sms;
  const int64_t nf3 = (int64_t)t.nf * t.nf * t.nf, n_w = t.n_patches * nf3;
  t.P_host = P;
  if (t.dtype == PMG_F64) t.P1d = upload(P);
  else t.P1d = upload(cast<float>(P));
  if (given_weights) {
    std::vector<double> w(given_weights, given_weights + n_w);
    if (t.dtype == PMG_F64) t.weights = upload(w);
    else t.weights = upload(cast<float>(w));
  } else {
    t.weights.allocate(dtype_size(t.dtype) * std::max<int64_t>(1, n_w));
    if (n_w > 0) {
      DeviceBuffer cnt(sizeof(uint32_t) * std::max<int64_t>(1, t.n_fine));
      PMG_CUDA(cudaMemset(cnt.get(), 0, cnt.bytes()));
      multiplicity_kernel<<<setup_grid(n_w, sms), 256>>>(t.fine_idx.as<uint32_t>(), n_w, cnt.as<uint32_t>());
      PMG_LAUNCH_CHECK();
      if (t.dtype == PMG_F64)
        weights_kernel<double><<<setup_grid(n_w, sms), 256>>>(t.fine_idx.as<uint32_t>(), n_w, cnt.as<uint32_t>(),
                                                              fine.dcons.as<uint8_t>(), t.weights.as<double>());
      else
        weights_kernel<float><<<setup_grid(n_w, sms), 256>>>(t.fine_idx.as<uint32_t>(), n_w, cnt.as<uint32_t>(),
                                                             fine.dcons.as<uint8_t>(), t.weights.as<float>());
      PMG_LAUNCH_CHECK();
      PMG_CUDA(cudaDeviceSynchronize()); // cnt is freed on return
    }
  }
  const size_t s = dtype_size(t.dtype);
  t.ppb = (int)std::max<size_t>(1, (32 * 1024) / (3 * nf3 * s));
  t.smem = s * (((t.nc * t.nf + 3) & ~3) + (size_t)t.ppb * 3 * nf3);
  t.patch_kernels = patch_kernels_enabled();
  t.grid = (int)std::max<int64_t>(1, std::min<int64_t>((t.n_patches + t.ppb - 1) / t.ppb, (int64_t)sms * 8));
  if (t.dtype == PMG_F64)
    PMG_CUDA(cudaFuncSetAttribute(transfer_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  else
    PMG_CUDA(cudaFuncSetAttribute(transfer_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
}

// coarse map with the sentinel from the coarse operator's device numbering
void coarse_map_from(pmg_transfer &t, const pmg_operator &coarse, const uint32_t *plain, int64_t n) {
  t.coarse_idx.allocate(sizeof(uint32_t) * std::max<int64_t>(1, n));
  if (n == 0) return;
  sentinel_map_kernel<<<setup_grid(n, t.sms > 0 ? t.sms : 148), 256>>>(plain, coarse.dcons.as<uint8_t>(), n,
                                                                      t.coarse_idx.as<uint32_t>());
  PMG_LAUNCH_CHECK();
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
  PMG_CUDA(cudaDeviceGetAttribute(&t.sms, cudaDevAttrMultiProcessorCount, t.device));
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
  const size_t n_c = (size_t)m.n_patches * nc3, n_f = (size_t)m.n_patches * nf3;
  for (size_t e = 0; e < n_c; ++e) {
    const uint32_t d = m.coarse_indices[e];
    if (d != kInvalid && (int64_t)d >= t.n_coarse)
      fail(PMG_EBOUNDS, "coarse_indices[" + std::to_string(e) + "] = " + std::to_string(d) + " >= " +
                            std::to_string(t.n_coarse));
  }
  for (size_t e = 0; e < n_f; ++e)
    if ((int64_t)m.fine_indices[e] >= t.n_fine)
      fail(PMG_EBOUNDS, "fine_indices[" + std::to_string(e) + "] = " + std::to_string(m.fine_indices[e]) + " >= " +
                            std::to_string(t.n_fine));
  // caller maps: coarse entries naming constrained coarse DoFs become the sentinel
  DeviceBuffer craw = upload(std::vector<uint32_t>(m.coarse_indices, m.coarse_indices + n_c));
  coarse_map_from(t, coarse, craw.as<uint32_t>(), (int64_t)n_c);
  t.fine_idx = upload(std::vector<uint32_t>(m.fine_indices, m.fine_indices + n_f));
  PMG_CUDA(cudaDeviceSynchronize()); // craw is freed on return
  transfer_finish(t, fine, P, m.weights);
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
  PMG_CUDA(cudaDeviceGetAttribute(&t.sms, cudaDevAttrMultiProcessorCount, t.device));
  const int pc = coarse.degree, pf = fine.degree;
  const int64_t cnm3 = (int64_t)(pc + 1) * (pc + 1) * (pc + 1);
  std::vector<double> P;
  if (fine.kind == PMG_OP_DG_SIPG || coarse.mesh.box.refine == fine.mesh.box.refine) {
    if (fine.kind == PMG_OP_DG_SIPG) {
      // DG <-> CG at equal degree (ContinuousTransfer): identity on every cell
      PMG_REQUIRE(coarse.kind == PMG_OP_LAPLACE, "the coarse level of a DG transfer must be continuous");
      PMG_REQUIRE(pc == pf && coarse.mesh.box.refine == fine.mesh.box.refine,
                  "DG <-> CG transfer needs equal degrees on the same mesh");
      t.kind = 2;
      t.nc = t.nf = pc + 1;
      P.assign(t.nc * t.nf, 0.0);
      for (int i = 0; i < t.nc; ++i) P[i * t.nf + i] = 1.0;
    } else {
      PMG_REQUIRE(coarse.kind == PMG_OP_LAPLACE, "a DG level can only be the finest level of a transfer");
      PMG_REQUIRE(pc < pf, "polynomial transfer needs degree_coarse < degree_fine");
      t.kind = 0;
      t.nc = pc + 1;
      t.nf = pf + 1;
      P = p_transfer_matrix(pc, pf);
    }
    // one patch per cell of the common mesh: the coarse map with the sentinel, the fine map
    t.n_patches = fine.n_cells;
    coarse_map_from(t, coarse, coarse.dplain.as<uint32_t>(), t.n_patches * cnm3);
    const int64_t n_f = t.n_patches * t.nf * t.nf * t.nf;
    t.fine_idx.allocate(sizeof(uint32_t) * std::max<int64_t>(1, n_f));
    if (n_f > 0)
      PMG_CUDA(cudaMemcpy(t.fine_idx.get(), fine.dplain.get(), sizeof(uint32_t) * n_f, cudaMemcpyDeviceToDevice));
  } else {
    PMG_REQUIRE(fine.mesh.box.refine == coarse.mesh.box.refine + 1,
                "geometric transfer needs the fine mesh refined exactly once more");
    PMG_REQUIRE(pc == pf, "geometric transfer needs equal degrees");
    PMG_REQUIRE(fine.dlattice.get() != nullptr, "fine operator has no node lattice");
    const int p = pc;
    t.kind = 1;
    t.nc = p + 1;
    t.nf = 2 * p + 1;
    t.n_patches = coarse.n_cells;
    P = h_transfer_matrix(p);
    coarse_map_from(t, coarse, coarse.dplain.as<uint32_t>(), t.n_patches * cnm3);
    const int64_t n_f = t.n_patches * t.nf * t.nf * t.nf;
    t.fine_idx.allocate(sizeof(uint32_t) * std::max<int64_t>(1, n_f));
    if (n_f > 0) {
      h_patch_kernel<<<setup_grid(n_f, t.sms), 256>>>(coarse.cell_xyz.as<int32_t>(), t.n_patches, p,
                                                       fine.dlattice.as<uint32_t>(), fine.num.L[0], fine.num.L[1],
                                                       t.fine_idx.as<uint32_t>());
      PMG_LAUNCH_CHECK();
    }
  }
  transfer_finish(t, fine, P, nullptr);
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
