// Multigrid transfers between levels: polynomial (same mesh, degree pc -> pf;
// include/multigrid/portable_polynomial_transfer.h + BK1 batched kernels
// include/kernels/bk1_kokkos_kernels.h:462-1051) and geometric (same degree, one global
// refinement; include/multigrid/portable_geometric_transfer.h).  Both are "patch"
// transfers: every patch (fine cell for p, coarse cell for h) maps its coarse DoFs
// (Dirichlet entries dropped) through the tensor product of a 1D matrix onto its fine
// DoFs, each fine entry scaled by 1/(number of patches holding it), 0 when constrained.
#include <algorithm>

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

template <typename T> std::vector<T> cast(const std::vector<double> &v) {
  return std::vector<T>(v.begin(), v.end());
}

bool same_box_geometry(const pmg_box &a, const pmg_box &b) {
  for (int d = 0; d < 3; ++d)
    if (a.coarse[d] != b.coarse[d] || a.lo[d] != b.lo[d] || a.hi[d] != b.hi[d]) return false;
  return a.deform == b.deform && a.amp == b.amp && a.dirichlet_mask == b.dirichlet_mask;
}

} // namespace

void transfer_setup(pmg_transfer &t, const pmg_operator &coarse, const pmg_operator &fine) {
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
  // weights: 1 / multiplicity of the fine DoF over all patches, 0 when constrained
  std::vector<double> mult(t.n_fine, 0.0);
  for (uint32_t d : fidx) mult[d] += 1.0;
  for (int64_t i = 0; i < t.n_fine; ++i)
    mult[i] = (fine.num.constrained[i] || mult[i] == 0.0) ? 0.0 : 1.0 / mult[i];
  std::vector<double> w(fidx.size());
  for (size_t e = 0; e < fidx.size(); ++e) w[e] = mult[fidx[e]];
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
  t.grid = (int)std::max<int64_t>(1, std::min<int64_t>((t.n_patches + t.ppb - 1) / t.ppb, (int64_t)sms * 8));
  if (t.dtype == PMG_F64)
    PMG_CUDA(cudaFuncSetAttribute(transfer_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  else
    PMG_CUDA(cudaFuncSetAttribute(transfer_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
}

void transfer_apply(const pmg_transfer &t, int dir, void *dst, const void *src, cudaStream_t s) {
  PMG_REQUIRE(dst && src, "null vector");
  if (t.n_patches == 0) return;
  prof::Scope scope(dir == 0 ? "transfer_prolongate" : "transfer_restrict", s);
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
