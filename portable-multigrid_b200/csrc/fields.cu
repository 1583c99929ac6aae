// Launchers of the adjoint-path kernels (field_kernels.cuh) for every degree, and the
// coefficient interpolation between nested box meshes.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "field_kernels.cuh"
#include "fields.hpp"

namespace pmg {
namespace {

constexpr int kWarps = 4; // warps per block of the mass kernels

template <int N, typename T> kern::Tab<N, T> tab_of(const Tables1D &t) {
  kern::Tab<N, T> k;
  for (int a = 0; a < N * N; ++a) {
    k.S[a] = (T)t.S[a];
    k.SD[a] = (T)t.SD[a];
    k.D[a] = (T)t.D[a];
  }
  for (int a = 0; a < N; ++a) k.W[a] = (T)t.W[a];
  kern::fill_even_odd(k, t.S.data(), t.SD.data());
  return k;
}

template <int N, typename T> kern::Tab2<N, T> tab2_of(const Tables1D &t) {
  kern::Tab2<N, T> k;
  for (int a = 0; a < N * N; ++a) {
    k.S2[a] = (T)(t.S[a] * t.S[a]);
    k.SS[a] = (T)(t.S[a] * t.SD[a]);
    k.D2[a] = (T)(t.SD[a] * t.SD[a]);
  }
  for (int a = 0; a < N; ++a) k.W[a] = (T)t.W[a];
  return k;
}

// grid of a grid-stride kernel: all resident blocks of the device (occupancy computed once
// per device and kernel), at most one block per `per_block` groups
template <typename K> int resident_grid(K kernel, int threads, size_t smem, int64_t work_blocks) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, int> cache;
  int dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(dev, reinterpret_cast<const void *>(kernel));
    auto it = cache.find(key);
    if (it == cache.end()) {
      PMG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
      cache[key] = per_sm;
    } else {
      per_sm = it->second;
    }
  }
  int sms = 0;
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t resident = (int64_t)std::max(1, per_sm) * sms;
  return (int)std::max<int64_t>(1, std::min<int64_t>(work_blocks, resident));
}

template <int N, typename T> void mass_launch(const pmg_operator &op, const void *src, void *dst,
                                              cudaStream_t s) {
  constexpr int CPW = kern::Layout<N>::CPW, CS = kern::Stride<N>::CELL;
  const size_t smem = size_t(kWarps) * CPW * CS * sizeof(T);
  const int64_t blocks = (op.n_groups + kWarps - 1) / kWarps;
  const auto tab = tab_of<N, T>(cached_tables(op.degree));
  if (op.mass_geom == 1) {
    auto k = kern::mass_slab_kernel<N, T, 1>;
    const int grid = resident_grid(k, 32 * kWarps, smem, blocks);
    k<<<grid, 32 * kWarps, smem, s>>>(tab, static_cast<const T *>(src), static_cast<T *>(dst),
                                      op.idx.as<uint32_t>(), op.geo.as<T>(), nullptr, op.n_groups);
    op.launch_par[PMG_KERNEL_MASS] = (int64_t)grid * kWarps;
  } else {
    auto k = kern::mass_slab_kernel<N, T, 0>;
    const int grid = resident_grid(k, 32 * kWarps, smem, blocks);
    k<<<grid, 32 * kWarps, smem, s>>>(tab, static_cast<const T *>(src), static_cast<T *>(dst),
                                      op.idx.as<uint32_t>(), nullptr, op.coef.as<T>(), op.n_groups);
    op.launch_par[PMG_KERNEL_MASS] = (int64_t)grid * kWarps;
  }
  op.launch_units[PMG_KERNEL_MASS] = op.n_groups;
  PMG_LAUNCH_CHECK();
}

template <int N, typename T> void mass_diag_launch(const pmg_operator &op, void *diag, cudaStream_t s) {
  constexpr int CPW = kern::Layout<N>::CPW, CS = kern::Stride<N>::CELL;
  const size_t smem = size_t(kWarps) * CPW * CS * sizeof(T);
  const int64_t blocks = (op.n_groups + kWarps - 1) / kWarps;
  const auto tab = tab2_of<N, T>(cached_tables(op.degree));
  if (op.mass_geom == 1) {
    auto k = kern::mass_diag_slab_kernel<N, T, 1>;
    const int grid = resident_grid(k, 32 * kWarps, smem, blocks);
    k<<<grid, 32 * kWarps, smem, s>>>(tab, static_cast<T *>(diag), op.idx.as<uint32_t>(), op.geo.as<T>(),
                                      nullptr, op.n_groups);
  } else {
    auto k = kern::mass_diag_slab_kernel<N, T, 0>;
    const int grid = resident_grid(k, 32 * kWarps, smem, blocks);
    k<<<grid, 32 * kWarps, smem, s>>>(tab, static_cast<T *>(diag), op.idx.as<uint32_t>(), nullptr,
                                      op.coef.as<T>(), op.n_groups);
  }
  PMG_LAUNCH_CHECK();
}

template <int N, typename T, int GEOM>
void qp_form_geom(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                  cudaStream_t s) {
  constexpr int CPW = kern::Layout<N>::CPW, CS = kern::Stride<N>::CELL;
  constexpr int W = 2; // warps per block
  const size_t smem = size_t(W) * 6 * CPW * CS * sizeof(T);
  auto k = kern::qp_form_slab_kernel<N, T, GEOM>;
  const int grid = resident_grid(k, 32 * W, smem, (op.n_groups + W - 1) / W);
  k<<<grid, 32 * W, smem, s>>>(tab_of<N, T>(cached_tables(op.degree)), static_cast<const T *>(u),
                               static_cast<const T *>(v), out, op.idx.as<uint32_t>(), op.geo.as<T>(),
                               op.coef.as<T>(), op.n_groups, op.n_cells, alpha);
  PMG_LAUNCH_CHECK();
  op.launch_units[PMG_KERNEL_QP_FORM] = op.n_groups;
  op.launch_par[PMG_KERNEL_QP_FORM] = (int64_t)grid * W;
}

template <int N, typename T>
void qp_form_launch(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                    cudaStream_t s) {
  PMG_REQUIRE(op.geometry != PMG_GEOMETRY_INVJAC, "the per-point form needs the G or affine geometry layout");
  if (op.geometry == PMG_GEOMETRY_FULL) qp_form_geom<N, T, 0>(op, u, v, alpha, out, s);
  else if (op.has_coeff_values) qp_form_geom<N, T, 2>(op, u, v, alpha, out, s);
  else qp_form_geom<N, T, 1>(op, u, v, alpha, out, s);
}

// compile-time degree from the runtime one
template <template <int, typename> class F, typename... A> void by_degree(const pmg_operator &op, A... a) {
  const bool d = op.dtype == PMG_F64;
  switch (op.degree) {
  case 1: d ? F<2, double>::run(op, a...) : F<2, float>::run(op, a...); break;
  case 2: d ? F<3, double>::run(op, a...) : F<3, float>::run(op, a...); break;
  case 3: d ? F<4, double>::run(op, a...) : F<4, float>::run(op, a...); break;
  case 4: d ? F<5, double>::run(op, a...) : F<5, float>::run(op, a...); break;
  case 5: d ? F<6, double>::run(op, a...) : F<6, float>::run(op, a...); break;
  case 6: d ? F<7, double>::run(op, a...) : F<7, float>::run(op, a...); break;
  default: fail(PMG_EINVAL, "degree must be in [1,6]");
  }
}
template <int N, typename T> struct MassF {
  static void run(const pmg_operator &op, const void *src, void *dst, cudaStream_t s) {
    mass_launch<N, T>(op, src, dst, s);
  }
};
template <int N, typename T> struct MassDiagF {
  static void run(const pmg_operator &op, void *diag, cudaStream_t s) { mass_diag_launch<N, T>(op, diag, s); }
};
template <int N, typename T> struct QpFormF {
  static void run(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                  cudaStream_t s) {
    qp_form_launch<N, T>(op, u, v, alpha, out, s);
  }
};

struct Gauss8 {
  double x[8];
};

// One thread per target point: the source cell containing it (nested lattices, ratio r per
// axis), the tensor Lagrange weights through the source cell's Gauss points, and
// exp(sum of weights * log(source values)).
__global__ void coef_interp_kernel(const double *__restrict__ src, const int32_t *__restrict__ src_lut,
                                   int64_t ns0, int64_t ns1, int64_t ns2, int nqs, const Gauss8 gs,
                                   const int32_t *__restrict__ dst_xyz, int64_t n_dst_cells, int nqd,
                                   const Gauss8 gd, int64_t ratio, double *__restrict__ dst) {
  const int nqd3 = nqd * nqd * nqd, nqs3 = nqs * nqs * nqs;
  const int64_t n = n_dst_cells * nqd3;
  const int64_t ns[3] = {ns0, ns1, ns2};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / nqd3;
    const int q = (int)(t - c * nqd3);
    const int qd[3] = {q % nqd, (q / nqd) % nqd, q / (nqd * nqd)};
    int64_t sc[3];
    double L[3][8];
    for (int d = 0; d < 3; ++d) {
      const double X = ((double)dst_xyz[3 * c + d] + gd.x[qd[d]]) * (double)ratio;
      int64_t si = (int64_t)floor(X);
      if (si > ns[d] - 1) si = ns[d] - 1;
      sc[d] = si;
      const double xi = X - (double)si;
      for (int a = 0; a < nqs; ++a) {
        double l = 1.0;
        for (int b = 0; b < nqs; ++b)
          if (b != a) l *= (xi - gs.x[b]) / (gs.x[a] - gs.x[b]);
        L[d][a] = l;
      }
    }
    const int64_t cell = src_lut[(sc[2] * ns[1] + sc[1]) * ns[0] + sc[0]];
    const double *sv = src + cell * nqs3;
    double acc = 0.0;
    for (int k = 0; k < nqs; ++k)
      for (int j = 0; j < nqs; ++j) {
        const double ljk = L[1][j] * L[2][k];
        for (int i = 0; i < nqs; ++i) acc += L[0][i] * ljk * log(sv[(k * nqs + j) * nqs + i]);
      }
    dst[t] = exp(acc);
  }
}

} // namespace

const Tables1D &cached_tables(int degree) {
  static std::mutex mu;
  static Tables1D tabs[kMaxDegree + 1];
  static bool ready[kMaxDegree + 1] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (!ready[degree]) {
    tabs[degree] = make_tables(degree, degree + 1);
    ready[degree] = true;
  }
  return tabs[degree];
}

void mass_vmult_cells(const pmg_operator &op, const void *src, void *dst, cudaStream_t s) {
  by_degree<MassF>(op, src, dst, s);
}

void mass_diagonal_cells(const pmg_operator &op, void *diag, cudaStream_t s) {
  by_degree<MassDiagF>(op, diag, s);
}

void qp_form_cells(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                   cudaStream_t s) {
  by_degree<QpFormF>(op, u, v, alpha, out, s);
}

void coefficient_interpolate(const pmg_operator &src, const pmg_operator &dst, double *dst_values,
                             cudaStream_t s) {
  const auto &bs = src.mesh.box, &bd = dst.mesh.box;
  for (int d = 0; d < 3; ++d) {
    PMG_REQUIRE(bs.coarse[d] == bd.coarse[d] && bs.lo[d] == bd.lo[d] && bs.hi[d] == bd.hi[d],
                "coefficient interpolation needs the same box on both meshes");
  }
  PMG_REQUIRE(bs.refine >= bd.refine, "the source mesh must be at least as fine as the target");
  PMG_REQUIRE(src.coef_qp.get() != nullptr, "the source operator has no coefficient values");
  const int64_t ratio = int64_t(1) << (bs.refine - bd.refine);
  if (ratio == 1 && src.nq == dst.nq) { // the same points: an exact copy
    PMG_CUDA(cudaMemcpyAsync(dst_values, src.coef_qp.get(), sizeof(double) * dst.n_cells * dst.nq * dst.nq * dst.nq,
                             cudaMemcpyDeviceToDevice, s));
    return;
  }
  Gauss8 gs{}, gd{};
  const Tables1D &ts = cached_tables(src.degree), &td = cached_tables(dst.degree);
  for (int q = 0; q < src.nq; ++q) gs.x[q] = ts.xg[q];
  for (int q = 0; q < dst.nq; ++q) gd.x[q] = td.xg[q];
  const int64_t n = dst.n_cells * dst.nq * dst.nq * dst.nq;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)dst.sms * 32));
  coef_interp_kernel<<<grid, 256, 0, s>>>(src.coef_qp.as<double>(), src.cell_lut.as<int32_t>(), src.mesh.n[0],
                                          src.mesh.n[1], src.mesh.n[2], src.nq, gs, dst.cell_xyz.as<int32_t>(),
                                          dst.n_cells, dst.nq, gd, ratio, dst_values);
  PMG_LAUNCH_CHECK();
}

} // namespace pmg
