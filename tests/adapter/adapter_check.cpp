// Compiles the header-only C++ layer (include/pmg/pmg.hpp) against the C ABI the way a
// maintainer of the reference would use it, with a stand-in for deal.II's device vector
// (get_values(), size()), and checks on the GPU:
//  1. an operator built from the caller's maps (here the box operator's own maps with the
//     DoF numbers reversed and the cells listed backwards) gives the box operator's vmult,
//     also when applied in two cell passes (vmult_cells, the split of a sharded vmult);
//  2. a mixed-precision ph-multigrid CG solve through LaplaceOperator / Transfer / Chebyshev /
//     VCycle / solve_cg converges.
// Prints "adapter ok" and exits 0 on success.  Without a GPU it exits 2 after linking.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "pmg/pmg.hpp"

template <typename Number> struct DeviceVector {
  explicit DeviceVector(size_t n) : n_(n) {
    if (cudaMalloc(&p_, n * sizeof(Number)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
    cudaMemset(p_, 0, n * sizeof(Number));
  }
  ~DeviceVector() { cudaFree(p_); }
  DeviceVector(const DeviceVector &) = delete;
  DeviceVector &operator=(const DeviceVector &) = delete;
  Number *get_values() const { return p_; }
  size_t size() const { return n_; }
  void upload(const std::vector<Number> &h) { cudaMemcpy(p_, h.data(), n_ * sizeof(Number), cudaMemcpyHostToDevice); }
  std::vector<Number> download() const {
    std::vector<Number> h(n_);
    cudaMemcpy(h.data(), p_, n_ * sizeof(Number), cudaMemcpyDeviceToHost);
    return h;
  }

private:
  Number *p_ = nullptr;
  size_t n_ = 0;
};

static pmg_box box(int refine) {
  pmg_box b{};
  b.coarse[0] = b.coarse[1] = b.coarse[2] = 1;
  b.refine = refine;
  b.hi[0] = b.hi[1] = b.hi[2] = 1.0;
  b.deform = 1;
  b.amp = 0.1;
  b.dirichlet_mask = 0x3F;
  return b;
}

int main() {
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    std::printf("adapter: no CUDA device, linked only\n");
    return 2;
  }
  try {
    // 1. caller maps against the box operator
    const int p = 3, nm3 = (p + 1) * (p + 1) * (p + 1);
    pmg::LaplaceOperator<double> A_box(box(2), p, 0, nullptr, PMG_GEOMETRY_FULL);
    const int64_t N = A_box.m();
    int64_t C = 0;
    pmg::check(pmg_operator_n_cells(A_box.handle(), &C));
    std::vector<uint32_t> idx(C * nm3);
    std::vector<uint8_t> cons(N);
    std::vector<double> G(C * 6 * nm3);
    pmg::check(pmg_operator_copy_dof_indices(A_box.handle(), idx.data()));
    pmg::check(pmg_operator_copy_constrained(A_box.handle(), cons.data()));
    pmg::check(pmg_operator_copy_geometry(A_box.handle(), G.data()));
    pmg::Discretisation d;
    d.n_dofs = N;
    auto perm = [N](uint32_t i) { return uint32_t(N - 1 - i); };
    for (int64_t c = C - 1; c >= 0; --c) {
      for (int l = 0; l < nm3; ++l) {
        const uint32_t v = idx[c * nm3 + l];
        d.dof_indices.push_back(v == PMG_INVALID_INDEX ? v : perm(v));
      }
      d.G.insert(d.G.end(), G.begin() + c * 6 * nm3, G.begin() + (c + 1) * 6 * nm3);
    }
    for (int64_t i = 0; i < N; ++i)
      if (cons[i]) d.constrained.push_back(perm((uint32_t)i));
    pmg::LaplaceOperator<double> A_maps(d, p);
    std::vector<double> x(N), xp(N);
    uint64_t s = 1234;
    for (int64_t i = 0; i < N; ++i) {
      s = s * 6364136223846793005ULL + 1442695040888963407ULL;
      x[i] = double(s >> 11) * 0x1.0p-53 * 2.0 - 1.0;
      xp[perm((uint32_t)i)] = x[i];
    }
    DeviceVector<double> src(N), srcp(N), dst(N), dstp(N);
    src.upload(x);
    srcp.upload(xp);
    A_box.vmult(dst, src);
    A_maps.vmult(dstp, srcp);
    const auto y = dst.download(), yp = dstp.download();
    double err = 0, ref = 0;
    for (int64_t i = 0; i < N; ++i) {
      err = std::fmax(err, std::fabs(y[i] - yp[perm((uint32_t)i)]));
      ref = std::fmax(ref, std::fabs(y[i]));
    }
    if (!(err <= 1e-12 * ref)) {
      std::printf("adapter: caller-map vmult differs: %.3e of %.3e\n", err, ref);
      return 1;
    }
    // 1b. the same product in two cell passes, as a sharded vmult splits it around the ghost
    //     update: the first cells with init, the rest added
    {
      const int64_t split = (A_maps.n_cells() / 2 / A_maps.cells_per_group()) * A_maps.cells_per_group();
      DeviceVector<double> dsplit(N);
      A_maps.vmult_cells(dsplit, srcp, 0, split, true);
      A_maps.vmult_cells(dsplit, srcp, split, A_maps.n_cells(), false);
      const auto ys = dsplit.download();
      double e2 = 0;
      for (int64_t i = 0; i < N; ++i) e2 = std::fmax(e2, std::fabs(ys[i] - yp[i]));
      if (!(e2 <= 1e-13 * ref)) {
        std::printf("adapter: split vmult differs: %.3e of %.3e\n", e2, ref);
        return 1;
      }
    }
    // 2. ph-multigrid: Q1 on 1^3, 2^3, 4^3 cells, then Q2, Q3 on 4^3; FP32 levels, FP64 CG
    std::vector<std::unique_ptr<pmg::LaplaceOperator<float>>> lv;
    for (int r = 0; r <= 2; ++r) lv.emplace_back(new pmg::LaplaceOperator<float>(box(r), 1));
    lv.emplace_back(new pmg::LaplaceOperator<float>(box(2), 2));
    lv.emplace_back(new pmg::LaplaceOperator<float>(box(2), 3));
    std::vector<std::unique_ptr<pmg::Transfer<float>>> tr(lv.size());
    std::vector<std::unique_ptr<pmg::Chebyshev<float>>> sm(lv.size());
    std::vector<pmg::LaplaceOperator<float> *> lp;
    std::vector<pmg::Transfer<float> *> tp;
    std::vector<pmg::Chebyshev<float> *> sp;
    for (size_t l = 0; l < lv.size(); ++l) {
      if (l > 0) tr[l].reset(new pmg::Transfer<float>(*lv[l - 1], *lv[l]));
      sm[l].reset(l == 0 ? new pmg::Chebyshev<float>(*lv[0], 0, 1e-3, (int)lv[0]->m())
                         : new pmg::Chebyshev<float>(*lv[l], 5, 15.0, 10));
      lp.push_back(lv[l].get());
      tp.push_back(tr[l].get());
      sp.push_back(sm[l].get());
    }
    pmg::VCycle<float> mg(lp, tp, sp);
    DeviceVector<double> b(N), u(N);
    pmg::check(pmg_operator_assemble_rhs(A_box.handle(), 0, 0, b.get_values(), nullptr));
    const pmg_cg_info info = pmg::solve_cg(A_box, &mg, u, b, 1e-10);
    if (!info.converged || info.iterations > 20) {
      std::printf("adapter: CG did not converge (%d iterations)\n", info.iterations);
      return 1;
    }
    std::printf("adapter ok: caller-map vmult rel err %.2e, CG %d iterations, reduction %.3e\n", err / ref,
                info.iterations, info.reduction_per_step);
  } catch (const pmg::Exception &e) {
    std::printf("adapter: %s\n", e.what());
    return 1;
  }
  return 0;
}
