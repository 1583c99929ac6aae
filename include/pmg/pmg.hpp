/*
 * pmg.hpp -- header-only C++ layer over the C ABI of libpmg_b200.so (pmg.h).
 *
 * The classes carry the member set of the reference's C++ interfaces, so a class deriving
 * from those interfaces forwards each virtual to one call here:
 *   pmg::LaplaceOperator<Number>  Portable::LaplaceOperatorBase<3,Number>
 *                                 (include/base/portable_laplace_operator_base.h:17-61)
 *   pmg::Transfer<Number>         Portable::MGTransferBase<3,number>
 *                                 (include/base/portable_mg_transfer_base.h:16-37)
 *   pmg::VCycle<Number>           Portable::VCycleMultigridBase<3,number>
 *                                 (include/base/portable_v_cycle_multigrid_base.h:18-27)
 * Vector arguments are any type with `Number *get_values()` (device memory, as
 * LinearAlgebra::distributed::Vector<Number, MemorySpace::Default> gives) and `size()`.
 * Failed calls throw pmg::Exception with the status and the library's message.  All work is
 * ordered on the stream given at construction (nullptr: the legacy default stream).
 */
#ifndef PMG_PMG_HPP
#define PMG_PMG_HPP

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "pmg/pmg.h"

namespace pmg {

class Exception : public std::runtime_error {
public:
  Exception(pmg_status s, const std::string &what) : std::runtime_error(what), status_(s) {}
  pmg_status status() const { return status_; }

private:
  pmg_status status_;
};

inline void check(pmg_status s) {
  if (s != PMG_OK) {
    char msg[1024];
    pmg_last_error(msg, sizeof(msg));
    throw Exception(s, std::string(pmg_status_string(s)) + ": " + msg);
  }
}

template <typename Number> constexpr int32_t dtype_of() {
  static_assert(std::is_same<Number, double>::value || std::is_same<Number, float>::value,
                "libpmg_b200 works on double or float vectors");
  return std::is_same<Number, double>::value ? PMG_F64 : PMG_F32;
}

/* The caller's discretisation of one level (pmg_operator_create_from_maps): the cell -> DoF
 * map with the 0xFFFFFFFF sentinel, the constrained DoFs and either G or the inverse Jacobian
 * with JxW, all host arrays. */
struct Discretisation {
  int64_t n_dofs = 0;
  std::vector<uint32_t> dof_indices;   // [cells][(degree+1)^3]
  std::vector<uint32_t> constrained;   // identity rows
  std::vector<double> G;               // [cells][6][nq^3], or empty
  std::vector<double> inv_jacobian;    // [cells][nq^3][3][3], with JxW, or empty
  std::vector<double> JxW;             // [cells][nq^3]
};

template <typename Number> class LaplaceOperator {
public:
  /* LaplaceOperatorBK3 on one of the library's box meshes. */
  LaplaceOperator(const pmg_box &box, int degree, int device = 0, void *stream = nullptr,
                  int32_t geometry = PMG_GEOMETRY_AUTO)
      : stream_(stream) {
    pmg_mesh *mesh = nullptr;
    check(pmg_mesh_create_box(&box, &mesh));
    mesh_.reset(mesh);
    pmg_operator_params p = params(degree, device);
    p.geometry = geometry;
    pmg_operator *op = nullptr;
    check(pmg_operator_create(mesh_.get(), &p, &op));
    op_.reset(op);
  }

  /* LaplaceOperatorBK3 on the caller's index map and geometry. */
  LaplaceOperator(const Discretisation &d, int degree, int device = 0, void *stream = nullptr)
      : stream_(stream) {
    const int64_t nm3 = int64_t(degree + 1) * (degree + 1) * (degree + 1);
    pmg_operator_maps m{};
    m.n_cells = nm3 > 0 ? int64_t(d.dof_indices.size()) / nm3 : 0;
    m.n_dofs = d.n_dofs;
    m.dof_indices = d.dof_indices.data();
    m.constrained = d.constrained.data();
    m.n_constrained = int64_t(d.constrained.size());
    if (!d.G.empty()) {
      m.geometry = PMG_MAPS_G;
      m.G = d.G.data();
    } else {
      m.geometry = PMG_MAPS_INVJAC;
      m.inv_jacobian = d.inv_jacobian.data();
      m.JxW = d.JxW.data();
    }
    pmg_operator_params p = params(degree, device);
    pmg_operator *op = nullptr;
    check(pmg_operator_create_from_maps(&m, &p, &op));
    op_.reset(op);
  }

  template <typename Vector> void vmult(Vector &dst, const Vector &src) const {
    check(pmg_operator_vmult(op_.get(), dst.get_values(), src.get_values(), stream_));
  }
  template <typename Vector> void Tvmult(Vector &dst, const Vector &src) const {
    check(pmg_operator_tvmult(op_.get(), dst.get_values(), src.get_values(), stream_));
  }
  template <typename Vector>
  void vmult_dummy(Vector &dst, const Vector &src, bool ghost_exchange_on, bool computation_on) const {
    check(pmg_operator_vmult_dummy(op_.get(), dst.get_values(), src.get_values(), ghost_exchange_on,
                                   computation_on, stream_));
  }
  /* dst += A_K src over the cells [cell_begin, cell_end); init sets dst as vmult does first
   * (the interior / boundary split of a sharded vmult). */
  template <typename Vector>
  void vmult_cells(Vector &dst, const Vector &src, int64_t cell_begin, int64_t cell_end, bool init) const {
    check(pmg_operator_vmult_cells(op_.get(), dst.get_values(), src.get_values(), cell_begin, cell_end, init,
                                   stream_));
  }
  int64_t n_cells() const {
    int64_t v = 0;
    check(pmg_operator_n_cells(op_.get(), &v));
    return v;
  }
  int cells_per_group() const {
    int32_t v = 0;
    check(pmg_operator_cells_per_group(op_.get(), &v));
    return v;
  }
  void compute_diagonal() { check(pmg_operator_compute_diagonal(op_.get(), stream_)); }
  /* get_matrix_diagonal_inverse(): copies the inverse diagonal into the caller's vector
   * (the storage behind the DiagonalMatrix the reference returns). */
  template <typename Vector> void copy_inverse_diagonal(Vector &dst) const {
    check(pmg_operator_copy_inverse_diagonal(op_.get(), dst.get_values(), stream_));
  }
  int64_t m() const {
    int64_t v = 0;
    check(pmg_operator_m(op_.get(), &v));
    return v;
  }
  int64_t n() const { return m(); }
  Number el(int64_t row, int64_t col) const {
    double v = 0;
    check(pmg_operator_el(op_.get(), row, col, &v));
    return Number(v);
  }
  pmg_operator *handle() const { return op_.get(); }
  void *stream() const { return stream_; }

private:
  static pmg_operator_params params(int degree, int device) {
    pmg_operator_params p{};
    p.degree = degree;
    p.dtype = dtype_of<Number>();
    p.geometry = PMG_GEOMETRY_AUTO;
    p.coeff_kind = PMG_COEFF_NONE;
    p.device = device;
    p.kind = PMG_OP_LAPLACE;
    return p;
  }
  struct MeshDel {
    void operator()(pmg_mesh *m) const { pmg_mesh_destroy(m); }
  };
  struct OpDel {
    void operator()(pmg_operator *o) const { pmg_operator_destroy(o); }
  };
  std::unique_ptr<pmg_mesh, MeshDel> mesh_;
  std::unique_ptr<pmg_operator, OpDel> op_;
  void *stream_ = nullptr;
};

template <typename Number> class Transfer {
public:
  /* reinit between two box-mesh levels (polynomial, geometric or DG <-> CG by the levels). */
  Transfer(const LaplaceOperator<Number> &coarse, const LaplaceOperator<Number> &fine) : stream_(fine.stream()) {
    pmg_transfer *t = nullptr;
    check(pmg_transfer_create(coarse.handle(), fine.handle(), &t));
    t_.reset(t);
  }
  /* reinit from the caller's patch maps (weights empty: 1 / multiplicity). */
  Transfer(const LaplaceOperator<Number> &coarse, const LaplaceOperator<Number> &fine, int32_t kind,
           const std::vector<uint32_t> &coarse_indices, const std::vector<uint32_t> &fine_indices,
           const std::vector<double> &weights = {})
      : stream_(fine.stream()) {
    const int64_t nc = coarse_nodes(coarse);
    pmg_transfer_maps m{};
    m.kind = kind;
    m.n_patches = nc > 0 ? int64_t(coarse_indices.size()) / (nc * nc * nc) : 0;
    m.coarse_indices = coarse_indices.data();
    m.fine_indices = fine_indices.data();
    m.weights = weights.empty() ? nullptr : weights.data();
    pmg_transfer *t = nullptr;
    check(pmg_transfer_create_from_maps(coarse.handle(), fine.handle(), &m, &t));
    t_.reset(t);
  }
  template <typename Vector> void prolongate_and_add(Vector &dst, const Vector &src) const {
    check(pmg_transfer_prolongate_and_add(t_.get(), dst.get_values(), src.get_values(), stream_));
  }
  template <typename Vector> void restrict_and_add(Vector &dst, const Vector &src) const {
    check(pmg_transfer_restrict_and_add(t_.get(), dst.get_values(), src.get_values(), stream_));
  }
  pmg_transfer *handle() const { return t_.get(); }

private:
  static int64_t coarse_nodes(const LaplaceOperator<Number> &coarse) {
    int32_t degree = 0, dtype = 0;
    check(pmg_operator_degree(coarse.handle(), &degree, &dtype));
    return degree + 1;
  }
  struct Del {
    void operator()(pmg_transfer *t) const { pmg_transfer_destroy(t); }
  };
  std::unique_ptr<pmg_transfer, Del> t_;
  void *stream_ = nullptr;
};

/* PreconditionChebyshev with the operator's inverse diagonal (deal.II's AdditionalData:
 * degree (<= 0: from the range), smoothing_range, eig_cg_n_iterations). */
template <typename Number> class Chebyshev {
public:
  Chebyshev(LaplaceOperator<Number> &op, int degree, double smoothing_range, int eig_cg_n_iterations)
      : stream_(op.stream()) {
    pmg_chebyshev_params p{degree, smoothing_range, eig_cg_n_iterations};
    pmg_chebyshev *c = nullptr;
    check(pmg_chebyshev_create(op.handle(), &p, &c));
    c_.reset(c);
  }
  template <typename Vector> void vmult(Vector &dst, const Vector &src) const {
    check(pmg_chebyshev_vmult(c_.get(), dst.get_values(), src.get_values(), stream_));
  }
  template <typename Vector> void step(Vector &dst, const Vector &src) const {
    check(pmg_chebyshev_step(c_.get(), dst.get_values(), src.get_values(), stream_));
  }
  pmg_chebyshev *handle() const { return c_.get(); }

private:
  struct Del {
    void operator()(pmg_chebyshev *c) const { pmg_chebyshev_destroy(c); }
  };
  std::unique_ptr<pmg_chebyshev, Del> c_;
  void *stream_ = nullptr;
};

/* VCycleMultigridBase::vmult over levels[0] (coarsest) .. levels.back() (finest); the
 * levels, transfers (transfers[0] unused) and smoothers are borrowed. */
template <typename Number> class VCycle {
public:
  VCycle(const std::vector<LaplaceOperator<Number> *> &levels, const std::vector<Transfer<Number> *> &transfers,
         const std::vector<Chebyshev<Number> *> &smoothers)
      : stream_(levels.empty() ? nullptr : levels.back()->stream()) {
    const size_t n = levels.size();
    if (transfers.size() != n || smoothers.size() != n)
      throw Exception(PMG_EINVAL, "VCycle: one transfer slot and one smoother per level");
    std::vector<pmg_operator *> ops(n);
    std::vector<pmg_transfer *> trs(n, nullptr);
    std::vector<pmg_chebyshev *> sms(n);
    for (size_t l = 0; l < n; ++l) {
      ops[l] = levels[l]->handle();
      if (l > 0) trs[l] = transfers[l]->handle();
      sms[l] = smoothers[l]->handle();
    }
    pmg_mg *mg = nullptr;
    check(pmg_mg_create(int32_t(n), ops.data(), trs.data(), sms.data(), &mg));
    mg_.reset(mg);
  }
  /* dst = V-cycle(src); the vectors may be of another precision than the levels (the FP64
   * outer CG of the mixed-precision solver, portable_multigrid_solver.h:185-191). */
  template <typename Vector> void vmult(Vector &dst, const Vector &src) const {
    using V = typename std::remove_pointer<decltype(dst.get_values())>::type;
    check(pmg_mg_vmult(mg_.get(), dst.get_values(), src.get_values(), dtype_of<typename std::remove_cv<V>::type>(),
                       stream_));
  }
  pmg_mg *handle() const { return mg_.get(); }

private:
  struct Del {
    void operator()(pmg_mg *m) const { pmg_mg_destroy(m); }
  };
  std::unique_ptr<pmg_mg, Del> mg_;
  void *stream_ = nullptr;
};

/* MultigridSolver::solve_cg: FP64 CG on A preconditioned by the V-cycle (nullptr: Jacobi). */
template <typename Vector, typename MG>
pmg_cg_info solve_cg(LaplaceOperator<double> &A, const MG *mg, Vector &x, const Vector &b, double reduce,
                     double abs_tol = 1e-16, int max_iterations = 100) {
  pmg_cg_info info{};
  check(pmg_cg_solve(A.handle(), mg ? mg->handle() : nullptr, x.get_values(), b.get_values(), reduce, abs_tol,
                     max_iterations, &info, A.stream()));
  return info;
}

} // namespace pmg

#endif /* PMG_PMG_HPP */
