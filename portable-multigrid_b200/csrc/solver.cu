// Chebyshev-Jacobi smoother, V-cycle and preconditioned CG, orchestrated on the host over
// the device kernels.  The algorithms restate deal.II's PreconditionChebyshev and SolverCG
// as the reference configures them (tests/poisson_cube_bk3/program.cc:474-515) and the
// reference's multigrid driver (tests/common/portable_multigrid_solver.h:147-271,
// include/multigrid/portable_v_cycle_multigrid.h:163-206).
#include <cmath>
#include <cstdlib>
#include <vector>

#include "pmg_internal.hpp"
#include "solver.hpp"
#include "transfer.hpp"
#include "vector_ops.hpp"

namespace pmg {
namespace {

int sturm_count(const std::vector<double> &a, const std::vector<double> &b, double x) {
  int cnt = 0;
  double d = 1.0;
  for (size_t i = 0; i < a.size(); ++i) {
    d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
    if (d == 0.0) d = -1e-300;
    if (d < 0) ++cnt;
  }
  return cnt;
}

// extreme eigenvalue of a symmetric tridiagonal matrix by Sturm-sequence bisection
double tridiag_extreme(const std::vector<double> &a, const std::vector<double> &b, bool largest) {
  const size_t n = a.size();
  double lo = 1e300, hi = -1e300;
  for (size_t i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  const int target = largest ? (int)n : 1;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (sturm_count(a, b, mid) >= target) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

void check_finite(double v, const char *what) {
  if (!std::isfinite(v)) fail(PMG_ENONFINITE, std::string("non-finite value in ") + what);
}

} // namespace

void chebyshev_setup(pmg_chebyshev &c, pmg_operator &op, const pmg_chebyshev_params &prm) {
  PMG_REQUIRE(prm.smoothing_range > 0, "smoothing_range must be positive");
  PMG_REQUIRE(prm.eig_cg_n_iterations >= 0, "eig_cg_n_iterations must be >= 0");
  c.op = &op;
  c.device = op.device;
  c.degree = prm.degree;
  c.requested_degree = prm.degree;
  c.range = prm.smoothing_range;
  c.eig_its = prm.eig_cg_n_iterations;
  const size_t bytes = dtype_size(op.dtype) * op.n_dofs;
  PMG_CUDA(cudaSetDevice(op.device));
  c.xo.allocate(bytes);
  c.Ax.allocate(bytes);
  if (!op.has_diag) {
    operator_compute_inverse_diagonal(op, nullptr);
    PMG_CUDA(cudaDeviceSynchronize());
  }
}

// deal.II PreconditionChebyshev::estimate_eigenvalues: at most eig_its CG steps (tolerance
// 1e-10) from x = 0 on v_i = (i mod 11) - mean with the Jacobi preconditioner; Lanczos
// matrix from the CG coefficients with a one-step lag; max scaled by 1.2; interval
// [alpha, max] with alpha = max/range (range > 1) or min(0.9 max, min); invalid degree
// chosen by the Chebyshev error bound for the target `range`.
void chebyshev_estimate(pmg_chebyshev &c, cudaStream_t s) {
  pmg_operator &op = *c.op;
  const int dt = op.dtype;
  const int64_t N = op.n_dofs;
  const size_t bytes = dtype_size(dt) * N;
  // work vectors: temporary for a first estimate; a smoother that is estimated again (new
  // coefficients) keeps them, so repeated estimates allocate nothing
  std::vector<DeviceBuffer> tmp;
  std::vector<DeviceBuffer> &w = c.generation > 0 ? c.est_work : tmp;
  if (w.size() != 5 || w[0].bytes() != bytes) {
    w.clear();
    for (int i = 0; i < 5; ++i) w.emplace_back(bytes);
  }
  DeviceBuffer &x = w[0], &r = w[1], &z = w[2], &p = w[3], &v = w[4];
  PMG_CUDA(cudaMemsetAsync(x.get(), 0, bytes, s));
  vec::fill_mod11(r.get(), dt, N, s);
  std::vector<double> diag, offd;
  double res = std::sqrt(vec::dot(r.get(), r.get(), dt, N, s));
  int it = 0;
  if (!(res <= 1e-10) && c.eig_its > 0) {
    double rho = vec::jacobi_dot(z.get(), op.inv_diag.get(), r.get(), dt, N, s);
    double rho_old = rho, alpha = 0, prev_alpha = 0, beta = 0, eig_beta_alpha = 0;
    while (true) {
      ++it;
      if (it > 1) {
        beta = rho / rho_old;
        vec::xpay(p.get(), z.get(), beta, dt, N, s);
      } else {
        PMG_CUDA(cudaMemcpyAsync(p.get(), z.get(), bytes, cudaMemcpyDeviceToDevice, s));
      }
      operator_vmult(op, v.get(), p.get(), s);
      prev_alpha = alpha;
      const double pv = vec::dot(p.get(), v.get(), dt, N, s);
      check_finite(pv, "Chebyshev eigenvalue estimate");
      alpha = rho / pv;
      res = std::sqrt(vec::cg_update(x.get(), r.get(), p.get(), v.get(), alpha, dt, N, s));
      rho_old = rho;
      rho = vec::jacobi_dot(z.get(), op.inv_diag.get(), r.get(), dt, N, s);
      if (it > 1) {
        diag.push_back(1.0 / prev_alpha + eig_beta_alpha);
        eig_beta_alpha = beta / prev_alpha;
        offd.push_back(std::sqrt(beta) / prev_alpha);
      }
      if (it >= c.eig_its || res <= 1e-10) break;
    }
  }
  c.cg_its = it;
  if (diag.empty()) {
    c.min_ev = c.max_ev = 1.0;
  } else {
    c.min_ev = tridiag_extreme(diag, offd, false);
    c.max_ev = 1.2 * tridiag_extreme(diag, offd, true);
  }
  const double alpha_ev = c.range > 1.0 ? c.max_ev / c.range : std::min(0.9 * c.max_ev, c.min_ev);
  if (c.requested_degree <= 0) {
    const double actual = c.max_ev / alpha_ev;
    const double sigma = (1.0 - std::sqrt(1.0 / actual)) / (1.0 + std::sqrt(1.0 / actual));
    const double eps = c.range;
    c.degree = 1 + (int)(std::log(1.0 / eps + std::sqrt(1.0 / eps / eps - 1.0)) / std::log(1.0 / sigma));
  }
  c.delta = (c.max_ev - alpha_ev) * 0.5;
  c.theta = (c.max_ev + alpha_ev) * 0.5;
  c.estimated = true;
  ++c.generation;
  PMG_CUDA(cudaStreamSynchronize(s)); // the work vectors are freed on return
}

// Chebyshev iteration of the first kind: vmult from x = 0 (degree-1 products), step from dst
// (degree products); x_{k+1} = x_k + f1 (x_k - x_{k-1}) + f2 D^{-1}(b - A x_k).  The iterates
// alternate between dst and the work vector xo, each update written over the previous
// iterate (one vector written per step); the first iterate goes where the parity of the
// remaining steps puts the last one into dst.  Per element the arithmetic is that of the
// two-vector form, so results are bit-identical to it.
void chebyshev_apply(pmg_chebyshev &c, void *dst, const void *src, bool from_zero, cudaStream_t s) {
  if (!c.estimated) chebyshev_estimate(c, s);
  pmg_operator &op = *c.op;
  const int dt = op.dtype;
  const int64_t N = op.n_dofs;
  const bool more = !(c.degree < 2 || std::fabs(c.delta) < 1e-40);
  const int d = more ? c.degree : 1; // iterates after x_0
  void *const A = dst, *const B = c.xo.get();
  void *cur = nullptr, *prev = nullptr; // x_k and x_{k-1} (null: x_{k-1} = 0)
  if (from_zero) {
    cur = ((d - 1) % 2 == 0) ? A : B;
    vec::cheb_init(cur, nullptr, src, op.inv_diag.get(), 1.0 / c.theta, dt, N, s);
  } else {
    operator_vmult(op, c.Ax.get(), dst, s);
    if (d % 2 == 0) { // x_1 into xo, x_0 stays in dst as the previous iterate
      vec::cheb_first_step_into(B, A, src, c.Ax.get(), op.inv_diag.get(), 1.0 / c.theta, dt, N, s);
      cur = B;
      prev = A;
    } else { // x_0 moved to xo, x_1 in dst
      vec::cheb_first_step(A, B, src, c.Ax.get(), op.inv_diag.get(), 1.0 / c.theta, dt, N, s);
      cur = A;
      prev = B;
    }
  }
  if (!more) return;
  double rhok = c.delta / c.theta;
  const double sigma = c.theta / c.delta;
  for (int k = 1; k < d; ++k) {
    const double rhokp = 1.0 / (2.0 * sigma - rhok);
    const double f1 = rhokp * rhok, f2 = 2.0 * rhokp / c.delta;
    rhok = rhokp;
    void *out = prev ? prev : (cur == A ? B : A);
    // DG operators on cell tiles apply the step inside their vmult kernel (A cur never stored)
    if (!operator_vmult_chebyshev(op, out, cur, prev, src, op.inv_diag.get(), f1, f2, s)) {
      operator_vmult(op, c.Ax.get(), cur, s);
      vec::cheb_update_into(out, cur, prev, src, c.Ax.get(), op.inv_diag.get(), f1, f2, dt, N, s);
    }
    prev = cur;
    cur = out;
  }
  PMG_REQUIRE(cur == A, "Chebyshev: the last iterate is not in dst");
}

void mg_setup(pmg_mg &mg, int n_levels, pmg_operator *const *levels, pmg_transfer *const *transfers,
              pmg_chebyshev *const *smoothers) {
  PMG_REQUIRE(n_levels >= 1, "need at least one level");
  mg.levels.assign(levels, levels + n_levels);
  mg.transfers.assign(transfers, transfers + n_levels);
  mg.smoothers.assign(smoothers, smoothers + n_levels);
  for (int l = 0; l < n_levels; ++l) {
    PMG_REQUIRE(mg.levels[l] && mg.smoothers[l], "null level operator or smoother");
    PMG_REQUIRE(mg.smoothers[l]->op == mg.levels[l], "smoother of level does not belong to its operator");
    if (l > 0) {
      PMG_REQUIRE(mg.transfers[l], "null transfer");
      PMG_REQUIRE(mg.transfers[l]->n_coarse == mg.levels[l - 1]->n_dofs &&
                      mg.transfers[l]->n_fine == mg.levels[l]->n_dofs,
                  "transfer does not connect consecutive levels");
    }
  }
  mg.device = mg.levels.back()->device;
  PMG_CUDA(cudaSetDevice(mg.device));
  mg.sol.resize(n_levels);
  mg.def.resize(n_levels);
  mg.t.resize(n_levels);
  for (int l = 0; l < n_levels; ++l) {
    const size_t bytes = dtype_size(mg.levels[l]->dtype) * mg.levels[l]->n_dofs;
    mg.sol[l].allocate(bytes);
    mg.def[l].allocate(bytes);
    mg.t[l].allocate(bytes);
  }
}

void mg_vcycle(pmg_mg &mg, int l, cudaStream_t s) {
  pmg_operator &op = *mg.levels[l];
  const int dt = op.dtype;
  const int64_t N = op.n_dofs;
  if (l == 0) { // coarse "solve" by the level-0 Chebyshev smoother
    chebyshev_apply(*mg.smoothers[0], mg.sol[0].get(), mg.def[0].get(), true, s);
    return;
  }
  pmg_operator &opc = *mg.levels[l - 1];
  chebyshev_apply(*mg.smoothers[l], mg.sol[l].get(), mg.def[l].get(), true, s);
  operator_vmult(op, mg.t[l].get(), mg.sol[l].get(), s);
  vec::residual(mg.t[l].get(), mg.def[l].get(), dt, N, s);
  PMG_CUDA(cudaMemsetAsync(mg.def[l - 1].get(), 0, dtype_size(opc.dtype) * opc.n_dofs, s));
  transfer_apply(*mg.transfers[l], 1, mg.def[l - 1].get(), mg.t[l].get(), s);
  mg_vcycle(mg, l - 1, s);
  transfer_apply(*mg.transfers[l], 0, mg.sol[l].get(), mg.sol[l - 1].get(), s);
  chebyshev_apply(*mg.smoothers[l], mg.sol[l].get(), mg.def[l].get(), false, s);
}

namespace {

// defect[level] = 0 below the top (portable_multigrid_solver.h:180-183), then the cycle
void mg_cycle_body(pmg_mg &mg, cudaStream_t s) {
  const int L = (int)mg.levels.size() - 1;
  for (int l = 0; l < L; ++l)
    PMG_CUDA(cudaMemsetAsync(mg.def[l].get(), 0, dtype_size(mg.levels[l]->dtype) * mg.levels[l]->n_dofs, s));
  mg_vcycle(mg, L, s);
}

bool graphs_allowed() {
  static const bool on = [] {
    const char *e = std::getenv("PMG_MG_GRAPH");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Capture the cycle into a graph on a private stream (the eigenvalue estimates, which
// synchronise and allocate, must have run before).  Any failure leaves graph == nullptr
// and the cycle runs as plain launches.
void mg_capture(pmg_mg &mg) {
  for (auto *sm : mg.smoothers)
    if (!sm->estimated) return;
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
    (void)cudaGetLastError();
    mg.graph_enabled = false;
    return;
  }
  cudaGraph_t g = nullptr;
  bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    try {
      mg_cycle_body(mg, cs);
    } catch (const Error &) {
      ok = false;
    }
    ok = (cudaStreamEndCapture(cs, &g) == cudaSuccess) && ok;
  }
  if (ok) ok = cudaGraphInstantiate(&mg.graph, g, 0) == cudaSuccess;
  mg.graph_generations.clear();
  for (auto *sm : mg.smoothers) mg.graph_generations.push_back(sm->generation);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  if (!ok) {
    (void)cudaGetLastError();
    mg.graph = nullptr;
    mg.graph_enabled = false;
  }
}

} // namespace

void mg_vmult(pmg_mg &mg, void *dst, const void *src, int vec_dtype, cudaStream_t s) {
  const int L = (int)mg.levels.size() - 1;
  const pmg_operator &top = *mg.levels[L];
  for (auto *sm : mg.smoothers)
    if (!sm->estimated) chebyshev_estimate(*sm, s);
  // a graph captured before a smoother was re-estimated holds the old Chebyshev coefficients
  if (mg.graph) {
    bool stale = mg.graph_generations.size() != mg.smoothers.size();
    for (size_t l = 0; !stale && l < mg.smoothers.size(); ++l)
      stale = mg.graph_generations[l] != mg.smoothers[l]->generation;
    if (stale) {
      PMG_CUDA(cudaStreamSynchronize(s));
      cudaGraphExecDestroy(mg.graph);
      mg.graph = nullptr;
    }
  }
  vec::convert(mg.def[L].get(), top.dtype, src, vec_dtype, top.n_dofs, s);
  if (mg.graph_enabled && graphs_allowed() && !prof::enabled() && !mg.graph) mg_capture(mg);
  if (mg.graph && !prof::enabled()) PMG_CUDA(cudaGraphLaunch(mg.graph, s));
  else mg_cycle_body(mg, s);
  vec::convert(dst, vec_dtype, mg.sol[L].get(), top.dtype, top.n_dofs, s);
}

// deal.II SolverCG with ReductionControl(max_it, abs_tol, reduce): stop at the first
// iterate with ||r|| <= max(abs_tol, reduce ||r_0||).
void cg_solve(pmg_operator &A, pmg_mg *mg, void *x, const void *b, double reduce, double abs_tol,
              int max_it, pmg_cg_info &info, cudaStream_t s) {
  PMG_REQUIRE(x && b, "null vector");
  PMG_REQUIRE(max_it >= 0, "max_iterations must be >= 0");
  if (mg) PMG_REQUIRE(mg->levels.back()->n_dofs == A.n_dofs, "preconditioner size mismatch");
  PMG_CUDA(cudaSetDevice(A.device));
  const int dt = A.dtype;
  const int64_t N = A.n_dofs;
  const size_t bytes = dtype_size(dt) * N;
  if (!mg && !A.has_diag) operator_compute_inverse_diagonal(A, s);
  // work vectors persist on the operator between solves (no allocation per solve)
  if (A.cg_work.size() != 4 || A.cg_work[0].bytes() != bytes) {
    A.cg_work.clear();
    for (int i = 0; i < 4; ++i) A.cg_work.emplace_back(bytes);
  }
  DeviceBuffer &r = A.cg_work[0], &z = A.cg_work[1], &p = A.cg_work[2], &v = A.cg_work[3];
  // r = b - A x and ||r|| in one pass
  operator_vmult(A, v.get(), x, s);
  double res = std::sqrt(vec::residual_dot(r.get(), b, v.get(), dt, N, s));
  check_finite(res, "CG residual");
  info = pmg_cg_info{};
  info.initial_residual = res;
  const double tol = std::max(abs_tol, reduce * res);
  int it = 0;
  double rho = 0, rho_old = 0;
  while (res > tol && it < max_it) {
    if (mg) {
      mg_vmult(*mg, z.get(), r.get(), dt, s);
      rho = vec::dot(r.get(), z.get(), dt, N, s);
    } else {
      rho = vec::jacobi_dot(z.get(), A.inv_diag.get(), r.get(), dt, N, s);
    }
    check_finite(rho, "CG preconditioned residual");
    if (it == 0) PMG_CUDA(cudaMemcpyAsync(p.get(), z.get(), bytes, cudaMemcpyDeviceToDevice, s));
    else vec::xpay(p.get(), z.get(), rho / rho_old, dt, N, s);
    rho_old = rho;
    ++it;
    operator_vmult(A, v.get(), p.get(), s);
    const double pv = vec::dot(p.get(), v.get(), dt, N, s);
    check_finite(pv, "CG curvature");
    if (pv <= 0) fail(PMG_ENOCONV, "CG breakdown: p.Ap <= 0");
    res = std::sqrt(vec::cg_update(x, r.get(), p.get(), v.get(), rho / pv, dt, N, s));
    check_finite(res, "CG residual");
  }
  info.iterations = it;
  info.final_residual = res;
  info.converged = res <= tol ? 1 : 0;
  info.reduction_per_step = it > 0 ? std::pow(res / info.initial_residual, 1.0 / it) : 1.0;
  PMG_CUDA(cudaStreamSynchronize(s));
}

// New coefficient values on a hierarchy: A (optional, the CG matrix) and the finest level get
// the values, every coarser level interpolates the level above it; then every level's
// inverse diagonal and smoother eigenvalue estimate are recomputed.
void mg_set_coefficient(pmg_mg &mg, pmg_operator *A, const double *values, bool on_device, cudaStream_t s) {
  for (auto *op : mg.levels)
    PMG_REQUIRE(op->coeff_kind == PMG_COEFF_VALUES, "every level needs PMG_COEFF_VALUES");
  pmg_operator *above = nullptr;
  if (A) {
    operator_set_coefficient(*A, values, on_device, s);
    above = A;
  }
  for (int l = (int)mg.levels.size() - 1; l >= 0; --l) {
    pmg_operator &op = *mg.levels[l];
    if (above) operator_interpolate_coefficient(op, *above, s);
    else operator_set_coefficient(op, values, on_device, s);
    above = &op;
  }
  if (A && A->has_diag) operator_compute_inverse_diagonal(*A, s);
  for (size_t l = 0; l < mg.levels.size(); ++l) {
    operator_compute_inverse_diagonal(*mg.levels[l], s);
    chebyshev_estimate(*mg.smoothers[l], s);
  }
}

// Gradient of J(m) = 1/2 (u - u_d)^T M (u - u_d) for A(m) u = b with A = sum_q exp(m_q) (...):
// lambda solves A lambda = M (u - u_d) (A is symmetric), and
// dJ/dm_q = -exp(m_q) grad lambda_q^T G_q grad u_q = the per-point form of (lambda, u) times -1.
void adjoint_gradient(pmg_operator &A, const pmg_operator &M, pmg_mg *mg, const void *u, const void *u_d,
                      void *lambda, double *g_qp, double &J, double reduce, double abs_tol, int max_it,
                      pmg_cg_info &info, cudaStream_t s) {
  PMG_REQUIRE(A.kind == PMG_OP_LAPLACE && M.kind == PMG_OP_MASS, "A must be a Laplace and M a mass operator");
  PMG_REQUIRE(A.dtype == PMG_F64 && M.dtype == PMG_F64, "the adjoint runs in FP64");
  PMG_REQUIRE(A.n_dofs == M.n_dofs && A.n_cells == M.n_cells && A.degree == M.degree,
              "A and M must share the mesh and the element");
  PMG_REQUIRE(u && u_d && lambda && g_qp, "null vector");
  PMG_CUDA(cudaSetDevice(A.device));
  const int64_t N = A.n_dofs;
  const size_t bytes = sizeof(double) * N;
  if (A.adj_work.size() != 2 || A.adj_work[0].bytes() != bytes) {
    A.adj_work.clear();
    for (int i = 0; i < 2; ++i) A.adj_work.emplace_back(bytes);
  }
  DeviceBuffer &e = A.adj_work[0], &r = A.adj_work[1];
  PMG_CUDA(cudaMemcpyAsync(e.get(), u_d, bytes, cudaMemcpyDeviceToDevice, s));
  vec::xpay(e.get(), u, -1.0, PMG_F64, N, s); // e = u - u_d
  operator_vmult(M, r.get(), e.get(), s);      // r = M e
  J = 0.5 * vec::dot(e.get(), r.get(), PMG_F64, N, s);
  check_finite(J, "the misfit");
  PMG_CUDA(cudaMemsetAsync(lambda, 0, bytes, s));
  cg_solve(A, mg, lambda, r.get(), reduce, abs_tol, max_it, info, s);
  operator_qp_form(A, lambda, u, -1.0, g_qp, s);
}

} // namespace pmg
