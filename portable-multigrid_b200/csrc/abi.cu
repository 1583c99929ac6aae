// extern "C" entry points of libpmg_b200.so (declared in include/pmg/pmg.h): argument
// checks, exception-to-status translation, per-thread error messages.
#include <cstdio>
#include <exception>
#include <new>
#include <string>

#include "pmg_internal.hpp"
#include "solver.hpp"
#include "transfer.hpp"
#include "vector_ops.hpp"

namespace {

thread_local std::string g_last_error;

template <typename F> pmg_status guarded(const char *fn, F &&f) {
  try {
    f();
    return PMG_OK;
  } catch (const pmg::Error &e) {
    g_last_error = std::string(fn) + ": " + e.what();
    return e.status;
  } catch (const std::bad_alloc &) {
    g_last_error = std::string(fn) + ": host allocation failed";
    return PMG_ENOMEM;
  } catch (const std::exception &e) {
    g_last_error = std::string(fn) + ": " + e.what();
    return PMG_EINVAL;
  } catch (...) {
    g_last_error = std::string(fn) + ": unknown error";
    return PMG_EINVAL;
  }
}

#define NEED(ptr) PMG_REQUIRE((ptr) != nullptr, #ptr " is NULL")

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

} // namespace

namespace pmg {
void vector_dot_noalloc(const void *a, const void *b, int dtype, int64_t n, double *result,
                        cudaStream_t s);                                 // noalloc.cu
void measure_peaks(int device, int64_t copy_bytes, pmg_peaks *out); // peaks.cu
}

extern "C" {

size_t pmg_last_error(char *buf, size_t n) {
  if (buf && n > 0) {
    const size_t m = std::min(n - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), m);
    buf[m] = '\0';
  }
  return g_last_error.size();
}

const char *pmg_status_string(pmg_status s) {
  switch (s) {
  case PMG_OK: return "PMG_OK";
  case PMG_EINVAL: return "PMG_EINVAL";
  case PMG_ENOMEM: return "PMG_ENOMEM";
  case PMG_ECUDA: return "PMG_ECUDA";
  case PMG_ENONFINITE: return "PMG_ENONFINITE";
  case PMG_ENOCONV: return "PMG_ENOCONV";
  case PMG_EBOUNDS: return "PMG_EBOUNDS";
  case PMG_ESTATE: return "PMG_ESTATE";
  case PMG_ENODEV: return "PMG_ENODEV";
  default: return "PMG_UNKNOWN";
  }
}

pmg_status pmg_version(int32_t *major, int32_t *minor) {
  return guarded(__func__, [&] {
    NEED(major);
    NEED(minor);
    *major = 0;
    *minor = 1;
  });
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_mesh_create_box(const pmg_box *box, pmg_mesh **mesh) {
  return guarded(__func__, [&] {
    NEED(box);
    NEED(mesh);
    auto m = std::make_unique<pmg_mesh>();
    m->m = pmg::make_box(*box);
    *mesh = m.release();
  });
}

pmg_status pmg_mesh_destroy(pmg_mesh *mesh) {
  delete mesh;
  return PMG_OK;
}

pmg_status pmg_mesh_n_cells(const pmg_mesh *mesh, int64_t *n) {
  return guarded(__func__, [&] {
    NEED(mesh);
    NEED(n);
    *n = mesh->m.n_cells;
  });
}

pmg_status pmg_mesh_cell_coordinates(const pmg_mesh *mesh, int32_t *xyz) {
  return guarded(__func__, [&] {
    NEED(mesh);
    NEED(xyz);
    std::memcpy(xyz, mesh->m.cell_xyz.data(), mesh->m.cell_xyz.size() * sizeof(int32_t));
  });
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_operator_create(const pmg_mesh *mesh, const pmg_operator_params *params,
                               pmg_operator **op) {
  return guarded(__func__, [&] {
    NEED(mesh);
    NEED(params);
    NEED(op);
    auto o = std::make_unique<pmg_operator>();
    pmg::operator_setup(*o, *mesh, *params);
    *op = o.release();
  });
}

pmg_status pmg_operator_create_from_maps(const pmg_operator_maps *maps, const pmg_operator_params *params,
                                         pmg_operator **op) {
  return guarded(__func__, [&] {
    NEED(maps);
    NEED(params);
    NEED(op);
    auto o = std::make_unique<pmg_operator>();
    pmg::operator_setup_from_maps(*o, *maps, *params);
    *op = o.release();
  });
}

pmg_status pmg_operator_destroy(pmg_operator *op) {
  if (op) {
    cudaSetDevice(op->device);
    delete op;
  }
  return PMG_OK;
}

pmg_status pmg_operator_m(const pmg_operator *op, int64_t *m) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(m);
    *m = op->n_dofs;
  });
}

pmg_status pmg_operator_n(const pmg_operator *op, int64_t *n) { return pmg_operator_m(op, n); }

pmg_status pmg_operator_n_cells(const pmg_operator *op, int64_t *n) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(n);
    *n = op->n_cells;
  });
}

pmg_status pmg_operator_degree(const pmg_operator *op, int32_t *degree, int32_t *dtype) {
  return guarded(__func__, [&] {
    NEED(op);
    if (degree) *degree = op->degree;
    if (dtype) *dtype = op->dtype;
  });
}

pmg_status pmg_operator_vmult(const pmg_operator *op, void *dst, const void *src, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    PMG_CUDA(cudaSetDevice(op->device));
    pmg::operator_vmult(*op, dst, src, as_stream(stream));
  });
}

pmg_status pmg_operator_tvmult(const pmg_operator *op, void *dst, const void *src, void *stream) {
  return pmg_operator_vmult(op, dst, src, stream);
}

pmg_status pmg_operator_vmult_dummy(const pmg_operator *op, void *dst, const void *src,
                                    int32_t ghost_exchange_on, int32_t computation_on,
                                    void *stream) {
  (void)ghost_exchange_on; // a single device has no ghost DoFs
  return guarded(__func__, [&] {
    NEED(op);
    PMG_CUDA(cudaSetDevice(op->device));
    pmg::operator_vmult(*op, dst, src, as_stream(stream), computation_on != 0);
  });
}

pmg_status pmg_operator_vmult_cells(const pmg_operator *op, void *dst, const void *src, int64_t cell_begin,
                                    int64_t cell_end, int32_t init, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    PMG_CUDA(cudaSetDevice(op->device));
    pmg::operator_vmult_cells(*op, dst, src, cell_begin, cell_end, init != 0, as_stream(stream));
  });
}

pmg_status pmg_operator_cells_per_group(const pmg_operator *op, int32_t *cells) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(cells);
    *cells = op->cpw;
  });
}

pmg_status pmg_operator_compute_diagonal(pmg_operator *op, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    pmg::operator_compute_inverse_diagonal(*op, as_stream(stream));
  });
}

pmg_status pmg_operator_get_inverse_diagonal(const pmg_operator *op, const void **inv_diag) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(inv_diag);
    if (!op->has_diag) pmg::fail(PMG_ESTATE, "compute_diagonal has not been called");
    *inv_diag = op->inv_diag.get();
  });
}

pmg_status pmg_operator_copy_inverse_diagonal(const pmg_operator *op, void *dst, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(dst);
    if (!op->has_diag) pmg::fail(PMG_ESTATE, "compute_diagonal has not been called");
    PMG_CUDA(cudaSetDevice(op->device));
    PMG_CUDA(cudaMemcpyAsync(dst, op->inv_diag.get(), op->inv_diag.bytes(), cudaMemcpyDeviceToDevice,
                             as_stream(stream)));
  });
}

pmg_status pmg_operator_el(const pmg_operator *op, int64_t row, int64_t col, double *value) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(value);
    PMG_REQUIRE(row == col, "el() is only defined on the diagonal");
    if (row < 0 || row >= op->n_dofs) pmg::fail(PMG_EBOUNDS, "row out of range");
    if (!op->has_diag) pmg::fail(PMG_ESTATE, "compute_diagonal has not been called");
    PMG_CUDA(cudaSetDevice(op->device));
    PMG_CUDA(cudaDeviceSynchronize());
    double inv = 0;
    if (op->dtype == PMG_F64) {
      PMG_CUDA(cudaMemcpy(&inv, op->inv_diag.as<double>() + row, 8, cudaMemcpyDeviceToHost));
    } else {
      float f = 0;
      PMG_CUDA(cudaMemcpy(&f, op->inv_diag.as<float>() + row, 4, cudaMemcpyDeviceToHost));
      inv = f;
    }
    *value = 1.0 / inv;
  });
}

pmg_status pmg_operator_bytes_per_vmult(const pmg_operator *op, int64_t *bytes) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(bytes);
    *bytes = pmg::operator_bytes(*op);
  });
}

pmg_status pmg_operator_assemble_rhs(const pmg_operator *op, int32_t f_kind, int32_t nq, void *b,
                                     void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(b);
    pmg::operator_assemble_rhs(*op, f_kind, nq, b, as_stream(stream));
  });
}

pmg_status pmg_operator_copy_dof_indices(const pmg_operator *op, uint32_t *host) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(host);
    const pmg::Numbering &num = pmg::host_numbering(*op);
    for (size_t e = 0; e < num.plain.size(); ++e) {
      const uint32_t d = num.plain[e];
      host[e] = (d == pmg::kInvalid || num.constrained[d]) ? pmg::kInvalid : d;
    }
  });
}

pmg_status pmg_operator_copy_constrained(const pmg_operator *op, uint8_t *host) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(host);
    const pmg::Numbering &num = pmg::host_numbering(*op);
    std::memcpy(host, num.constrained.data(), num.constrained.size());
  });
}

pmg_status pmg_operator_copy_geometry(const pmg_operator *op, double *host) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(host);
    PMG_CUDA(cudaSetDevice(op->device));
    pmg::operator_copy_geometry(*op, host);
  });
}

pmg_status pmg_operator_set_tensor_cores(pmg_operator *op, int32_t mode) {
  return guarded(__func__, [&] {
    NEED(op);
    PMG_REQUIRE(mode == 0 || mode == 1 || mode == 3, "mode must be 0, 1 or 3");
    if (mode != 0) {
      PMG_REQUIRE(op->dtype == PMG_F32, "the tensor-core cell kernel is an FP32 (TF32) kernel");
      PMG_REQUIRE(op->kind == PMG_OP_LAPLACE && op->geometry == PMG_GEOMETRY_AFFINE && !op->dg,
                  "the tensor-core cell kernel needs the continuous Laplace operator with affine geometry");
    }
    op->tensor_cores = mode;
  });
}

pmg_status pmg_operator_dof_lattice(const pmg_operator *op, int32_t *ijk) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(ijk);
    if (op->from_maps || op->kind == PMG_OP_DG_SIPG || !op->dlattice.get())
      pmg::fail(PMG_ESTATE, "DoF lattice coordinates exist for continuous operators on box meshes only");
    const pmg::Numbering &num = pmg::host_numbering(*op);
    const int64_t L0 = num.L[0], L1 = num.L[1];
    const int64_t n_lat = (int64_t)num.lattice.size();
    for (int64_t t = 0; t < n_lat; ++t) {
      const uint32_t d = num.lattice[t];
      if (d == pmg::kInvalid) continue;
      ijk[3 * (int64_t)d + 0] = (int32_t)(t % L0);
      ijk[3 * (int64_t)d + 1] = (int32_t)((t / L0) % L1);
      ijk[3 * (int64_t)d + 2] = (int32_t)(t / (L0 * L1));
    }
  });
}

pmg_status pmg_operator_last_launch(const pmg_operator *op, int32_t kernel, int64_t *units,
                                   int64_t *parallel) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(units);
    NEED(parallel);
    PMG_REQUIRE(kernel >= PMG_KERNEL_VMULT_CELL && kernel <= PMG_KERNEL_QP_FORM, "bad kernel id");
    *units = op->launch_units[kernel];
    *parallel = op->launch_par[kernel];
  });
}

pmg_status pmg_operator_set_coefficient(pmg_operator *op, const double *coeff_qp, int32_t on_device,
                                        void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(coeff_qp);
    PMG_CUDA(cudaSetDevice(op->device));
    pmg::operator_set_coefficient(*op, coeff_qp, on_device != 0, as_stream(stream));
  });
}

pmg_status pmg_operator_interpolate_coefficient(pmg_operator *dst, pmg_operator *src, void *stream) {
  return guarded(__func__, [&] {
    NEED(dst);
    NEED(src);
    pmg::operator_interpolate_coefficient(*dst, *src, as_stream(stream));
  });
}

pmg_status pmg_operator_l2_error(const pmg_operator *op, const void *u, int32_t exact_kind, int32_t nq,
                                 double *error, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(u);
    NEED(error);
    *error = pmg::operator_l2_error(*op, u, exact_kind, nq, as_stream(stream));
  });
}

pmg_status pmg_operator_dof_coordinates(const pmg_operator *op, double *xyz, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(xyz);
    pmg::operator_dof_coordinates(*op, xyz, as_stream(stream));
  });
}

pmg_status pmg_operator_quadrature_points(const pmg_operator *op, double *xq, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(xq);
    pmg::operator_quadrature_points(*op, xq, as_stream(stream));
  });
}

pmg_status pmg_operator_qp_form(const pmg_operator *op, const void *u, const void *v, double alpha,
                                double *out, void *stream) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(u);
    NEED(v);
    NEED(out);
    pmg::operator_qp_form(*op, u, v, alpha, out, as_stream(stream));
  });
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_transfer_create(const pmg_operator *coarse, const pmg_operator *fine,
                               pmg_transfer **transfer) {
  return guarded(__func__, [&] {
    NEED(coarse);
    NEED(fine);
    NEED(transfer);
    auto t = std::make_unique<pmg_transfer>();
    pmg::transfer_setup(*t, *coarse, *fine);
    *transfer = t.release();
  });
}

pmg_status pmg_transfer_create_from_maps(const pmg_operator *coarse, const pmg_operator *fine,
                                         const pmg_transfer_maps *maps, pmg_transfer **transfer) {
  return guarded(__func__, [&] {
    NEED(coarse);
    NEED(fine);
    NEED(maps);
    NEED(transfer);
    auto t = std::make_unique<pmg_transfer>();
    pmg::transfer_setup_from_maps(*t, *coarse, *fine, *maps);
    *transfer = t.release();
  });
}

pmg_status pmg_transfer_destroy(pmg_transfer *t) {
  if (t) {
    cudaSetDevice(t->device);
    delete t;
  }
  return PMG_OK;
}

pmg_status pmg_transfer_prolongate_and_add(const pmg_transfer *t, void *dst_fine,
                                           const void *src_coarse, void *stream) {
  return guarded(__func__, [&] {
    NEED(t);
    PMG_CUDA(cudaSetDevice(t->device));
    pmg::transfer_apply(*t, 0, dst_fine, src_coarse, as_stream(stream));
  });
}

pmg_status pmg_transfer_restrict_and_add(const pmg_transfer *t, void *dst_coarse,
                                         const void *src_fine, void *stream) {
  return guarded(__func__, [&] {
    NEED(t);
    PMG_CUDA(cudaSetDevice(t->device));
    pmg::transfer_apply(*t, 1, dst_coarse, src_fine, as_stream(stream));
  });
}

pmg_status pmg_transfer_last_launch(const pmg_transfer *t, int64_t *units, int64_t *parallel) {
  return guarded(__func__, [&] {
    NEED(t);
    NEED(units);
    NEED(parallel);
    *units = t->launch_units;
    *parallel = t->launch_par;
  });
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_chebyshev_create(pmg_operator *op, const pmg_chebyshev_params *params,
                                pmg_chebyshev **smoother) {
  return guarded(__func__, [&] {
    NEED(op);
    NEED(params);
    NEED(smoother);
    auto c = std::make_unique<pmg_chebyshev>();
    pmg::chebyshev_setup(*c, *op, *params);
    *smoother = c.release();
  });
}

pmg_status pmg_chebyshev_destroy(pmg_chebyshev *c) {
  if (c) {
    // the operator is borrowed and may already be destroyed: use the recorded device
    cudaSetDevice(c->device);
    delete c;
  }
  return PMG_OK;
}

pmg_status pmg_chebyshev_estimate(pmg_chebyshev *c, void *stream) {
  return guarded(__func__, [&] {
    NEED(c);
    PMG_CUDA(cudaSetDevice(c->op->device));
    pmg::chebyshev_estimate(*c, as_stream(stream));
  });
}

pmg_status pmg_chebyshev_vmult(pmg_chebyshev *c, void *dst, const void *src, void *stream) {
  return guarded(__func__, [&] {
    NEED(c);
    NEED(dst);
    NEED(src);
    PMG_CUDA(cudaSetDevice(c->op->device));
    pmg::chebyshev_apply(*c, dst, src, true, as_stream(stream));
  });
}

pmg_status pmg_chebyshev_step(pmg_chebyshev *c, void *dst, const void *src, void *stream) {
  return guarded(__func__, [&] {
    NEED(c);
    NEED(dst);
    NEED(src);
    PMG_CUDA(cudaSetDevice(c->op->device));
    pmg::chebyshev_apply(*c, dst, src, false, as_stream(stream));
  });
}

pmg_status pmg_chebyshev_info(const pmg_chebyshev *c, double *min_ev, double *max_ev,
                              int32_t *degree, int32_t *cg_its) {
  return guarded(__func__, [&] {
    NEED(c);
    if (!c->estimated) pmg::fail(PMG_ESTATE, "eigenvalues not estimated yet");
    if (min_ev) *min_ev = c->min_ev;
    if (max_ev) *max_ev = c->max_ev;
    if (degree) *degree = c->degree;
    if (cg_its) *cg_its = c->cg_its;
  });
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_mg_create(int32_t n_levels, pmg_operator *const *levels,
                         pmg_transfer *const *transfers, pmg_chebyshev *const *smoothers,
                         pmg_mg **mg) {
  return guarded(__func__, [&] {
    NEED(levels);
    NEED(smoothers);
    NEED(mg);
    PMG_REQUIRE(n_levels == 1 || transfers, "transfers is NULL");
    auto m = std::make_unique<pmg_mg>();
    std::vector<pmg_transfer *> tr(n_levels, nullptr);
    for (int l = 1; l < n_levels; ++l) tr[l] = transfers[l];
    pmg::mg_setup(*m, n_levels, levels, tr.data(), smoothers);
    *mg = m.release();
  });
}

pmg_status pmg_mg_destroy(pmg_mg *mg) {
  if (mg) {
    cudaSetDevice(mg->device); // the levels are borrowed and may already be destroyed
    delete mg;
  }
  return PMG_OK;
}

pmg_status pmg_mg_vmult(pmg_mg *mg, void *dst, const void *src, int32_t vec_dtype, void *stream) {
  return guarded(__func__, [&] {
    NEED(mg);
    NEED(dst);
    NEED(src);
    PMG_REQUIRE(vec_dtype == PMG_F64 || vec_dtype == PMG_F32, "bad vec_dtype");
    PMG_CUDA(cudaSetDevice(mg->levels.back()->device));
    pmg::mg_vmult(*mg, dst, src, vec_dtype, as_stream(stream));
  });
}

pmg_status pmg_cg_solve(pmg_operator *A, pmg_mg *precond, void *x, const void *b, double reduce,
                        double abs_tol, int32_t max_iterations, pmg_cg_info *info, void *stream) {
  pmg_cg_info local{};
  pmg_status st = guarded(__func__, [&] {
    NEED(A);
    pmg::cg_solve(*A, precond, x, b, reduce, abs_tol, max_iterations, local, as_stream(stream));
  });
  if (info) *info = local;
  if (st == PMG_OK && !local.converged) {
    g_last_error = "pmg_cg_solve: iteration limit reached";
    return PMG_ENOCONV;
  }
  return st;
}

pmg_status pmg_mg_set_coefficient(pmg_mg *mg, pmg_operator *A, const double *coeff_qp, int32_t on_device,
                                  void *stream) {
  return guarded(__func__, [&] {
    NEED(mg);
    NEED(coeff_qp);
    PMG_CUDA(cudaSetDevice(mg->levels.back()->device));
    pmg::mg_set_coefficient(*mg, A, coeff_qp, on_device != 0, as_stream(stream));
    PMG_CUDA(cudaStreamSynchronize(as_stream(stream)));
  });
}

pmg_status pmg_adjoint_gradient(pmg_operator *A, const pmg_operator *M, pmg_mg *precond, const void *u,
                                const void *u_d, void *lambda, double *g_qp, double *J, double reduce,
                                double abs_tol, int32_t max_iterations, pmg_cg_info *info,
                                void *stream) {
  pmg_cg_info local{};
  double j = 0.0;
  pmg_status st = guarded(__func__, [&] {
    NEED(A);
    NEED(M);
    NEED(J);
    pmg::adjoint_gradient(*A, *M, precond, u, u_d, lambda, g_qp, j, reduce, abs_tol, max_iterations, local,
                          as_stream(stream));
    PMG_CUDA(cudaStreamSynchronize(as_stream(stream)));
  });
  if (info) *info = local;
  if (J) *J = j;
  if (st == PMG_OK && !local.converged) {
    g_last_error = "pmg_adjoint_gradient: iteration limit reached in the adjoint solve";
    return PMG_ENOCONV;
  }
  return st;
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_vector_dot(const void *a, const void *b, int32_t dtype, int64_t n, double *result,
                          void *stream) {
  return guarded(__func__, [&] {
    NEED(a);
    NEED(b);
    NEED(result);
    PMG_REQUIRE(dtype == PMG_F64 || dtype == PMG_F32, "bad dtype");
    PMG_REQUIRE(n >= 0, "n must be >= 0");
    *result = n == 0 ? 0.0 : pmg::vec::dot(a, b, dtype, n, as_stream(stream));
  });
}

pmg_status pmg_vector_dot_noalloc(const void *a, const void *b, int32_t dtype, int64_t n,
                                  double *result_dev, void *stream) {
  return guarded(__func__, [&] {
    pmg::vector_dot_noalloc(a, b, dtype, n, result_dev, as_stream(stream));
  });
}

pmg_status pmg_vector_axpy(void *y, const void *x, double alpha, int32_t dtype, int64_t n, void *stream) {
  return guarded(__func__, [&] {
    NEED(y);
    NEED(x);
    PMG_REQUIRE(dtype == PMG_F64 || dtype == PMG_F32, "bad dtype");
    PMG_REQUIRE(n >= 0, "n must be >= 0");
    if (n > 0) pmg::vec::axpy(y, x, alpha, dtype, n, as_stream(stream));
  });
}

pmg_status pmg_vector_xpay(void *y, const void *x, double alpha, int32_t dtype, int64_t n, void *stream) {
  return guarded(__func__, [&] {
    NEED(y);
    NEED(x);
    PMG_REQUIRE(dtype == PMG_F64 || dtype == PMG_F32, "bad dtype");
    PMG_REQUIRE(n >= 0, "n must be >= 0");
    if (n > 0) pmg::vec::xpay(y, x, alpha, dtype, n, as_stream(stream));
  });
}

pmg_status pmg_vector_pointwise_mult(void *z, const void *d, const void *r, int32_t dtype, int64_t n,
                                     void *stream) {
  return guarded(__func__, [&] {
    NEED(z);
    NEED(d);
    NEED(r);
    PMG_REQUIRE(dtype == PMG_F64 || dtype == PMG_F32, "bad dtype");
    PMG_REQUIRE(n >= 0, "n must be >= 0");
    if (n > 0) pmg::vec::jacobi(z, d, r, dtype, n, as_stream(stream));
  });
}

pmg_status pmg_vector_chebyshev_step(void *out, const void *cur, const void *prev, const void *src,
                                     const void *Ax, const void *inv_diag, double f1, double f2, int32_t dtype,
                                     int64_t n, void *stream) {
  return guarded(__func__, [&] {
    NEED(out);
    NEED(cur);
    NEED(src);
    NEED(Ax);
    NEED(inv_diag);
    PMG_REQUIRE(dtype == PMG_F64 || dtype == PMG_F32, "bad dtype");
    PMG_REQUIRE(n >= 0, "n must be >= 0");
    if (n > 0) pmg::vec::cheb_update_into(out, cur, prev, src, Ax, inv_diag, f1, f2, dtype, n, as_stream(stream));
  });
}

pmg_status pmg_vector_copy(void *dst, int32_t dt_dst, const void *src, int32_t dt_src, int64_t n,
                           void *stream) {
  return guarded(__func__, [&] {
    NEED(dst);
    NEED(src);
    PMG_REQUIRE((dt_dst == PMG_F64 || dt_dst == PMG_F32) && (dt_src == PMG_F64 || dt_src == PMG_F32),
                "bad dtype");
    PMG_REQUIRE(n >= 0, "n must be >= 0");
    if (n > 0) pmg::vec::convert(dst, dt_dst, src, dt_src, n, as_stream(stream));
  });
}

// ---------------------------------------------------------------------------------------
pmg_status pmg_profile_enable(int32_t on) {
  return guarded(__func__, [&] { pmg::prof::set_enabled(on != 0); });
}

pmg_status pmg_profile_reset(void) {
  return guarded(__func__, [&] { pmg::prof::reset(); });
}

pmg_status pmg_measure_peaks(int32_t device, int64_t copy_bytes, pmg_peaks *out) {
  return guarded(__func__, [&] {
    NEED(out);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) pmg::fail(PMG_ENODEV, "no CUDA device available");
    PMG_REQUIRE(device >= 0 && device < n, "device out of range");
    pmg::measure_peaks(device, copy_bytes, out);
  });
}

pmg_status pmg_profile_query(const char *kernel, double *total_ms, int64_t *launches) {
  return guarded(__func__, [&] {
    NEED(kernel);
    NEED(total_ms);
    NEED(launches);
    pmg::prof::query(kernel, total_ms, launches);
  });
}

} // extern "C"
