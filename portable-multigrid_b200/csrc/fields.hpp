// Adjoint-path kernels (fields.cu): FE mass matrix, per-point form, coefficient fields.
#pragma once

#include "pmg_internal.hpp"

namespace pmg {
const Tables1D &cached_tables(int degree); // make_tables(degree, degree + 1), built once
// dst += M src over the cells (dst zeroed and constrained rows set by the caller)
void mass_vmult_cells(const pmg_operator &op, const void *src, void *dst, cudaStream_t s);
// diag += diag(M) over the cells
void mass_diagonal_cells(const pmg_operator &op, void *diag, cudaStream_t s);
// out[c][q] = alpha * grad u^T G_q grad v (coefficient included), FP64
void qp_form_cells(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                   cudaStream_t s);
// dst_values[C_dst][nq_dst^3] = the source operator's coefficient field at dst's points
void coefficient_interpolate(const pmg_operator &src, const pmg_operator &dst, double *dst_values,
                             cudaStream_t s);
} // namespace pmg
