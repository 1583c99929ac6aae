// Vector kernels used by the smoother, the V-cycle and CG (vector_ops.cu).  Every function
// enqueues on `s`; the ones returning a double synchronise `s` to read the reduction.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pmg {
namespace vec {

void fill_mod11(void *x, int dtype, int64_t n, cudaStream_t s);
void convert(void *dst, int dt_dst, const void *src, int dt_src, int64_t n, cudaStream_t s);
// Chebyshev vector steps (x_{k+1} = x_k + f1 (x_k - x_{k-1}) + f2 D^{-1} (b - A x_k)):
// cheb_init: dst = scale D^{-1} src, xo = 0 unless xo is null; cheb_first_step: xo = dst,
// dst += scale D^{-1} (src - Ax); cheb_first_step_into: out = x0 + scale D^{-1} (src - Ax);
// cheb_update_into: out = the update from cur and prev (null: zero), out == prev allowed
void cheb_init(void *dst, void *xo, const void *src, const void *invd, double scale, int dtype,
               int64_t n, cudaStream_t s);
void cheb_first_step(void *dst, void *xo, const void *src, const void *Ax, const void *invd,
                     double scale, int dtype, int64_t n, cudaStream_t s);
void cheb_first_step_into(void *out, const void *x0, const void *src, const void *Ax, const void *invd,
                          double scale, int dtype, int64_t n, cudaStream_t s);
void cheb_update_into(void *out, const void *cur, const void *prev, const void *src, const void *Ax,
                      const void *invd, double f1, double f2, int dtype, int64_t n, cudaStream_t s);
void residual(void *t, const void *def, int dtype, int64_t n, cudaStream_t s);
void jacobi(void *z, const void *invd, const void *r, int dtype, int64_t n, cudaStream_t s);
void xpay(void *p, const void *z, double beta, int dtype, int64_t n, cudaStream_t s);
void axpy(void *y, const void *x, double alpha, int dtype, int64_t n, cudaStream_t s); // y += alpha x
double dot(const void *a, const void *b, int dtype, int64_t n, cudaStream_t s);
double cg_update(void *x, void *r, const void *p, const void *v, double alpha, int dtype, int64_t n,
                 cudaStream_t s);
double jacobi_dot(void *z, const void *invd, const void *r, int dtype, int64_t n, cudaStream_t s);
// r = b - Ax; returns r.r
double residual_dot(void *r, const void *b, const void *Ax, int dtype, int64_t n, cudaStream_t s);

} // namespace vec
} // namespace pmg
