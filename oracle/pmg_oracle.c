/*
 * pmg_oracle.c -- CPU restatement of the portable-multigrid matrix-free hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links or calls this file;
 * only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline and reference arms)
 * load liboracle.so, and only as the checker / the timed CPU restatement.
 *
 * Parity status.  The reference's arithmetic lives in deal.II 9.8.0-pre (+ Kokkos, MPI,
 * p4est), none of which is vendored in the reference or installed here, so the reference
 * cannot be compiled or run.  The reference ships no golden vectors.  What pins this
 * restatement:
 *   - known-answer checks of the 1D tables (tests/test_oracle_tables.py);
 *   - two independent formulations of the cell operator (the BK3 collocation form of
 *     include/kernels/bk3_kokkos_kernel.h and the inverse-Jacobian form of
 *     include/kernels/portable_local_laplace_operator.h) agreeing to round-off;
 *   - the reference's own logged CG iteration counts and per-iteration reduction factors
 *     for the Q4 ph-multigrid solve on the "doubling" mesh
 *     (tests/poisson_cube_bk3_fp64/results/single-gpu-batched.out, the cg_its /
 *     cg_reduction table), reproduced by orc_solve_box() (tests/test_oracle_pin.py).
 * vmult values of the deformed-mesh, variable-coefficient and DG paths are not in any
 * reference log: for those the pin is the chain above plus mathematical checks.
 *
 * Conventions (all follow the reference):
 *   - cell-local DoF order is lexicographic, x fastest: l = (k*nm + j)*nm + i
 *     (include/kernels/bk3_kokkos_kernel.h:175);
 *   - dof index arrays are cell-contiguous [cell][nm^3] (Kokkos LayoutLeft (local,cell)),
 *     Dirichlet-constrained entries hold the sentinel 0xFFFFFFFF
 *     (include/operators/portable_laplace_operator_bk3.h:426-429);
 *   - geometry tensor G[cell][6][nq^3] in the order rr, rs, rt, ss, st, tt
 *     (include/operators/portable_laplace_operator_bk3.h:493-508);
 *   - 1D tables: shape_values[i*nq+q] (GLL Lagrange basis at Gauss points) and
 *     co_shape_gradients[n*nq+q] (derivative of the Gauss-point Lagrange basis n at
 *     Gauss point q), as consumed by bk3_kokkos_kernel.h:339-461.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INVALID 0xFFFFFFFFu

typedef long double ld;

/* ------------------------------------------------------------------------------------ */
/* 1. Quadrature and 1D tables                                                           */
/* ------------------------------------------------------------------------------------ */

static void legendre_eval(int n, ld x, ld *P, ld *dP)
{
  /* Bonnet recursion for P_n and its derivative; |x| < 1 for the derivative formula */
  ld p0 = 1.0L, p1 = x;
  if (n == 0) { *P = 1.0L; *dP = 0.0L; return; }
  for (int k = 2; k <= n; ++k) {
    ld p2 = ((2.0L * k - 1.0L) * x * p1 - (k - 1.0L) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  *P = p1;
  *dP = n * (x * p1 - p0) / (x * x - 1.0L);
}

static void gauss_ld(int n, ld *x, ld *w)
{
  /* Gauss-Legendre on [0,1], ascending: Newton on P_n from Chebyshev-like guesses */
  const ld pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < n; ++i) {
    ld t = cosl(pi * (i + 0.75L) / (n + 0.5L));
    for (int it = 0; it < 100; ++it) {
      ld P, dP;
      legendre_eval(n, t, &P, &dP);
      ld dt = P / dP;
      t -= dt;
      if (fabsl(dt) < 1e-19L) break;
    }
    ld P, dP;
    legendre_eval(n, t, &P, &dP);
    x[i] = (1.0L - t) * 0.5L;
    w[i] = 1.0L / ((1.0L - t * t) * dP * dP); /* 2/((1-t^2)P'^2) halved for [0,1] */
  }
}

static void gauss_lobatto_ld(int n, ld *x, ld *w)
{
  /* Gauss-Lobatto on [0,1], ascending: end points plus the roots of P'_{n-1} */
  const ld pi = 3.141592653589793238462643383279502884L;
  const int m = n - 1;
  x[0] = 0.0L;
  x[n - 1] = 1.0L;
  w[0] = w[n - 1] = 1.0L / (m * (m + 1.0L));
  for (int i = 1; i < n - 1; ++i) {
    ld t = cosl(pi * i / m);
    for (int it = 0; it < 100; ++it) {
      ld P, dP;
      legendre_eval(m, t, &P, &dP);
      /* P'' from the Legendre equation (1-t^2)P'' - 2tP' + m(m+1)P = 0 */
      ld d2P = (2.0L * t * dP - m * (m + 1.0L) * P) / (1.0L - t * t);
      ld dt = dP / d2P;
      t -= dt;
      if (fabsl(dt) < 1e-19L) break;
    }
    ld P, dP;
    legendre_eval(m, t, &P, &dP);
    x[i] = (1.0L - t) * 0.5L;
    w[i] = 1.0L / (m * (m + 1.0L) * P * P);
  }
}

static ld lagrange(int n, const ld *nodes, int i, ld x)
{
  ld v = 1.0L;
  for (int j = 0; j < n; ++j)
    if (j != i) v *= (x - nodes[j]) / (nodes[i] - nodes[j]);
  return v;
}

static ld lagrange_deriv(int n, const ld *nodes, int i, ld x)
{
  ld s = 0.0L;
  for (int m = 0; m < n; ++m) {
    if (m == i) continue;
    ld v = 1.0L / (nodes[i] - nodes[m]);
    for (int j = 0; j < n; ++j)
      if (j != i && j != m) v *= (x - nodes[j]) / (nodes[i] - nodes[j]);
    s += v;
  }
  return s;
}

void orc_gauss(int n, double *x, double *w)
{
  ld xl[32], wl[32];
  gauss_ld(n, xl, wl);
  for (int i = 0; i < n; ++i) { x[i] = (double)xl[i]; w[i] = (double)wl[i]; }
}

void orc_gauss_lobatto(int n, double *x, double *w)
{
  ld xl[32], wl[32];
  gauss_lobatto_ld(n, xl, wl);
  for (int i = 0; i < n; ++i) { x[i] = (double)xl[i]; w[i] = (double)wl[i]; }
}

/* Shape tables of FE_Q(p) (Lagrange on p+1 Gauss-Lobatto nodes) at nq Gauss points.
 * S[i*nq+q]  = phi_i(g_q)                 (shape_values,       bk3_kokkos_kernel.h:69)
 * SD[i*nq+q] = phi_i'(g_q)                (used by the inverse-Jacobian formulation)
 * D[n*nq+q]  = l_n'(g_q), l_n = Lagrange basis on the Gauss points (co_shape_gradients)
 * W[q]       = Gauss weight on [0,1].                                                   */
void orc_shape_tables(int p, int nq, double *S, double *SD, double *D, double *W)
{
  const int nm = p + 1;
  ld xg[32], wg[32], xl[32], wl[32];
  gauss_ld(nq, xg, wg);
  gauss_lobatto_ld(nm, xl, wl);
  for (int i = 0; i < nm; ++i)
    for (int q = 0; q < nq; ++q) {
      if (S) S[i * nq + q] = (double)lagrange(nm, xl, i, xg[q]);
      if (SD) SD[i * nq + q] = (double)lagrange_deriv(nm, xl, i, xg[q]);
    }
  for (int n = 0; n < nq; ++n)
    for (int q = 0; q < nq; ++q)
      if (D) D[n * nq + q] = (double)lagrange_deriv(nq, xg, n, xg[q]);
  for (int q = 0; q < nq; ++q)
    if (W) W[q] = (double)wg[q];
}

/* 1D p-transfer matrix FE_Q(pc) -> FE_Q(pf): the projection between nested Lagrange spaces
 * equals interpolation at the fine nodes.  Stored [i_c*nm_f + j_f] as the reference does
 * (include/multigrid/portable_polynomial_transfer.h:1093-1108).                         */
void orc_projection_matrix(int pc, int pf, double *P)
{
  const int nc = pc + 1, nf = pf + 1;
  ld xc[32], wc[32], xf[32], wf[32];
  gauss_lobatto_ld(nc, xc, wc);
  gauss_lobatto_ld(nf, xf, wf);
  for (int i = 0; i < nc; ++i)
    for (int j = 0; j < nf; ++j) P[i * nf + j] = (double)lagrange(nc, xc, i, xf[j]);
}

/* 1D h-transfer matrix for FE_Q(p) and isotropic refinement: coarse basis evaluated at the
 * fine nodes of both children, fine nodes numbered 0..2p over the coarse cell
 * (include/multigrid/portable_geometric_transfer.h:1285-1337).  Stored [i_c*(2p+1)+j_f]. */
void orc_h_prolongation_matrix(int p, double *P)
{
  const int n = p + 1, nf = 2 * p + 1;
  ld x[32], w[32];
  gauss_lobatto_ld(n, x, w);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < nf; ++j) {
      ld y = (j <= p) ? 0.5L * x[j] : 0.5L + 0.5L * x[j - p];
      P[i * nf + j] = (double)lagrange(n, x, i, y);
    }
}

/* ------------------------------------------------------------------------------------ */
/* 2. Structured box meshes                                                              */
/* ------------------------------------------------------------------------------------ */

/* A box [lo,hi] made of coarse[0] x coarse[1] x coarse[2] coarse cells, each refined
 * globally `refine` times (GridGenerator::subdivided_hyper_rectangle + refine_global, as in
 * tests/poisson_cube_bk3/program.cc:937-957).  deform = 1 moves every mapping node by
 * x' = x + amp*sin(pi x)sin(pi y)sin(pi z) in each component.                            */
typedef struct {
  int32_t coarse[3];
  int32_t refine;
  double lo[3];
  double hi[3];
  int32_t deform;
  double amp;
  int32_t dirichlet_mask; /* bit f set: face f (x-,x+,y-,y+,z-,z+) is Dirichlet */
} orc_box;

static void box_ncells(const orc_box *b, int64_t n[3])
{
  for (int d = 0; d < 3; ++d) n[d] = (int64_t)b->coarse[d] << b->refine;
}

int64_t orc_box_ncells(const orc_box *b)
{
  int64_t n[3];
  box_ncells(b, n);
  return n[0] * n[1] * n[2];
}

/* Cell order: coarse cells lexicographically (x fastest), inside each coarse cell the
 * Morton (z-order) curve with x in the lowest bit -- the order p4est gives the active
 * cells of a globally refined parallel::distributed::Triangulation.                      */
void orc_box_cell_coords(const orc_box *b, int32_t *cx, int32_t *cy, int32_t *cz)
{
  const int L = b->refine;
  const int64_t per_tree = (int64_t)1 << (3 * L);
  int64_t c = 0;
  for (int tz = 0; tz < b->coarse[2]; ++tz)
    for (int ty = 0; ty < b->coarse[1]; ++ty)
      for (int tx = 0; tx < b->coarse[0]; ++tx)
        for (int64_t m = 0; m < per_tree; ++m, ++c) {
          int32_t x = 0, y = 0, z = 0;
          for (int bit = 0; bit < L; ++bit) {
            x |= (int32_t)((m >> (3 * bit)) & 1) << bit;
            y |= (int32_t)((m >> (3 * bit + 1)) & 1) << bit;
            z |= (int32_t)((m >> (3 * bit + 2)) & 1) << bit;
          }
          cx[c] = (tx << L) + x;
          cy[c] = (ty << L) + y;
          cz[c] = (tz << L) + z;
        }
}

/* DoF numbering of FE_Q(p) on the box: global DoFs are numbered in order of first visit,
 * walking the cells in cell order and each cell's nodes in lexicographic order.
 * plain[c*nm^3 + l] receives the global DoF of local node l of cell c; constrained[dof] = 1
 * for DoFs on a Dirichlet face; lattice (optional) maps the global node lattice
 * (x fastest, extents p*n_d+1) to DoF numbers.  Returns the number of DoFs.            */
int64_t orc_box_dofs(const orc_box *b, int p, uint32_t *plain, uint8_t *constrained,
                     uint32_t *lattice_out)
{
  int64_t n[3];
  box_ncells(b, n);
  const int nm = p + 1;
  const int64_t L0 = p * n[0] + 1, L1 = p * n[1] + 1, L2 = p * n[2] + 1;
  const int64_t n_lattice = L0 * L1 * L2;
  const int64_t C = n[0] * n[1] * n[2];
  uint32_t *lat = lattice_out ? lattice_out : (uint32_t *)malloc(sizeof(uint32_t) * n_lattice);
  for (int64_t i = 0; i < n_lattice; ++i) lat[i] = ORC_INVALID;
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * C * 3);
  int32_t *cy = cx + C, *cz = cy + C;
  orc_box_cell_coords(b, cx, cy, cz);
  uint32_t next = 0;
  for (int64_t c = 0; c < C; ++c)
    for (int k = 0; k < nm; ++k)
      for (int j = 0; j < nm; ++j)
        for (int i = 0; i < nm; ++i) {
          const int64_t gx = (int64_t)p * cx[c] + i, gy = (int64_t)p * cy[c] + j,
                        gz = (int64_t)p * cz[c] + k;
          const int64_t id = (gz * L1 + gy) * L0 + gx;
          if (lat[id] == ORC_INVALID) {
            lat[id] = next;
            if (constrained) {
              int on = 0;
              const int m = b->dirichlet_mask;
              if ((m & 1) && gx == 0) on = 1;
              if ((m & 2) && gx == L0 - 1) on = 1;
              if ((m & 4) && gy == 0) on = 1;
              if ((m & 8) && gy == L1 - 1) on = 1;
              if ((m & 16) && gz == 0) on = 1;
              if ((m & 32) && gz == L2 - 1) on = 1;
              constrained[next] = (uint8_t)on;
            }
            ++next;
          }
          if (plain) plain[c * nm * nm * nm + (k * nm + j) * nm + i] = lat[id];
        }
  free(cx);
  if (!lattice_out) free(lat);
  return (int64_t)next;
}

/* dof_indices with the sentinel for constrained DoFs
 * (include/operators/portable_laplace_operator_bk3.h:421-430). */
void orc_apply_sentinel(int64_t n_entries, const uint32_t *plain, const uint8_t *constrained,
                        uint32_t *idx)
{
  for (int64_t e = 0; e < n_entries; ++e)
    idx[e] = constrained[plain[e]] ? ORC_INVALID : plain[e];
}

/* ------------------------------------------------------------------------------------ */
/* 3. Geometry                                                                           */
/* ------------------------------------------------------------------------------------ */

static const double ORC_PI = 3.14159265358979323846;

static void map_point(const orc_box *b, const double xr[3], double xp[3])
{
  for (int d = 0; d < 3; ++d) xp[d] = xr[d];
  if (b->deform == 1) {
    const double s = b->amp * sin(ORC_PI * xr[0]) * sin(ORC_PI * xr[1]) * sin(ORC_PI * xr[2]);
    for (int d = 0; d < 3; ++d) xp[d] = xr[d] + s;
  }
}

/* physical positions of the Q_p mapping nodes (Gauss-Lobatto) of cell (cx,cy,cz):
 * X[d*nm^3 + l] */
static void cell_nodes(const orc_box *b, int p, int32_t cx, int32_t cy, int32_t cz,
                       const double *xgll, double *X)
{
  int64_t n[3];
  box_ncells(b, n);
  const int nm = p + 1;
  double h[3];
  for (int d = 0; d < 3; ++d) h[d] = (b->hi[d] - b->lo[d]) / (double)n[d];
  const int32_t cc[3] = {cx, cy, cz};
  for (int k = 0; k < nm; ++k)
    for (int j = 0; j < nm; ++j)
      for (int i = 0; i < nm; ++i) {
        const int l = (k * nm + j) * nm + i;
        const double xi[3] = {xgll[i], xgll[j], xgll[k]};
        double xr[3], xp[3];
        for (int d = 0; d < 3; ++d) xr[d] = b->lo[d] + (cc[d] + xi[d]) * h[d];
        map_point(b, xr, xp);
        for (int d = 0; d < 3; ++d) X[d * nm * nm * nm + l] = xp[d];
      }
}

static double coefficient(int kind, const double x[3])
{
  if (kind == 1)
    return 1.0 + 0.9 * sin(2 * ORC_PI * x[0]) * sin(2 * ORC_PI * x[1]) * sin(2 * ORC_PI * x[2]);
  return 1.0;
}

/* Per quadrature point: J (d,e) = dx_d/dxi_e, the mapped point and the tensor weight. */
static void cell_jacobians(int p, int nq, const double *X, const double *S, const double *SD,
                           const double *W, double *J /*[q][9]*/, double *xq /*[q][3]*/,
                           double *wq /*[q]*/)
{
  const int nm = p + 1, nm3 = nm * nm * nm;
  for (int q2 = 0; q2 < nq; ++q2)
    for (int q1 = 0; q1 < nq; ++q1)
      for (int q0 = 0; q0 < nq; ++q0) {
        const int q = (q2 * nq + q1) * nq + q0;
        double jac[9] = {0}, pos[3] = {0};
        for (int k = 0; k < nm; ++k)
          for (int j = 0; j < nm; ++j)
            for (int i = 0; i < nm; ++i) {
              const int l = (k * nm + j) * nm + i;
              const double v = S[i * nq + q0] * S[j * nq + q1] * S[k * nq + q2];
              const double g0 = SD[i * nq + q0] * S[j * nq + q1] * S[k * nq + q2];
              const double g1 = S[i * nq + q0] * SD[j * nq + q1] * S[k * nq + q2];
              const double g2 = S[i * nq + q0] * S[j * nq + q1] * SD[k * nq + q2];
              for (int d = 0; d < 3; ++d) {
                const double xv = X[d * nm3 + l];
                pos[d] += xv * v;
                jac[d * 3 + 0] += xv * g0;
                jac[d * 3 + 1] += xv * g1;
                jac[d * 3 + 2] += xv * g2;
              }
            }
        memcpy(J + 9 * q, jac, sizeof(jac));
        memcpy(xq + 3 * q, pos, sizeof(pos));
        wq[q] = W[q0] * W[q1] * W[q2];
      }
}

static double invert3(const double *J, double *inv)
{
  const double a = J[0], b = J[1], c = J[2], d = J[3], e = J[4], f = J[5], g = J[6],
               h = J[7], i = J[8];
  const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  const double det = a * A + b * B + c * C;
  const double r = 1.0 / det;
  inv[0] = A * r;
  inv[1] = -(b * i - c * h) * r;
  inv[2] = (b * f - c * e) * r;
  inv[3] = B * r;
  inv[4] = (a * i - c * g) * r;
  inv[5] = -(a * f - c * d) * r;
  inv[6] = C * r;
  inv[7] = -(a * h - b * g) * r;
  inv[8] = (a * e - b * d) * r;
  return det;
}

/* G_c(q) = kappa(x_q) * JxW(q) * J^{-1} J^{-T} with (J^{-1})_{ek} = dxi_e/dx_k, stored
 * G[cell][6][nq^3] in the order rr, rs, rt, ss, st, tt
 * (include/operators/portable_laplace_operator_bk3.h:484-511). kappa_qp (optional,
 * [C][nq^3]) multiplies on top of coeff_kind. */
void orc_box_G(const orc_box *b, int p, int coeff_kind, const double *kappa_qp, double *G)
{
  const int nm = p + 1, nq = p + 1, nq3 = nq * nq * nq;
  const int64_t C = orc_box_ncells(b);
  double S[64], SD[64], D[64], W[8], xgll[8], wgll[8];
  orc_shape_tables(p, nq, S, SD, D, W);
  orc_gauss_lobatto(nm, xgll, wgll);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  int32_t *cy = cx + C, *cz = cy + C;
  orc_box_cell_coords(b, cx, cy, cz);
#pragma omp parallel
  {
    double *X = (double *)malloc(sizeof(double) * 3 * nm * nm * nm);
    double *J = (double *)malloc(sizeof(double) * 9 * nq3);
    double *xq = (double *)malloc(sizeof(double) * 3 * nq3);
    double *wq = (double *)malloc(sizeof(double) * nq3);
#pragma omp for schedule(static)
    for (int64_t c = 0; c < C; ++c) {
      cell_nodes(b, p, cx[c], cy[c], cz[c], xgll, X);
      cell_jacobians(p, nq, X, S, SD, W, J, xq, wq);
      for (int q = 0; q < nq3; ++q) {
        double inv[9];
        const double det = invert3(J + 9 * q, inv);
        double f = fabs(det) * wq[q] * coefficient(coeff_kind, xq + 3 * q);
        if (kappa_qp) f *= kappa_qp[c * nq3 + q];
        int comp = 0;
        for (int d1 = 0; d1 < 3; ++d1)
          for (int d2 = d1; d2 < 3; ++d2) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += inv[d1 * 3 + k] * inv[d2 * 3 + k];
            G[(c * 6 + comp) * nq3 + q] = f * s;
            ++comp;
          }
      }
    }
    free(X); free(J); free(xq); free(wq);
  }
  free(cx);
}

/* Inverse Jacobians and JxW per quadrature point (the data layout of the deal.II-style
 * operator, include/kernels/portable_local_laplace_operator.h:329-347):
 * invJ[cell][q][9] (row e = reference direction, column k = physical direction),
 * JxW[cell][q] including the coefficient. */
void orc_box_invjac(const orc_box *b, int p, int coeff_kind, double *invJ, double *JxW)
{
  const int nm = p + 1, nq = p + 1, nq3 = nq * nq * nq;
  const int64_t C = orc_box_ncells(b);
  double S[64], SD[64], D[64], W[8], xgll[8], wgll[8];
  orc_shape_tables(p, nq, S, SD, D, W);
  orc_gauss_lobatto(nm, xgll, wgll);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  int32_t *cy = cx + C, *cz = cy + C;
  orc_box_cell_coords(b, cx, cy, cz);
  double *X = (double *)malloc(sizeof(double) * 3 * nm * nm * nm);
  double *J = (double *)malloc(sizeof(double) * 9 * nq3);
  double *xq = (double *)malloc(sizeof(double) * 3 * nq3);
  double *wq = (double *)malloc(sizeof(double) * nq3);
  for (int64_t c = 0; c < C; ++c) {
    cell_nodes(b, p, cx[c], cy[c], cz[c], xgll, X);
    cell_jacobians(p, nq, X, S, SD, W, J, xq, wq);
    for (int q = 0; q < nq3; ++q) {
      const double det = invert3(J + 9 * q, invJ + (c * nq3 + q) * 9);
      JxW[c * nq3 + q] = fabs(det) * wq[q] * coefficient(coeff_kind, xq + 3 * q);
    }
  }
  free(X); free(J); free(xq); free(wq); free(cx);
}

/* Quadrature point positions and JxW for an nq-point Gauss rule on every cell
 * (xq[cell][q][3], jxw[cell][q]); used for right-hand sides and error norms. */
void orc_box_quadrature(const orc_box *b, int p, int nq, double *xq_out, double *jxw_out)
{
  const int nm = p + 1, nq3 = nq * nq * nq;
  const int64_t C = orc_box_ncells(b);
  double *S = (double *)malloc(sizeof(double) * nm * nq);
  double *SD = (double *)malloc(sizeof(double) * nm * nq);
  double *W = (double *)malloc(sizeof(double) * nq);
  double xgll[16], wgll[16];
  orc_shape_tables(p, nq, S, SD, NULL, W);
  orc_gauss_lobatto(nm, xgll, wgll);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  int32_t *cy = cx + C, *cz = cy + C;
  orc_box_cell_coords(b, cx, cy, cz);
  double *X = (double *)malloc(sizeof(double) * 3 * nm * nm * nm);
  double *J = (double *)malloc(sizeof(double) * 9 * nq3);
  double *wq = (double *)malloc(sizeof(double) * nq3);
  for (int64_t c = 0; c < C; ++c) {
    cell_nodes(b, p, cx[c], cy[c], cz[c], xgll, X);
    cell_jacobians(p, nq, X, S, SD, W, J, xq_out + c * nq3 * 3, wq);
    for (int q = 0; q < nq3; ++q) {
      double inv[9];
      jxw_out[c * nq3 + q] = fabs(invert3(J + 9 * q, inv)) * wq[q];
    }
  }
  free(X); free(J); free(wq); free(cx); free(S); free(SD); free(W);
}

/* ------------------------------------------------------------------------------------ */
/* 4. Cell operator                                                                      */
/* ------------------------------------------------------------------------------------ */

/* One cell of the BK3 operator, following the twelve steps of
 * include/kernels/bk3_kokkos_kernel.h:113-738: interpolate nodes -> Gauss points along
 * x, y, z (steps 2-4), collocation gradients times G (step 5), transposed gradients
 * (step 6), back-interpolation along z, y, x (steps 7-9). u and out are [n^3]. */
static void bk3_cell(int n, const double *S, const double *D, const double *Gc,
                     const double *u, double *out, double *w0, double *w1, double *rr,
                     double *rs, double *rt)
{
  const int n3 = n * n * n;
  /* step 2: direction 0 */
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int p = 0; p < n; ++p) {
        double t = 0;
        for (int i = 0; i < n; ++i) t += S[i * n + p] * u[(k * n + j) * n + i];
        w1[(k * n + j) * n + p] = t;
      }
  /* step 3: direction 1 */
  for (int k = 0; k < n; ++k)
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p) {
        double t = 0;
        for (int j = 0; j < n; ++j) t += S[j * n + q] * w1[(k * n + j) * n + p];
        w0[(k * n + q) * n + p] = t;
      }
  /* step 4: direction 2 */
  for (int r = 0; r < n; ++r)
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p) {
        double t = 0;
        for (int k = 0; k < n; ++k) t += S[k * n + r] * w0[(k * n + q) * n + p];
        w1[(r * n + q) * n + p] = t;
      }
  /* step 5: collocation gradients and the geometric factors */
  for (int r = 0; r < n; ++r)
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p) {
        const int qq = (r * n + q) * n + p;
        double gr = 0, gs = 0, gt = 0;
        for (int m = 0; m < n; ++m) {
          gr += D[m * n + p] * w1[(r * n + q) * n + m];
          gs += D[m * n + q] * w1[(r * n + m) * n + p];
          gt += D[m * n + r] * w1[(m * n + q) * n + p];
        }
        const double Grr = Gc[0 * n3 + qq], Grs = Gc[1 * n3 + qq], Grt = Gc[2 * n3 + qq],
                     Gss = Gc[3 * n3 + qq], Gst = Gc[4 * n3 + qq], Gtt = Gc[5 * n3 + qq];
        rr[qq] = Grr * gr + Grs * gs + Grt * gt;
        rs[qq] = Grs * gr + Gss * gs + Gst * gt;
        rt[qq] = Grt * gr + Gst * gs + Gtt * gt;
      }
  /* step 6: integrate with the transposed gradients */
  for (int r = 0; r < n; ++r)
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p) {
        double t = 0;
        for (int m = 0; m < n; ++m) {
          t += D[p * n + m] * rr[(r * n + q) * n + m];
          t += D[q * n + m] * rs[(r * n + m) * n + p];
          t += D[r * n + m] * rt[(m * n + q) * n + p];
        }
        w1[(r * n + q) * n + p] = t;
      }
  /* step 7: direction 2 back to nodes */
  for (int k = 0; k < n; ++k)
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < n; ++p) {
        double t = 0;
        for (int r = 0; r < n; ++r) t += S[k * n + r] * w1[(r * n + q) * n + p];
        w0[(k * n + q) * n + p] = t;
      }
  /* step 8: direction 1 */
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int p = 0; p < n; ++p) {
        double t = 0;
        for (int q = 0; q < n; ++q) t += S[j * n + q] * w0[(k * n + q) * n + p];
        w1[(k * n + j) * n + p] = t;
      }
  /* step 9: direction 0 */
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double t = 0;
        for (int p = 0; p < n; ++p) t += S[i * n + p] * w1[(k * n + j) * n + p];
        out[(k * n + j) * n + i] = t;
      }
}

typedef struct {
  int p;
  int64_t C, N;
  const uint32_t *idx;        /* [C][nm^3], sentinel for constrained */
  const double *G;            /* [C][6][nq^3] */
  const uint8_t *constrained; /* [N] */
  const uint8_t *color;       /* [C] in 0..7 or NULL (serial) */
} orc_op;

static void orc_op_vmult_impl(const orc_op *op, const double *src, double *dst)
{
  const int n = op->p + 1, n3 = n * n * n;
  double S[64], D[64];
  orc_shape_tables(op->p, n, S, NULL, D, NULL);
  for (int64_t i = 0; i < op->N; ++i) dst[i] = 0.0; /* dst = 0 (bk3.h:134) */
  const int n_colors = op->color ? 8 : 1;
  for (int col = 0; col < n_colors; ++col) {
#pragma omp parallel if (op->color != NULL)
    {
      double *buf = (double *)malloc(sizeof(double) * 7 * n3);
      double *u = buf, *out = buf + n3, *w0 = buf + 2 * n3, *w1 = buf + 3 * n3,
             *rr = buf + 4 * n3, *rs = buf + 5 * n3, *rt = buf + 6 * n3;
#pragma omp for schedule(static)
      for (int64_t c = 0; c < op->C; ++c) {
        if (op->color && op->color[c] != col) continue;
        const uint32_t *ci = op->idx + c * n3;
        for (int l = 0; l < n3; ++l) u[l] = (ci[l] == ORC_INVALID) ? 0.0 : src[ci[l]];
        bk3_cell(n, S, D, op->G + c * 6 * n3, u, out, w0, w1, rr, rs, rt);
        for (int l = 0; l < n3; ++l)
          if (ci[l] != ORC_INVALID) dst[ci[l]] += out[l];
      }
      free(buf);
    }
  }
  /* copy_constrained_values (portable_laplace_operator_bk3.h:230): identity rows */
  for (int64_t i = 0; i < op->N; ++i)
    if (op->constrained[i]) dst[i] = src[i];
}

void orc_vmult(int p, int64_t C, int64_t N, const uint32_t *idx, const double *G,
               const uint8_t *constrained, const uint8_t *color, const double *src,
               double *dst)
{
  orc_op op = {p, C, N, idx, G, constrained, color};
  orc_op_vmult_impl(&op, src, dst);
}

/* The same operator in the formulation of include/kernels/portable_local_laplace_operator.h
 * (deal.II Portable FEEvaluation): reference gradients straight from the nodal values with
 * the derivative table SD, physical gradient = J^{-T} grad_ref, times JxW, and back with
 * J^{-1}.  Independent of the collocation tables, so agreement with orc_vmult checks both.*/
void orc_vmult_invjac(int p, int64_t C, int64_t N, const uint32_t *idx, const double *invJ,
                      const double *JxW, const uint8_t *constrained, const double *src,
                      double *dst)
{
  const int n = p + 1, n3 = n * n * n;
  double S[64], SD[64];
  orc_shape_tables(p, n, S, SD, NULL, NULL);
  double *u = (double *)malloc(sizeof(double) * n3 * 5);
  double *out = u + n3, *fx = out + n3, *fy = fx + n3, *fz = fy + n3;
  for (int64_t i = 0; i < N; ++i) dst[i] = 0.0;
  for (int64_t c = 0; c < C; ++c) {
    const uint32_t *ci = idx + c * n3;
    for (int l = 0; l < n3; ++l) u[l] = (ci[l] == ORC_INVALID) ? 0.0 : src[ci[l]];
    for (int q2 = 0; q2 < n; ++q2)
      for (int q1 = 0; q1 < n; ++q1)
        for (int q0 = 0; q0 < n; ++q0) {
          const int q = (q2 * n + q1) * n + q0;
          double g[3] = {0, 0, 0};
          for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
              for (int i = 0; i < n; ++i) {
                const double v = u[(k * n + j) * n + i];
                g[0] += v * SD[i * n + q0] * S[j * n + q1] * S[k * n + q2];
                g[1] += v * S[i * n + q0] * SD[j * n + q1] * S[k * n + q2];
                g[2] += v * S[i * n + q0] * S[j * n + q1] * SD[k * n + q2];
              }
          const double *iJ = invJ + (c * n3 + q) * 9;
          double gx[3];
          for (int kk = 0; kk < 3; ++kk)
            gx[kk] = iJ[0 * 3 + kk] * g[0] + iJ[1 * 3 + kk] * g[1] + iJ[2 * 3 + kk] * g[2];
          const double jw = JxW[c * n3 + q];
          double f[3];
          for (int e = 0; e < 3; ++e)
            f[e] = jw * (iJ[e * 3 + 0] * gx[0] + iJ[e * 3 + 1] * gx[1] + iJ[e * 3 + 2] * gx[2]);
          fx[q] = f[0];
          fy[q] = f[1];
          fz[q] = f[2];
        }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double s = 0;
          for (int q2 = 0; q2 < n; ++q2)
            for (int q1 = 0; q1 < n; ++q1)
              for (int q0 = 0; q0 < n; ++q0) {
                const int q = (q2 * n + q1) * n + q0;
                s += fx[q] * SD[i * n + q0] * S[j * n + q1] * S[k * n + q2];
                s += fy[q] * S[i * n + q0] * SD[j * n + q1] * S[k * n + q2];
                s += fz[q] * S[i * n + q0] * S[j * n + q1] * SD[k * n + q2];
              }
          out[(k * n + j) * n + i] = s;
        }
    for (int l = 0; l < n3; ++l)
      if (ci[l] != ORC_INVALID) dst[ci[l]] += out[l];
  }
  for (int64_t i = 0; i < N; ++i)
    if (constrained[i]) dst[i] = src[i];
  free(u);
}

/* Diagonal by probing every cell with local unit vectors, summed over cells, 1 on
 * constrained rows; the restated deal.II MatrixFreeTools::compute_diagonal called at
 * include/operators/portable_laplace_operator_bk3.h:545-550. Returns diag (not inverted). */
void orc_diagonal(int p, int64_t C, int64_t N, const uint32_t *idx, const double *G,
                  const uint8_t *constrained, double *diag)
{
  const int n = p + 1, n3 = n * n * n;
  double S[64], D[64];
  orc_shape_tables(p, n, S, NULL, D, NULL);
  double *buf = (double *)malloc(sizeof(double) * 7 * n3);
  double *u = buf, *out = buf + n3, *w0 = buf + 2 * n3, *w1 = buf + 3 * n3, *rr = buf + 4 * n3,
         *rs = buf + 5 * n3, *rt = buf + 6 * n3;
  for (int64_t i = 0; i < N; ++i) diag[i] = 0.0;
  for (int64_t c = 0; c < C; ++c) {
    const uint32_t *ci = idx + c * n3;
    for (int l = 0; l < n3; ++l) {
      if (ci[l] == ORC_INVALID) continue;
      for (int m = 0; m < n3; ++m) u[m] = (m == l) ? 1.0 : 0.0;
      bk3_cell(n, S, D, G + c * 6 * n3, u, out, w0, w1, rr, rs, rt);
      diag[ci[l]] += out[l];
    }
  }
  for (int64_t i = 0; i < N; ++i)
    if (constrained[i]) diag[i] = 1.0;
  free(buf);
}

/* Right-hand side b_i = sum_cells sum_q phi_i(x_q) f(x_q) JxW_q with QGauss(nq), zero on
 * constrained DoFs (tests/poisson_cube_bk3/program.cc:517-566 for f = 1).
 * f_kind 0: f = 1;  f_kind 1: f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z). */
void orc_box_rhs(const orc_box *b, int p, int nq, int f_kind, const uint32_t *plain,
                 const uint8_t *constrained, int64_t N, double *rhs)
{
  const int nm = p + 1, nm3 = nm * nm * nm, nq3 = nq * nq * nq;
  const int64_t C = orc_box_ncells(b);
  double *xq = (double *)malloc(sizeof(double) * C * nq3 * 3);
  double *jxw = (double *)malloc(sizeof(double) * C * nq3);
  double *S = (double *)malloc(sizeof(double) * nm * nq);
  orc_box_quadrature(b, p, nq, xq, jxw);
  orc_shape_tables(p, nq, S, NULL, NULL, NULL);
  for (int64_t i = 0; i < N; ++i) rhs[i] = 0.0;
  for (int64_t c = 0; c < C; ++c)
    for (int k = 0; k < nm; ++k)
      for (int j = 0; j < nm; ++j)
        for (int i = 0; i < nm; ++i) {
          double s = 0;
          for (int q2 = 0; q2 < nq; ++q2)
            for (int q1 = 0; q1 < nq; ++q1)
              for (int q0 = 0; q0 < nq; ++q0) {
                const int q = (q2 * nq + q1) * nq + q0;
                const double *x = xq + (c * nq3 + q) * 3;
                double f = 1.0;
                if (f_kind == 1)
                  f = 3.0 * ORC_PI * ORC_PI * sin(ORC_PI * x[0]) * sin(ORC_PI * x[1]) *
                      sin(ORC_PI * x[2]);
                s += S[i * nq + q0] * S[j * nq + q1] * S[k * nq + q2] * f * jxw[c * nq3 + q];
              }
          rhs[plain[c * nm3 + (k * nm + j) * nm + i]] += s;
        }
  for (int64_t i = 0; i < N; ++i)
    if (constrained[i]) rhs[i] = 0.0;
  free(xq); free(jxw); free(S);
}

/* L2 error of the FE function u against sin(pi x) sin(pi y) sin(pi z), QGauss(nq). */
double orc_box_l2_error_sine(const orc_box *b, int p, int nq, const uint32_t *plain,
                             const double *u)
{
  const int nm = p + 1, nm3 = nm * nm * nm, nq3 = nq * nq * nq;
  const int64_t C = orc_box_ncells(b);
  double *xq = (double *)malloc(sizeof(double) * C * nq3 * 3);
  double *jxw = (double *)malloc(sizeof(double) * C * nq3);
  double *S = (double *)malloc(sizeof(double) * nm * nq);
  orc_box_quadrature(b, p, nq, xq, jxw);
  orc_shape_tables(p, nq, S, NULL, NULL, NULL);
  double err = 0;
  for (int64_t c = 0; c < C; ++c)
    for (int q2 = 0; q2 < nq; ++q2)
      for (int q1 = 0; q1 < nq; ++q1)
        for (int q0 = 0; q0 < nq; ++q0) {
          const int q = (q2 * nq + q1) * nq + q0;
          double v = 0;
          for (int k = 0; k < nm; ++k)
            for (int j = 0; j < nm; ++j)
              for (int i = 0; i < nm; ++i)
                v += u[plain[c * nm3 + (k * nm + j) * nm + i]] * S[i * nq + q0] *
                     S[j * nq + q1] * S[k * nq + q2];
          const double *x = xq + (c * nq3 + q) * 3;
          const double ex = sin(ORC_PI * x[0]) * sin(ORC_PI * x[1]) * sin(ORC_PI * x[2]);
          err += (v - ex) * (v - ex) * jxw[c * nq3 + q];
        }
  free(xq); free(jxw); free(S);
  return sqrt(err);
}

/* ------------------------------------------------------------------------------------ */
/* 5. Multigrid transfers                                                                */
/* ------------------------------------------------------------------------------------ */

/* A transfer between two levels on cell patches: every patch carries the coarse DoFs
 * (with the sentinel) and the fine DoFs without it, plus a weight per fine patch entry
 * (1/number of patches holding the DoF, 0 when constrained;
 * portable_polynomial_transfer.h:1155-1245 and portable_geometric_transfer.h:1344-1397).
 * P1d is [nc*nf] stored [i_c*nf + j_f]. */
typedef struct {
  int nc, nf;
  int64_t n_patches;
  uint32_t *coarse_idx; /* [patch][nc^3] */
  uint32_t *fine_idx;   /* [patch][nf^3] */
  double *weights;      /* [patch][nf^3] */
  double *P1d;
  int prolong_times; /* 1, or 2 to mimic the double add of the reference h-prolongation */
} orc_transfer;

static void transfer_weights(orc_transfer *t, int64_t n_fine, const uint8_t *constrained_f)
{
  const int nf3 = t->nf * t->nf * t->nf;
  double *mult = (double *)calloc(n_fine, sizeof(double));
  for (int64_t e = 0; e < t->n_patches * nf3; ++e) mult[t->fine_idx[e]] += 1.0;
  for (int64_t i = 0; i < n_fine; ++i) mult[i] = (mult[i] > 0) ? 1.0 / mult[i] : 0.0;
  for (int64_t i = 0; i < n_fine; ++i)
    if (constrained_f[i]) mult[i] = 0.0;
  t->weights = (double *)malloc(sizeof(double) * t->n_patches * nf3);
  for (int64_t e = 0; e < t->n_patches * nf3; ++e) t->weights[e] = mult[t->fine_idx[e]];
  free(mult);
}

/* apply the tensor-product 1D matrix: in [a^3] -> out [b^3], M[i_in*b + j_out] (forward)
 * or transposed (M[j_out*a + i_in] read as M[i_out*... ]) */
static void tensor_apply(int a, int b, const double *M, int transpose, const double *in,
                         double *out, double *t1, double *t2)
{
  /* out(x3,y3,z3) = sum M(.)(.) in ; M indexed so that forward: out_j = sum_i M[i*b+j] in_i,
   * transposed (a = fine size, b = coarse size): out_i = sum_j M[i*a+j] in_j */
#define MM(i_in, j_out) (transpose ? M[(j_out) * a + (i_in)] : M[(i_in) * b + (j_out)])
  /* x */
  for (int k = 0; k < a; ++k)
    for (int j = 0; j < a; ++j)
      for (int q = 0; q < b; ++q) {
        double s = 0;
        for (int i = 0; i < a; ++i) s += MM(i, q) * in[(k * a + j) * a + i];
        t1[(k * a + j) * b + q] = s;
      }
  /* y */
  for (int k = 0; k < a; ++k)
    for (int q = 0; q < b; ++q)
      for (int x = 0; x < b; ++x) {
        double s = 0;
        for (int j = 0; j < a; ++j) s += MM(j, q) * t1[(k * a + j) * b + x];
        t2[(k * b + q) * b + x] = s;
      }
  /* z */
  for (int r = 0; r < b; ++r)
    for (int y = 0; y < b; ++y)
      for (int x = 0; x < b; ++x) {
        double s = 0;
        for (int k = 0; k < a; ++k) s += MM(k, r) * t2[(k * b + y) * b + x];
        out[(r * b + y) * b + x] = s;
      }
#undef MM
}

/* prolongate_and_add: dst_fine += W o (P x P x P) src_coarse (bk1_kokkos_kernels.h:462-759) */
void orc_transfer_prolongate_add(const orc_transfer *t, double *dst_f, const double *src_c)
{
  const int nc = t->nc, nf = t->nf, nc3 = nc * nc * nc, nf3 = nf * nf * nf;
  double *u = (double *)malloc(sizeof(double) * (nc3 + 3 * nf3));
  double *v = u + nc3, *t1 = v + nf3, *t2 = t1 + nf3;
  for (int rep = 0; rep < t->prolong_times; ++rep)
    for (int64_t c = 0; c < t->n_patches; ++c) {
      const uint32_t *ci = t->coarse_idx + c * nc3;
      for (int l = 0; l < nc3; ++l) u[l] = (ci[l] == ORC_INVALID) ? 0.0 : src_c[ci[l]];
      tensor_apply(nc, nf, t->P1d, 0, u, v, t1, t2);
      for (int l = 0; l < nf3; ++l)
        dst_f[t->fine_idx[c * nf3 + l]] += t->weights[c * nf3 + l] * v[l];
    }
  free(u);
}

/* restrict_and_add: dst_coarse += (P^T x P^T x P^T)(W o src_fine), constrained coarse
 * entries skipped (bk1_kokkos_kernels.h:761-1051) */
void orc_transfer_restrict_add(const orc_transfer *t, double *dst_c, const double *src_f)
{
  const int nc = t->nc, nf = t->nf, nc3 = nc * nc * nc, nf3 = nf * nf * nf;
  double *u = (double *)malloc(sizeof(double) * (nc3 + 3 * nf3));
  double *v = u + nc3, *t1 = v + nf3, *t2 = t1 + nf3;
  for (int64_t c = 0; c < t->n_patches; ++c) {
    for (int l = 0; l < nf3; ++l)
      v[l] = t->weights[c * nf3 + l] * src_f[t->fine_idx[c * nf3 + l]];
    tensor_apply(nf, nc, t->P1d, 1, v, u, t1, t2);
    const uint32_t *ci = t->coarse_idx + c * nc3;
    for (int l = 0; l < nc3; ++l)
      if (ci[l] != ORC_INVALID) dst_c[ci[l]] += u[l];
  }
  free(u);
}

/* ------------------------------------------------------------------------------------ */
/* 6. Levels, Chebyshev smoother, V-cycle and CG                                          */
/* ------------------------------------------------------------------------------------ */

typedef struct {
  orc_box box;
  int p;
  int dg;       /* 1: DG-SIPG level (orc_dg_vmult), numbering cell * (p+1)^3 + l */
  double c_pen; /* DG penalty factor */
  int64_t C, N;
  uint32_t *plain, *idx, *lattice;
  uint8_t *constrained, *color;
  double *G, *invdiag;
  /* Chebyshev state (deal.II PreconditionChebyshev, restated) */
  int cheb_degree, eig_iterations, eig_done;
  double smoothing_range, theta, delta, min_ev, max_ev;
  int cg_eig_its;
  double *sol, *def, *t, *old, *tmp;
} orc_level;

static void level_init(orc_level *L, const orc_box *b, int p, int coeff_kind)
{
  memset(L, 0, sizeof(*L));
  L->box = *b;
  L->p = p;
  L->C = orc_box_ncells(b);
  const int nm3 = (p + 1) * (p + 1) * (p + 1);
  int64_t n[3];
  box_ncells(b, n);
  const int64_t nlat = (p * n[0] + 1) * (p * n[1] + 1) * (p * n[2] + 1);
  L->plain = (uint32_t *)malloc(sizeof(uint32_t) * L->C * nm3);
  L->idx = (uint32_t *)malloc(sizeof(uint32_t) * L->C * nm3);
  L->lattice = (uint32_t *)malloc(sizeof(uint32_t) * nlat);
  L->constrained = (uint8_t *)malloc(nlat);
  L->N = orc_box_dofs(b, p, L->plain, L->constrained, L->lattice);
  orc_apply_sentinel(L->C * nm3, L->plain, L->constrained, L->idx);
  L->G = (double *)malloc(sizeof(double) * L->C * 6 * nm3);
  orc_box_G(b, p, coeff_kind, NULL, L->G);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * L->C);
  orc_box_cell_coords(b, cx, cx + L->C, cx + 2 * L->C);
  L->color = (uint8_t *)malloc(L->C);
  for (int64_t c = 0; c < L->C; ++c)
    L->color[c] = (uint8_t)((cx[c] & 1) | ((cx[L->C + c] & 1) << 1) | ((cx[2 * L->C + c] & 1) << 2));
  free(cx);
  L->invdiag = (double *)malloc(sizeof(double) * L->N);
  orc_diagonal(p, L->C, L->N, L->idx, L->G, L->constrained, L->invdiag);
  for (int64_t i = 0; i < L->N; ++i) L->invdiag[i] = 1.0 / L->invdiag[i];
  L->sol = (double *)calloc(L->N, sizeof(double));
  L->def = (double *)calloc(L->N, sizeof(double));
  L->t = (double *)calloc(L->N, sizeof(double));
  L->old = (double *)calloc(L->N, sizeof(double));
  L->tmp = (double *)calloc(L->N, sizeof(double));
}

static void level_free(orc_level *L)
{
  free(L->plain); free(L->idx); free(L->lattice); free(L->constrained); free(L->color);
  free(L->G); free(L->invdiag); free(L->sol); free(L->def); free(L->t); free(L->old);
  free(L->tmp);
}

void orc_dg_vmult(const orc_box *b, int p, double c_pen, const double *src, double *dst);
void orc_dg_diagonal(const orc_box *b, int p, double c_pen, double *diag);

static void level_vmult(const orc_level *L, double *dst, const double *src)
{
  if (L->dg) orc_dg_vmult(&L->box, L->p, L->c_pen, src, dst);
  else orc_vmult(L->p, L->C, L->N, L->idx, L->G, L->constrained, L->color, src, dst);
}

static void level_init_dg(orc_level *L, const orc_box *b, int p, double c_pen)
{
  memset(L, 0, sizeof(*L));
  L->box = *b;
  L->p = p;
  L->dg = 1;
  L->c_pen = c_pen;
  L->C = orc_box_ncells(b);
  const int nm3 = (p + 1) * (p + 1) * (p + 1);
  L->N = L->C * nm3;
  L->plain = (uint32_t *)malloc(sizeof(uint32_t) * L->N);
  L->idx = (uint32_t *)malloc(sizeof(uint32_t) * L->N);
  for (int64_t i = 0; i < L->N; ++i) L->plain[i] = L->idx[i] = (uint32_t)i;
  L->constrained = (uint8_t *)calloc(L->N, 1);
  L->invdiag = (double *)malloc(sizeof(double) * L->N);
  orc_dg_diagonal(b, p, c_pen, L->invdiag);
  for (int64_t i = 0; i < L->N; ++i) L->invdiag[i] = 1.0 / L->invdiag[i];
  L->sol = (double *)calloc(L->N, sizeof(double));
  L->def = (double *)calloc(L->N, sizeof(double));
  L->t = (double *)calloc(L->N, sizeof(double));
  L->old = (double *)calloc(L->N, sizeof(double));
  L->tmp = (double *)calloc(L->N, sizeof(double));
}

static double dot(int64_t n, const double *a, const double *b)
{
  double s = 0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* extreme eigenvalues of a symmetric tridiagonal matrix by Sturm-sequence bisection */
static int sturm_count(int n, const double *a, const double *b, double x)
{
  int cnt = 0;
  double d = 1.0;
  for (int i = 0; i < n; ++i) {
    const double bb = (i > 0) ? b[i - 1] * b[i - 1] : 0.0;
    d = a[i] - x - ((i > 0) ? bb / d : 0.0);
    if (d == 0.0) d = -1e-300;
    if (d < 0) ++cnt;
  }
  return cnt;
}

static double tridiag_eig(int n, const double *a, const double *b, int which /*0 min,1 max*/)
{
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < n; ++i) {
    const double r = ((i > 0) ? fabs(b[i - 1]) : 0.0) + ((i < n - 1) ? fabs(b[i]) : 0.0);
    if (a[i] - r < lo) lo = a[i] - r;
    if (a[i] + r > hi) hi = a[i] + r;
  }
  const int target = (which == 0) ? 1 : n; /* count(<x) >= target */
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (sturm_count(n, a, b, mid) >= target) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

/* Eigenvalue estimate of deal.II PreconditionChebyshev: a preconditioned CG run of at most
 * eig_iterations steps (IterationNumberControl, tolerance 1e-10) from x = 0 on the
 * right-hand side v_i = (i mod 11) - mean, the Lanczos matrix assembled from the CG
 * coefficients with deal.II's one-step lag, max scaled by 1.2; then the interval
 * [alpha, max] with alpha = max/range (range > 1) or min(0.9 max, min), and for an
 * invalid degree the degree reaching `range` by the Chebyshev error bound.
 * Called from the smoothers set up at tests/poisson_cube_bk3/program.cc:474-515. */
static void cheb_estimate(orc_level *L)
{
  const int64_t N = L->N;
  double *x = (double *)calloc(N, sizeof(double));
  double *r = (double *)malloc(sizeof(double) * N);
  double *z = (double *)malloc(sizeof(double) * N);
  double *pv = (double *)malloc(sizeof(double) * N);
  double *v = (double *)malloc(sizeof(double) * N);
  double mean = 0;
  for (int64_t i = 0; i < N; ++i) { r[i] = (double)(i % 11); mean += r[i]; }
  mean /= (double)N;
  for (int64_t i = 0; i < N; ++i) r[i] -= mean;
  int maxit = L->eig_iterations;
  double *diag = (double *)malloc(sizeof(double) * (maxit + 2));
  double *offd = (double *)malloc(sizeof(double) * (maxit + 2));
  int n_t = 0;
  double res = sqrt(dot(N, r, r));
  int it = 0;
  if (!(res <= 1e-10) && maxit > 0) {
    for (int64_t i = 0; i < N; ++i) z[i] = L->invdiag[i] * r[i];
    double rho = dot(N, r, z), rho_old = rho;
    double alpha = 0, prev_alpha = 0, beta = 0, eig_beta_alpha = 0;
    while (1) {
      ++it;
      if (it > 1) {
        beta = rho / rho_old;
        for (int64_t i = 0; i < N; ++i) pv[i] = z[i] + beta * pv[i];
      } else {
        for (int64_t i = 0; i < N; ++i) pv[i] = z[i];
      }
      level_vmult(L, v, pv);
      prev_alpha = alpha;
      alpha = rho / dot(N, pv, v);
      for (int64_t i = 0; i < N; ++i) { x[i] += alpha * pv[i]; r[i] -= alpha * v[i]; }
      res = sqrt(dot(N, r, r));
      for (int64_t i = 0; i < N; ++i) z[i] = L->invdiag[i] * r[i];
      rho_old = rho;
      rho = dot(N, r, z);
      if (it > 1) {
        diag[n_t] = 1.0 / prev_alpha + eig_beta_alpha;
        eig_beta_alpha = beta / prev_alpha;
        offd[n_t] = sqrt(beta) / prev_alpha;
        ++n_t;
      }
      if (it >= maxit || res <= 1e-10) break;
    }
  }
  L->cg_eig_its = it;
  if (n_t == 0) {
    L->min_ev = L->max_ev = 1.0;
  } else {
    L->min_ev = tridiag_eig(n_t, diag, offd, 0);
    L->max_ev = 1.2 * tridiag_eig(n_t, diag, offd, 1);
  }
  const double alpha_ev = (L->smoothing_range > 1.0)
                              ? L->max_ev / L->smoothing_range
                              : fmin(0.9 * L->max_ev, L->min_ev);
  if (L->cheb_degree <= 0) {
    const double actual_range = L->max_ev / alpha_ev;
    const double sigma = (1.0 - sqrt(1.0 / actual_range)) / (1.0 + sqrt(1.0 / actual_range));
    const double eps = L->smoothing_range;
    L->cheb_degree =
        1 + (int)(log(1.0 / eps + sqrt(1.0 / eps / eps - 1.0)) / log(1.0 / sigma));
  }
  L->delta = (L->max_ev - alpha_ev) * 0.5;
  L->theta = (L->max_ev + alpha_ev) * 0.5;
  L->eig_done = 1;
  free(x); free(r); free(z); free(pv); free(v); free(diag); free(offd);
}

/* Chebyshev iteration (first kind) with the Jacobi preconditioner:
 * vmult: x_0 = 0, degree-1 matrix-vector products; step: x_0 = dst, degree products. */
static void cheb_run(orc_level *L, double *dst, const double *src, int from_zero)
{
  const int64_t N = L->N;
  if (!L->eig_done) cheb_estimate(L);
  double *xo = L->old, *Ax = L->tmp;
  if (from_zero) {
    for (int64_t i = 0; i < N; ++i) { xo[i] = 0.0; dst[i] = L->invdiag[i] * src[i] / L->theta; }
  } else {
    level_vmult(L, Ax, dst);
    for (int64_t i = 0; i < N; ++i) {
      xo[i] = dst[i];
      dst[i] += L->invdiag[i] * (src[i] - Ax[i]) / L->theta;
    }
  }
  if (L->cheb_degree < 2 || fabs(L->delta) < 1e-40) return;
  double rhok = L->delta / L->theta;
  const double sigma = L->theta / L->delta;
  for (int k = 1; k < L->cheb_degree; ++k) {
    level_vmult(L, Ax, dst);
    const double rhokp = 1.0 / (2.0 * sigma - rhok);
    const double f1 = rhokp * rhok, f2 = 2.0 * rhokp / L->delta;
    rhok = rhokp;
    for (int64_t i = 0; i < N; ++i) {
      const double xn = dst[i] + f1 * (dst[i] - xo[i]) + f2 * L->invdiag[i] * (src[i] - Ax[i]);
      xo[i] = dst[i];
      dst[i] = xn;
    }
  }
}

typedef struct {
  int n_levels;
  orc_level *levels;
  orc_transfer *transfers; /* transfers[l] between level l-1 and l, l >= 1 */
} orc_mg;

static void vcycle(orc_mg *mg, int l)
{
  orc_level *L = &mg->levels[l];
  if (l == 0) {
    cheb_run(L, L->sol, L->def, 1);
    return;
  }
  orc_level *Lc = &mg->levels[l - 1];
  cheb_run(L, L->sol, L->def, 1);
  level_vmult(L, L->t, L->sol);
  for (int64_t i = 0; i < L->N; ++i) L->t[i] = L->def[i] - L->t[i];
  for (int64_t i = 0; i < Lc->N; ++i) Lc->def[i] = 0.0;
  orc_transfer_restrict_add(&mg->transfers[l], Lc->def, L->t);
  vcycle(mg, l - 1);
  orc_transfer_prolongate_add(&mg->transfers[l], L->sol, Lc->sol);
  cheb_run(L, L->sol, L->def, 0);
}

static void build_h_transfer(orc_transfer *t, const orc_level *Lc, const orc_level *Lf,
                             int times)
{
  const int p = Lc->p, nc = p + 1, nf = 2 * p + 1, nc3 = nc * nc * nc, nf3 = nf * nf * nf;
  int64_t nfine[3];
  box_ncells(&Lf->box, nfine);
  const int64_t L0 = p * nfine[0] + 1, L1 = p * nfine[1] + 1;
  t->nc = nc;
  t->nf = nf;
  t->n_patches = Lc->C;
  t->prolong_times = times;
  t->coarse_idx = (uint32_t *)malloc(sizeof(uint32_t) * Lc->C * nc3);
  t->fine_idx = (uint32_t *)malloc(sizeof(uint32_t) * Lc->C * nf3);
  memcpy(t->coarse_idx, Lc->idx, sizeof(uint32_t) * Lc->C * nc3);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * Lc->C);
  orc_box_cell_coords(&Lc->box, cx, cx + Lc->C, cx + 2 * Lc->C);
  for (int64_t c = 0; c < Lc->C; ++c)
    for (int k = 0; k < nf; ++k)
      for (int j = 0; j < nf; ++j)
        for (int i = 0; i < nf; ++i) {
          const int64_t gx = 2LL * p * cx[c] + i, gy = 2LL * p * cx[Lc->C + c] + j,
                        gz = 2LL * p * cx[2 * Lc->C + c] + k;
          t->fine_idx[c * nf3 + (k * nf + j) * nf + i] = Lf->lattice[(gz * L1 + gy) * L0 + gx];
        }
  free(cx);
  t->P1d = (double *)malloc(sizeof(double) * nc * nf);
  orc_h_prolongation_matrix(p, t->P1d);
  transfer_weights(t, Lf->N, Lf->constrained);
}

static void build_p_transfer(orc_transfer *t, const orc_level *Lc, const orc_level *Lf)
{
  const int nc = Lc->p + 1, nf = Lf->p + 1, nc3 = nc * nc * nc, nf3 = nf * nf * nf;
  t->nc = nc;
  t->nf = nf;
  t->n_patches = Lc->C;
  t->prolong_times = 1;
  t->coarse_idx = (uint32_t *)malloc(sizeof(uint32_t) * Lc->C * nc3);
  t->fine_idx = (uint32_t *)malloc(sizeof(uint32_t) * Lf->C * nf3);
  memcpy(t->coarse_idx, Lc->idx, sizeof(uint32_t) * Lc->C * nc3);
  memcpy(t->fine_idx, Lf->plain, sizeof(uint32_t) * Lf->C * nf3);
  t->P1d = (double *)malloc(sizeof(double) * nc * nf);
  orc_projection_matrix(Lc->p, Lf->p, t->P1d);
  transfer_weights(t, Lf->N, Lf->constrained);
}

static void transfer_free(orc_transfer *t)
{
  free(t->coarse_idx); free(t->fine_idx); free(t->weights); free(t->P1d);
}

/* Result of one ph-multigrid preconditioned CG solve. */
typedef struct {
  int32_t iterations;
  int32_t n_levels;
  double initial_residual;
  double final_residual;
  double reduction_per_step;
  double l2_error; /* against sin(pi x)sin(pi y)sin(pi z) when rhs_kind == 1, else -1 */
  int64_t n_dofs;
  int32_t level_degree[32];
  int32_t level_cheb_degree[32];
  double level_max_ev[32];
  double level_min_ev[32];
  int64_t level_dofs[32];
} orc_solve_info;

/* The multigrid solver of tests/common/portable_multigrid_solver.h restated on the CPU:
 * h-levels 0..refine with FE_Q(h_degree) on every refinement of the box, then p-levels on
 * the finest mesh for the degrees in pseq (descending, last = h_degree).  h_degree = 1 is the
 * ph-multigrid of tests/poisson_cube_bk3/program.cc:263-292 (p_levels as at :289-292); pseq =
 * {p} with h_degree = p is the plain geometric multigrid of
 * source/geometric_multigrid/program.cc:245-249 (GeometricTransfer<dim, fe_degree> between
 * consecutive refinements at one degree).  Chebyshev degree `cheb` with range 15 and 10
 * eigenvalue iterations on levels > 0, Chebyshev-to-1e-3 on level 0; PCG with
 * ReductionControl(maxit, abs_tol, reduce) (portable_multigrid_solver.h:147-169).
 * x_out (nullable) receives the solution on the finest level. */
int orc_solve_box_hdeg(const orc_box *box, const int32_t *pseq, int n_pseq, int h_degree, int cheb,
                       int h_times, int rhs_kind, int coeff_kind, double reduce, double abs_tol,
                       int maxit, orc_solve_info *info, double *x_out)
{
  memset(info, 0, sizeof(*info));
  const int n_h = box->refine + 1;
  const int n_levels = n_h + n_pseq - 1;
  if (n_levels > 32 || h_degree < 1 || pseq[n_pseq - 1] != h_degree) return -1;
  orc_mg mg;
  mg.n_levels = n_levels;
  mg.levels = (orc_level *)calloc(n_levels, sizeof(orc_level));
  mg.transfers = (orc_transfer *)calloc(n_levels, sizeof(orc_transfer));
  for (int l = 0; l < n_levels; ++l) {
    orc_box b = *box;
    int p = h_degree;
    if (l < n_h) b.refine = l;
    else p = pseq[n_pseq - 1 - (l - n_h + 1)];
    level_init(&mg.levels[l], &b, p, coeff_kind);
    orc_level *L = &mg.levels[l];
    if (l > 0) {
      L->cheb_degree = cheb;
      L->smoothing_range = 15.0;
      L->eig_iterations = 10;
    } else {
      L->cheb_degree = 0; /* invalid: chosen from the range */
      L->smoothing_range = 1e-3;
      L->eig_iterations = (int)L->N;
    }
    cheb_estimate(L);
    info->level_degree[l] = p;
    info->level_cheb_degree[l] = L->cheb_degree;
    info->level_max_ev[l] = L->max_ev;
    info->level_min_ev[l] = L->min_ev;
    info->level_dofs[l] = L->N;
  }
  for (int l = 1; l < n_levels; ++l) {
    if (l < n_h) build_h_transfer(&mg.transfers[l], &mg.levels[l - 1], &mg.levels[l], h_times);
    else build_p_transfer(&mg.transfers[l], &mg.levels[l - 1], &mg.levels[l]);
  }
  orc_level *F = &mg.levels[n_levels - 1];
  const int64_t N = F->N;
  info->n_dofs = N;
  info->n_levels = n_levels;
  double *b = (double *)malloc(sizeof(double) * N);
  orc_box_rhs(box, F->p, F->p + (rhs_kind == 1 ? 2 : 1), rhs_kind, F->plain, F->constrained, N,
              b);
  double *x = (double *)calloc(N, sizeof(double));
  double *r = (double *)malloc(sizeof(double) * N);
  double *z = (double *)malloc(sizeof(double) * N);
  double *pv = (double *)malloc(sizeof(double) * N);
  double *v = (double *)malloc(sizeof(double) * N);
  memcpy(r, b, sizeof(double) * N);
  double res = sqrt(dot(N, r, r));
  info->initial_residual = res;
  const double tol = fmax(abs_tol, reduce * res);
  int it = 0;
  if (res > tol) {
    double rho = 0, rho_old = 0;
    while (1) {
      /* preconditioner: V-cycle on the residual */
      for (int l = 0; l < n_levels - 1; ++l)
        for (int64_t i = 0; i < mg.levels[l].N; ++i) mg.levels[l].def[i] = 0.0;
      memcpy(F->def, r, sizeof(double) * N);
      vcycle(&mg, n_levels - 1);
      memcpy(z, F->sol, sizeof(double) * N);
      rho_old = rho;
      rho = dot(N, r, z);
      if (it == 0) memcpy(pv, z, sizeof(double) * N);
      else {
        const double beta = rho / rho_old;
        for (int64_t i = 0; i < N; ++i) pv[i] = z[i] + beta * pv[i];
      }
      ++it;
      level_vmult(F, v, pv);
      const double alpha = rho / dot(N, pv, v);
      for (int64_t i = 0; i < N; ++i) { x[i] += alpha * pv[i]; r[i] -= alpha * v[i]; }
      res = sqrt(dot(N, r, r));
      if (res <= tol || it >= maxit) break;
    }
  }
  info->iterations = it;
  info->final_residual = res;
  info->reduction_per_step = (it > 0) ? pow(res / info->initial_residual, 1.0 / it) : 1.0;
  info->l2_error = (rhs_kind == 1) ? orc_box_l2_error_sine(box, F->p, F->p + 2, F->plain, x) : -1;
  if (x_out) memcpy(x_out, x, sizeof(double) * N);
  free(b); free(x); free(r); free(z); free(pv); free(v);
  for (int l = 1; l < n_levels; ++l) transfer_free(&mg.transfers[l]);
  for (int l = 0; l < n_levels; ++l) level_free(&mg.levels[l]);
  free(mg.levels);
  free(mg.transfers);
  return 0;
}

/* ph-multigrid with FE_Q(1) h-levels (pseq ends in 1). */
int orc_solve_box(const orc_box *box, const int32_t *pseq, int n_pseq, int cheb, int h_times,
                  int rhs_kind, int coeff_kind, double reduce, double abs_tol, int maxit,
                  orc_solve_info *info, double *x_out)
{
  return orc_solve_box_hdeg(box, pseq, n_pseq, 1, cheb, h_times, rhs_kind, coeff_kind, reduce, abs_tol,
                            maxit, info, x_out);
}

/* Single-level transfer construction for tests: p-transfer between degrees pc < pf on the
 * same box, or h-transfer (pc == pf) from box refine-1 to box. Outputs sized by the
 * caller via orc_transfer_sizes. */
int orc_transfer_sizes(const orc_box *fine_box, int pc, int pf, int64_t *n_patches,
                       int64_t *n_coarse, int64_t *n_fine)
{
  orc_box cb = *fine_box;
  if (pc == pf) {
    if (fine_box->refine < 1) return -1;
    cb.refine -= 1;
    *n_patches = orc_box_ncells(&cb);
  } else {
    *n_patches = orc_box_ncells(fine_box);
  }
  *n_coarse = orc_box_dofs(&cb, pc, NULL, NULL, NULL);
  *n_fine = orc_box_dofs(fine_box, pf, NULL, NULL, NULL);
  return 0;
}

int orc_transfer_apply(const orc_box *fine_box, int pc, int pf, int h_times, int direction,
                       const double *src, double *dst)
{
  orc_box cb = *fine_box;
  if (pc == pf) cb.refine -= 1;
  orc_level Lc, Lf;
  level_init(&Lc, &cb, pc, 0);
  level_init(&Lf, fine_box, pf, 0);
  orc_transfer t;
  if (pc == pf) build_h_transfer(&t, &Lc, &Lf, h_times);
  else build_p_transfer(&t, &Lc, &Lf);
  if (direction == 0) orc_transfer_prolongate_add(&t, dst, src);
  else orc_transfer_restrict_add(&t, dst, src);
  transfer_free(&t);
  level_free(&Lc);
  level_free(&Lf);
  return 0;
}

/* Chebyshev smoother of one level (for tests): returns the estimated interval and degree,
 * and applies vmult (mode 0) or step (mode 1) once. */
int orc_chebyshev_apply(const orc_box *box, int p, int degree, double range, int eig_its,
                        int mode, const double *src, double *dst, double *min_ev,
                        double *max_ev, int *degree_out)
{
  orc_level L;
  level_init(&L, box, p, 0);
  L.cheb_degree = degree;
  L.smoothing_range = range;
  L.eig_iterations = eig_its;
  cheb_estimate(&L);
  cheb_run(&L, dst, src, mode == 0);
  *min_ev = L.min_ev;
  *max_ev = L.max_ev;
  *degree_out = L.cheb_degree;
  level_free(&L);
  return 0;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------------------ */
/* 7. DG-SIPG operator on axis-aligned boxes                                             */
/* ------------------------------------------------------------------------------------ */

/* Discontinuous FE_DGQ(p) (Lagrange on Gauss-Lobatto points) with the symmetric interior
 * penalty form of source/plain_laplace_solver_dg/program.cc:106-217 (and the GPU operator
 * include/operators/portable_laplace_operator_dg.h + include/kernels/laplace_dg_kokkos_kernels.h):
 *   inner faces:    [[v]] (sigma [[u]] - {d_n u}) - {d_n v} [[u]]
 *   Dirichlet faces (mirror u+ = -u-, d_n u+ = d_n u-, laplace_dg_kokkos_kernels.h:1560-1569):
 *                   v (2 sigma u - d_n u) - u d_n v
 *   sigma = c_pen * (1/h- + 1/h+)/2 on inner faces, c_pen / h on boundary faces, h the cell
 *   extent normal to the face; the reference uses c_pen = p (p+1)
 *   (portable_laplace_operator_dg.h:147-151).
 * DoFs are numbered cell by cell, dof = cell * (p+1)^3 + lexicographic local index. Faces are
 * integrated with the (p+1)-point Gauss rule in each tangential direction. */

static void box_cell_h(const orc_box *b, double h[3])
{
  int64_t n[3];
  box_ncells(b, n);
  for (int d = 0; d < 3; ++d) h[d] = (b->hi[d] - b->lo[d]) / (double)n[d];
}

/* cell index of coordinates (or -1), inverse of orc_box_cell_coords */
static int64_t *box_cell_lookup(const orc_box *b, int32_t *cx)
{
  int64_t n[3];
  box_ncells(b, n);
  const int64_t C = n[0] * n[1] * n[2];
  int64_t *lut = (int64_t *)malloc(sizeof(int64_t) * C);
  for (int64_t c = 0; c < C; ++c) lut[((int64_t)cx[2 * C + c] * n[1] + cx[C + c]) * n[0] + cx[c]] = c;
  return lut;
}

/* evaluate value and derivative along d of cell data u at reference point xi */
static void eval_point(int N, const double *xl_unused, const double *u, const ld *nodes,
                       const double xi[3], int d, double *val, double *dd)
{
  double phi[3][16], dphi[3][16];
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < N; ++i) {
      phi[a][i] = (double)lagrange(N, nodes, i, (ld)xi[a]);
      dphi[a][i] = (double)lagrange_deriv(N, nodes, i, (ld)xi[a]);
    }
  double v = 0, g = 0;
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        const double x = u[(k * N + j) * N + i];
        v += x * phi[0][i] * phi[1][j] * phi[2][k];
        const double f0 = d == 0 ? dphi[0][i] : phi[0][i];
        const double f1 = d == 1 ? dphi[1][j] : phi[1][j];
        const double f2 = d == 2 ? dphi[2][k] : phi[2][k];
        g += x * f0 * f1 * f2;
      }
  *val = v;
  *dd = g;
}

/* add test contributions tv * phi_l(xi) + tn * d_d phi_l(xi) to out[l] */
static void test_point(int N, const ld *nodes, const double xi[3], int d, double tv, double tn,
                       double *out)
{
  double phi[3][16], dphi[3][16];
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < N; ++i) {
      phi[a][i] = (double)lagrange(N, nodes, i, (ld)xi[a]);
      dphi[a][i] = (double)lagrange_deriv(N, nodes, i, (ld)xi[a]);
    }
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        const double f0 = d == 0 ? dphi[0][i] : phi[0][i];
        const double f1 = d == 1 ? dphi[1][j] : phi[1][j];
        const double f2 = d == 2 ? dphi[2][k] : phi[2][k];
        out[(k * N + j) * N + i] += tv * phi[0][i] * phi[1][j] * phi[2][k] + tn * f0 * f1 * f2;
      }
}

void orc_dg_vmult(const orc_box *b, int p, double c_pen, const double *src, double *dst)
{
  const int N = p + 1, N3 = N * N * N;
  const int64_t C = orc_box_ncells(b);
  double h[3];
  box_cell_h(b, h);
  ld nodes[16], wl[16], xg[16], wg[16];
  gauss_lobatto_ld(N, nodes, wl);
  gauss_ld(N, xg, wg);
  double S[64], D[64], W[8];
  orc_shape_tables(p, N, S, NULL, D, W);
  int64_t n[3];
  box_ncells(b, n);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  orc_box_cell_coords(b, cx, cx + C, cx + 2 * C);
  int64_t *lut = box_cell_lookup(b, cx);
  for (int64_t i = 0; i < C * N3; ++i) dst[i] = 0.0;
  /* cell term: affine G = w_q vol / h_d^2 on the diagonal */
  double *Gc = (double *)calloc(6 * N3, sizeof(double));
  const double vol = h[0] * h[1] * h[2];
  for (int q2 = 0; q2 < N; ++q2)
    for (int q1 = 0; q1 < N; ++q1)
      for (int q0 = 0; q0 < N; ++q0) {
        const int q = (q2 * N + q1) * N + q0;
        const double w = W[q0] * W[q1] * W[q2] * vol;
        Gc[0 * N3 + q] = w / (h[0] * h[0]);
        Gc[3 * N3 + q] = w / (h[1] * h[1]);
        Gc[5 * N3 + q] = w / (h[2] * h[2]);
      }
  double *buf = (double *)malloc(sizeof(double) * 7 * N3);
  for (int64_t c = 0; c < C; ++c) {
    bk3_cell(N, S, D, Gc, src + c * N3, buf + N3, buf + 2 * N3, buf + 3 * N3, buf + 4 * N3,
             buf + 5 * N3, buf + 6 * N3);
    for (int l = 0; l < N3; ++l) dst[c * N3 + l] += buf[N3 + l];
  }
  /* faces: every cell handles its +d inner faces and its boundary faces */
  for (int64_t c = 0; c < C; ++c) {
    const int32_t cc[3] = {cx[c], cx[C + c], cx[2 * C + c]};
    for (int d = 0; d < 3; ++d) {
      const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
      for (int s = 0; s < 2; ++s) {
        int32_t nc[3] = {cc[0], cc[1], cc[2]};
        nc[d] += s ? 1 : -1;
        const int outside = nc[d] < 0 || nc[d] >= n[d];
        if (!outside && s == 0) continue; /* inner faces handled from the minus side */
        const double sign = s ? 1.0 : -1.0; /* outward normal of c: sign * e_d */
        const int64_t nb = outside ? -1 : lut[((int64_t)nc[2] * n[1] + nc[1]) * n[0] + nc[0]];
        const int dirichlet = (b->dirichlet_mask >> (2 * d + s)) & 1;
        if (outside && !dirichlet) continue;
        const double sigma = c_pen / h[d];
        const double jxw_face = h[ta] * h[tb];
        for (int qb = 0; qb < N; ++qb)
          for (int qa = 0; qa < N; ++qa) {
            double xi[3], xin[3];
            xi[d] = s ? 1.0 : 0.0;
            xi[ta] = (double)xg[qa];
            xi[tb] = (double)xg[qb];
            xin[0] = xi[0]; xin[1] = xi[1]; xin[2] = xi[2];
            xin[d] = s ? 0.0 : 1.0;
            const double wq = (double)(wg[qa] * wg[qb]) * jxw_face;
            double um, dm;
            eval_point(N, NULL, src + c * N3, nodes, xi, d, &um, &dm);
            dm *= sign / h[d]; /* normal derivative along the outward normal of c */
            double up, dp;
            if (outside) {
              up = -um;
              dp = dm;
            } else {
              eval_point(N, NULL, src + nb * N3, nodes, xin, d, &up, &dp);
              dp *= sign / h[d];
            }
            const double jump = um - up, avg = 0.5 * (dm + dp);
            const double tv = (sigma * jump - avg) * wq, tn = -0.5 * jump * wq;
            test_point(N, nodes, xi, d, tv, tn * sign / h[d], dst + c * N3);
            if (!outside) test_point(N, nodes, xin, d, -tv, tn * sign / h[d], dst + nb * N3);
          }
      }
    }
  }
  free(buf); free(Gc); free(cx); free(lut);
}

static double dg_exact(const double x[3])
{
  return exp(x[0]) * sin(ORC_PI * x[1]) * cos(ORC_PI * x[2]);
}

/* right-hand side for -lap u = f with u = exp(x) sin(pi y) cos(pi z), f = (2 pi^2 - 1) u, and
 * the Dirichlet data imposed weakly through the mirror: b_l = (f, phi_l) + sum over Dirichlet
 * faces of (g, 2 sigma phi_l - d_n phi_l); nq-point Gauss rules */
void orc_dg_rhs(const orc_box *b, int p, int nq, double c_pen, double *rhs)
{
  const int N = p + 1, N3 = N * N * N;
  const int64_t C = orc_box_ncells(b);
  double h[3];
  box_cell_h(b, h);
  ld nodes[16], wl[16], xg[16], wg[16];
  gauss_lobatto_ld(N, nodes, wl);
  gauss_ld(nq, xg, wg);
  int64_t n[3];
  box_ncells(b, n);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  orc_box_cell_coords(b, cx, cx + C, cx + 2 * C);
  for (int64_t i = 0; i < C * N3; ++i) rhs[i] = 0.0;
  for (int64_t c = 0; c < C; ++c) {
    const int32_t cc[3] = {cx[c], cx[C + c], cx[2 * C + c]};
    for (int q2 = 0; q2 < nq; ++q2)
      for (int q1 = 0; q1 < nq; ++q1)
        for (int q0 = 0; q0 < nq; ++q0) {
          const double xi[3] = {(double)xg[q0], (double)xg[q1], (double)xg[q2]};
          double x[3];
          for (int d = 0; d < 3; ++d) x[d] = b->lo[d] + (cc[d] + xi[d]) * h[d];
          const double w = (double)(wg[q0] * wg[q1] * wg[q2]) * h[0] * h[1] * h[2];
          const double f = (2.0 * ORC_PI * ORC_PI - 1.0) * dg_exact(x);
          test_point(N, nodes, xi, 0, f * w, 0.0, rhs + c * N3);
        }
    for (int d = 0; d < 3; ++d) {
      const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
      for (int s = 0; s < 2; ++s) {
        const int outside = s ? (cc[d] == n[d] - 1) : (cc[d] == 0);
        if (!outside || !((b->dirichlet_mask >> (2 * d + s)) & 1)) continue;
        const double sign = s ? 1.0 : -1.0, sigma = c_pen / h[d];
        for (int qb = 0; qb < nq; ++qb)
          for (int qa = 0; qa < nq; ++qa) {
            double xi[3], x[3];
            xi[d] = s ? 1.0 : 0.0;
            xi[ta] = (double)xg[qa];
            xi[tb] = (double)xg[qb];
            for (int a = 0; a < 3; ++a) x[a] = b->lo[a] + (cc[a] + xi[a]) * h[a];
            const double w = (double)(wg[qa] * wg[qb]) * h[ta] * h[tb];
            const double g = dg_exact(x);
            test_point(N, nodes, xi, d, 2.0 * sigma * g * w, -g * w * sign / h[d], rhs + c * N3);
          }
      }
    }
  }
  free(cx);
}

double orc_dg_l2_error(const orc_box *b, int p, int nq, const double *u)
{
  const int N = p + 1, N3 = N * N * N;
  const int64_t C = orc_box_ncells(b);
  double h[3];
  box_cell_h(b, h);
  ld nodes[16], wl[16], xg[16], wg[16];
  gauss_lobatto_ld(N, nodes, wl);
  gauss_ld(nq, xg, wg);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  orc_box_cell_coords(b, cx, cx + C, cx + 2 * C);
  double err = 0;
  for (int64_t c = 0; c < C; ++c) {
    const int32_t cc[3] = {cx[c], cx[C + c], cx[2 * C + c]};
    for (int q2 = 0; q2 < nq; ++q2)
      for (int q1 = 0; q1 < nq; ++q1)
        for (int q0 = 0; q0 < nq; ++q0) {
          const double xi[3] = {(double)xg[q0], (double)xg[q1], (double)xg[q2]};
          double x[3], v, dummy;
          for (int d = 0; d < 3; ++d) x[d] = b->lo[d] + (cc[d] + xi[d]) * h[d];
          eval_point(N, NULL, u + c * N3, nodes, xi, 0, &v, &dummy);
          const double w = (double)(wg[q0] * wg[q1] * wg[q2]) * h[0] * h[1] * h[2];
          err += (v - dg_exact(x)) * (v - dg_exact(x)) * w;
        }
  }
  free(cx);
  return sqrt(err);
}

/* DG <-> CG transfer at equal degree on the same mesh (ContinuousTransfer,
 * include/multigrid/portable_continuous_transfer.h:110-319): prolongate u_dg[i] += u_cg[map(i)]
 * for CG DoFs that are not constrained; restrict u_cg[map(i)] += u_dg[i] likewise. */
void orc_dg_cg_transfer(const orc_box *b, int p, int direction, const double *src, double *dst)
{
  const int N3 = (p + 1) * (p + 1) * (p + 1);
  const int64_t C = orc_box_ncells(b);
  int64_t n[3];
  box_ncells(b, n);
  const int64_t nlat = (p * n[0] + 1) * (p * n[1] + 1) * (p * n[2] + 1);
  uint32_t *plain = (uint32_t *)malloc(sizeof(uint32_t) * C * N3);
  uint8_t *cons = (uint8_t *)malloc(nlat);
  orc_box_dofs(b, p, plain, cons, NULL);
  for (int64_t c = 0; c < C; ++c)
    for (int l = 0; l < N3; ++l) {
      const uint32_t g = plain[c * N3 + l];
      if (cons[g]) continue;
      if (direction == 0) dst[c * N3 + l] += src[g];
      else dst[g] += src[c * N3 + l];
    }
  free(plain);
  free(cons);
}

/* DG diagonal, brute force: a(phi_l, phi_l) by applying the operator to unit vectors (tiny
 * meshes only; checks the closed form below). */
void orc_dg_diagonal_probe(const orc_box *b, int p, double c_pen, double *diag)
{
  const int64_t n = orc_box_ncells(b) * (p + 1) * (p + 1) * (p + 1);
  double *e = (double *)calloc(n, sizeof(double));
  double *y = (double *)malloc(sizeof(double) * n);
  for (int64_t i = 0; i < n; ++i) {
    e[i] = 1.0;
    orc_dg_vmult(b, p, c_pen, e, y);
    diag[i] = y[i];
    e[i] = 0.0;
  }
  free(e);
  free(y);
}

/* DG diagonal: the cell term by local probing, plus the face self terms in closed form.
 * A node (i along d, tangential (a,b)) on the face layer of face (d, side s) with
 * g = phi_i'(s) * (+-1)/h (normal derivative of its basis function) gets
 *   m (sigma - g) on inner faces and m (2 sigma - 2 g) on Dirichlet faces,
 * m = h_a h_b M1[a][a] M1[b][b] with M1 the exact 1D mass matrix on the GLL basis. */
void orc_dg_diagonal(const orc_box *b, int p, double c_pen, double *diag)
{
  const int N = p + 1, N3 = N * N * N;
  const int64_t C = orc_box_ncells(b);
  double h[3];
  box_cell_h(b, h);
  double S[64], SD[64], D[64], W[8];
  orc_shape_tables(p, N, S, SD, D, W);
  ld nodes[16], wl[16];
  gauss_lobatto_ld(N, nodes, wl);
  double M1[64], dphi0[8], dphi1[8];
  for (int i = 0; i < N; ++i) {
    for (int j = 0; j < N; ++j) {
      double s = 0;
      for (int q = 0; q < N; ++q) s += S[i * N + q] * S[j * N + q] * W[q];
      M1[i * N + j] = s;
    }
    dphi0[i] = (double)lagrange_deriv(N, nodes, i, 0.0L);
    dphi1[i] = (double)lagrange_deriv(N, nodes, i, 1.0L);
  }
  int64_t n[3];
  box_ncells(b, n);
  int32_t *cx = (int32_t *)malloc(sizeof(int32_t) * 3 * C);
  orc_box_cell_coords(b, cx, cx + C, cx + 2 * C);
  double *Gc = (double *)calloc(6 * N3, sizeof(double));
  const double vol = h[0] * h[1] * h[2];
  for (int q = 0; q < N3; ++q) {
    const int q0 = q % N, q1 = (q / N) % N, q2 = q / (N * N);
    const double w = W[q0] * W[q1] * W[q2] * vol;
    Gc[q] = w / (h[0] * h[0]);
    Gc[3 * N3 + q] = w / (h[1] * h[1]);
    Gc[5 * N3 + q] = w / (h[2] * h[2]);
  }
  double *buf = (double *)malloc(sizeof(double) * 7 * N3);
  for (int64_t c = 0; c < C; ++c) {
    for (int l = 0; l < N3; ++l) {
      for (int m = 0; m < N3; ++m) buf[m] = (m == l) ? 1.0 : 0.0;
      bk3_cell(N, S, D, Gc, buf, buf + N3, buf + 2 * N3, buf + 3 * N3, buf + 4 * N3, buf + 5 * N3,
               buf + 6 * N3);
      diag[c * N3 + l] = buf[N3 + l];
    }
    const int32_t cc[3] = {cx[c], cx[C + c], cx[2 * C + c]};
    for (int d = 0; d < 3; ++d) {
      const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
      for (int s = 0; s < 2; ++s) {
        const int outside = s ? (cc[d] == n[d] - 1) : (cc[d] == 0);
        const int dirichlet = (b->dirichlet_mask >> (2 * d + s)) & 1;
        if (outside && !dirichlet) continue;
        const double sigma = c_pen / h[d];
        const int il = s ? N - 1 : 0;
        const double g = (s ? dphi1[il] : dphi0[il]) * (s ? 1.0 : -1.0) / h[d];
        for (int bb = 0; bb < N; ++bb)
          for (int aa = 0; aa < N; ++aa) {
            int idx[3];
            idx[d] = il;
            idx[ta] = aa;
            idx[tb] = bb;
            const int l = (idx[2] * N + idx[1]) * N + idx[0];
            const double m = h[ta] * h[tb] * M1[aa * N + aa] * M1[bb * N + bb];
            diag[c * N3 + l] += outside ? m * (2.0 * sigma - 2.0 * g) : m * (sigma - g);
          }
      }
    }
  }
  free(buf); free(Gc); free(cx);
}

/* DG <-> CG patch transfer for the multigrid: P = identity, unit weights */
static void build_dg_transfer(orc_transfer *t, const orc_level *Lc, const orc_level *Lf)
{
  const int n = Lc->p + 1, n3 = n * n * n;
  t->nc = n;
  t->nf = n;
  t->n_patches = Lc->C;
  t->prolong_times = 1;
  t->coarse_idx = (uint32_t *)malloc(sizeof(uint32_t) * Lc->C * n3);
  t->fine_idx = (uint32_t *)malloc(sizeof(uint32_t) * Lc->C * n3);
  memcpy(t->coarse_idx, Lc->idx, sizeof(uint32_t) * Lc->C * n3);
  for (int64_t e = 0; e < Lc->C * n3; ++e) t->fine_idx[e] = (uint32_t)e;
  t->P1d = (double *)calloc(n * n, sizeof(double));
  for (int i = 0; i < n; ++i) t->P1d[i * n + i] = 1.0;
  t->weights = (double *)malloc(sizeof(double) * Lc->C * n3);
  for (int64_t e = 0; e < Lc->C * n3; ++e) t->weights[e] = 1.0;
}

/* The DG multigrid of the DG benchmark restated: FE_DGQ(p) on the box, ContinuousTransfer
 * to FE_Q(p), then the continuous hierarchy of orc_solve_box (p-levels pseq, Q1 h-levels);
 * PCG on the DG operator with rhs_kind 2 (exp(x) sin(pi y) cos(pi z), weak Dirichlet data). */
int orc_solve_dg(const orc_box *box, int p, const int32_t *pseq, int n_pseq, int cheb,
                 double c_pen, double reduce, int maxit, int nq_rhs, orc_solve_info *info,
                 double *x_out)
{
  memset(info, 0, sizeof(*info));
  const int n_h = box->refine + 1;
  const int n_cg = n_h + n_pseq - 1;
  const int n_levels = n_cg + 1;
  if (n_levels > 32 || pseq[n_pseq - 1] != 1 || pseq[0] != p) return -1;
  orc_mg mg;
  mg.n_levels = n_levels;
  mg.levels = (orc_level *)calloc(n_levels, sizeof(orc_level));
  mg.transfers = (orc_transfer *)calloc(n_levels, sizeof(orc_transfer));
  for (int l = 0; l < n_levels; ++l) {
    orc_level *L = &mg.levels[l];
    if (l < n_cg) {
      orc_box b = *box;
      int pl = 1;
      if (l < n_h) b.refine = l;
      else pl = pseq[n_pseq - 1 - (l - n_h + 1)];
      level_init(L, &b, pl, 0);
    } else {
      level_init_dg(L, box, p, c_pen);
    }
    if (l > 0) {
      L->cheb_degree = cheb;
      L->smoothing_range = 15.0;
      L->eig_iterations = 10;
    } else {
      L->cheb_degree = 0;
      L->smoothing_range = 1e-3;
      L->eig_iterations = (int)L->N;
    }
    cheb_estimate(L);
    info->level_degree[l] = L->p;
    info->level_cheb_degree[l] = L->cheb_degree;
    info->level_max_ev[l] = L->max_ev;
    info->level_min_ev[l] = L->min_ev;
    info->level_dofs[l] = L->N;
  }
  for (int l = 1; l < n_levels; ++l) {
    if (l < n_h) build_h_transfer(&mg.transfers[l], &mg.levels[l - 1], &mg.levels[l], 1);
    else if (l < n_cg) build_p_transfer(&mg.transfers[l], &mg.levels[l - 1], &mg.levels[l]);
    else build_dg_transfer(&mg.transfers[l], &mg.levels[l - 1], &mg.levels[l]);
  }
  orc_level *F = &mg.levels[n_levels - 1];
  const int64_t N = F->N;
  info->n_dofs = N;
  info->n_levels = n_levels;
  double *b = (double *)malloc(sizeof(double) * N);
  orc_dg_rhs(box, p, nq_rhs, c_pen, b);
  double *x = (double *)calloc(N, sizeof(double));
  double *r = (double *)malloc(sizeof(double) * N);
  double *z = (double *)malloc(sizeof(double) * N);
  double *pv = (double *)malloc(sizeof(double) * N);
  double *v = (double *)malloc(sizeof(double) * N);
  memcpy(r, b, sizeof(double) * N);
  double res = sqrt(dot(N, r, r));
  info->initial_residual = res;
  const double tol = reduce * res;
  int it = 0;
  double rho = 0, rho_old = 0;
  while (res > tol && it < maxit) {
    for (int l = 0; l < n_levels - 1; ++l)
      for (int64_t i = 0; i < mg.levels[l].N; ++i) mg.levels[l].def[i] = 0.0;
    memcpy(F->def, r, sizeof(double) * N);
    vcycle(&mg, n_levels - 1);
    memcpy(z, F->sol, sizeof(double) * N);
    rho_old = rho;
    rho = dot(N, r, z);
    if (it == 0) memcpy(pv, z, sizeof(double) * N);
    else {
      const double beta = rho / rho_old;
      for (int64_t i = 0; i < N; ++i) pv[i] = z[i] + beta * pv[i];
    }
    ++it;
    level_vmult(F, v, pv);
    const double alpha = rho / dot(N, pv, v);
    for (int64_t i = 0; i < N; ++i) { x[i] += alpha * pv[i]; r[i] -= alpha * v[i]; }
    res = sqrt(dot(N, r, r));
  }
  info->iterations = it;
  info->final_residual = res;
  info->reduction_per_step = it > 0 ? pow(res / info->initial_residual, 1.0 / it) : 1.0;
  info->l2_error = orc_dg_l2_error(box, p, p + 2, x);
  if (x_out) memcpy(x_out, x, sizeof(double) * N);
  free(b); free(x); free(r); free(z); free(pv); free(v);
  for (int l = 1; l < n_levels; ++l) transfer_free(&mg.transfers[l]);
  for (int l = 0; l < n_levels; ++l) level_free(&mg.levels[l]);
  free(mg.levels);
  free(mg.transfers);
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* 8. Mass matrix, per-quadrature-point forms and coefficient fields (adjoint path)       */
/* ------------------------------------------------------------------------------------ */
/* Not in the reference: the adjoint gradient of J(m) = 1/2 ||u(m) - u_d||^2_{L2} for
 * -div(exp(m) grad u) = f needs the FE mass matrix (values-only sum factorization), the
 * per-quadrature-point density of the Laplace form, and coefficient fields carried across
 * the multigrid levels.  Restated here from the definitions; the pins are the round trips
 * in tests/test_oracle_adjoint.py (mass matrix against exact integrals, the adjoint
 * gradient against central finite differences). */

/* dst = sum_c P_c^T S^T diag(jxw_c) S P_c src with identity rows on constrained DoFs;
 * jxw[C][nq^3] holds |det J| w_q (times any weight) at the (p+1)-point Gauss rule. */
void orc_mass_vmult(int p, int64_t C, int64_t N, const uint32_t *idx, const double *jxw,
                    const uint8_t *constrained, const double *src, double *dst)
{
  const int n = p + 1, n3 = n * n * n;
  double S[64];
  orc_shape_tables(p, n, S, NULL, NULL, NULL);
  double *buf = (double *)malloc(sizeof(double) * 5 * n3);
  double *u = buf, *v = buf + n3, *out = buf + 2 * n3, *t1 = buf + 3 * n3, *t2 = buf + 4 * n3;
  for (int64_t i = 0; i < N; ++i) dst[i] = 0.0;
  for (int64_t c = 0; c < C; ++c) {
    const uint32_t *ci = idx + c * n3;
    for (int l = 0; l < n3; ++l) u[l] = (ci[l] == ORC_INVALID) ? 0.0 : src[ci[l]];
    tensor_apply(n, n, S, 0, u, v, t1, t2);
    for (int q = 0; q < n3; ++q) v[q] *= jxw[c * n3 + q];
    tensor_apply(n, n, S, 1, v, out, t1, t2);
    for (int l = 0; l < n3; ++l)
      if (ci[l] != ORC_INVALID) dst[ci[l]] += out[l];
  }
  for (int64_t i = 0; i < N; ++i)
    if (constrained[i]) dst[i] = src[i];
  free(buf);
}

/* diag(M)_i = sum_c sum_q phi_i(x_q)^2 jxw_c(q); 1 on constrained rows. */
void orc_mass_diagonal(int p, int64_t C, int64_t N, const uint32_t *idx, const double *jxw,
                       const uint8_t *constrained, double *diag)
{
  const int n = p + 1, n3 = n * n * n;
  double S[64];
  orc_shape_tables(p, n, S, NULL, NULL, NULL);
  for (int64_t i = 0; i < N; ++i) diag[i] = 0.0;
  for (int64_t c = 0; c < C; ++c)
    for (int l = 0; l < n3; ++l) {
      const uint32_t d = idx[c * n3 + l];
      if (d == ORC_INVALID) continue;
      const int i = l % n, j = (l / n) % n, k = l / (n * n);
      double s = 0;
      for (int q2 = 0; q2 < n; ++q2)
        for (int q1 = 0; q1 < n; ++q1)
          for (int q0 = 0; q0 < n; ++q0) {
            const double phi = S[i * n + q0] * S[j * n + q1] * S[k * n + q2];
            s += phi * phi * jxw[c * n3 + (q2 * n + q1) * n + q0];
          }
      diag[d] += s;
    }
  for (int64_t i = 0; i < N; ++i)
    if (constrained[i]) diag[i] = 1.0;
}

/* out[c][q] = alpha * grad_ref(u)(x_q)^T G_c(q) grad_ref(v)(x_q), with G[C][6][nq^3] as
 * orc_box_G stores it (coefficient included): the integrand of a(u, v) = sum_c sum_q out.
 * Reference gradients are taken straight from the nodal values with the derivative table
 * SD (constrained entries of idx read as 0). */
void orc_qp_form(int p, int64_t C, const uint32_t *idx, const double *G, const double *u,
                 const double *v, double alpha, double *out)
{
  const int n = p + 1, n3 = n * n * n;
  double S[64], SD[64];
  orc_shape_tables(p, n, S, SD, NULL, NULL);
#pragma omp parallel
  {
    double *cu = (double *)malloc(sizeof(double) * 2 * n3);
    double *cv = cu + n3;
#pragma omp for schedule(static)
    for (int64_t c = 0; c < C; ++c) {
      const uint32_t *ci = idx + c * n3;
      for (int l = 0; l < n3; ++l) {
        cu[l] = (ci[l] == ORC_INVALID) ? 0.0 : u[ci[l]];
        cv[l] = (ci[l] == ORC_INVALID) ? 0.0 : v[ci[l]];
      }
      for (int q2 = 0; q2 < n; ++q2)
        for (int q1 = 0; q1 < n; ++q1)
          for (int q0 = 0; q0 < n; ++q0) {
            double gu[3] = {0, 0, 0}, gv[3] = {0, 0, 0};
            for (int k = 0; k < n; ++k)
              for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                  const double b0 = SD[i * n + q0] * S[j * n + q1] * S[k * n + q2];
                  const double b1 = S[i * n + q0] * SD[j * n + q1] * S[k * n + q2];
                  const double b2 = S[i * n + q0] * S[j * n + q1] * SD[k * n + q2];
                  const int l = (k * n + j) * n + i;
                  gu[0] += b0 * cu[l]; gu[1] += b1 * cu[l]; gu[2] += b2 * cu[l];
                  gv[0] += b0 * cv[l]; gv[1] += b1 * cv[l]; gv[2] += b2 * cv[l];
                }
            const int q = (q2 * n + q1) * n + q0;
            const double *g = G + c * 6 * n3;
            const double g00 = g[0 * n3 + q], g01 = g[1 * n3 + q], g02 = g[2 * n3 + q];
            const double g11 = g[3 * n3 + q], g12 = g[4 * n3 + q], g22 = g[5 * n3 + q];
            const double Gv0 = g00 * gv[0] + g01 * gv[1] + g02 * gv[2];
            const double Gv1 = g01 * gv[0] + g11 * gv[1] + g12 * gv[2];
            const double Gv2 = g02 * gv[0] + g12 * gv[1] + g22 * gv[2];
            out[c * n3 + q] = alpha * (gu[0] * Gv0 + gu[1] * Gv1 + gu[2] * Gv2);
          }
    }
    free(cu);
  }
}

/* A positive field given at the nq_src-point Gauss points of every cell of src_box, carried
 * to the nq_dst-point Gauss points of dst_box (the same box, equally or less refined): the
 * logarithm is interpolated by the tensor-product Lagrange polynomial through the source
 * cell's Gauss points at the target point, then exponentiated (so the result stays
 * positive).  A target point on a face of two source cells takes the upper cell. */
void orc_coef_interpolate(const orc_box *src_box, int nq_src, const double *src,
                          const orc_box *dst_box, int nq_dst, double *dst)
{
  int64_t ns[3], nd[3];
  box_ncells(src_box, ns);
  box_ncells(dst_box, nd);
  const int64_t Cs = ns[0] * ns[1] * ns[2], Cd = nd[0] * nd[1] * nd[2];
  int32_t *cs = (int32_t *)malloc(sizeof(int32_t) * 3 * Cs);
  int32_t *cd = (int32_t *)malloc(sizeof(int32_t) * 3 * Cd);
  orc_box_cell_coords(src_box, cs, cs + Cs, cs + 2 * Cs);
  orc_box_cell_coords(dst_box, cd, cd + Cd, cd + 2 * Cd);
  int64_t *lut = box_cell_lookup(src_box, cs);
  ld xs[32], ws[32], xd[32], wd[32];
  gauss_ld(nq_src, xs, ws);
  gauss_ld(nq_dst, xd, wd);
  const int64_t r = ns[0] / nd[0];
  const int nqs3 = nq_src * nq_src * nq_src, nqd3 = nq_dst * nq_dst * nq_dst;
  for (int64_t c = 0; c < Cd; ++c)
    for (int q = 0; q < nqd3; ++q) {
      const int qd[3] = {q % nq_dst, (q / nq_dst) % nq_dst, q / (nq_dst * nq_dst)};
      int64_t sc[3];
      double L[3][32];
      for (int d = 0; d < 3; ++d) {
        const double X = ((double)cd[d * Cd + c] + (double)xd[qd[d]]) * (double)r;
        int64_t s = (int64_t)floor(X);
        if (s > ns[d] - 1) s = ns[d] - 1;
        sc[d] = s;
        const ld xi = (ld)(X - (double)s);
        for (int a = 0; a < nq_src; ++a) L[d][a] = (double)lagrange(nq_src, xs, a, xi);
      }
      const int64_t cell = lut[(sc[2] * ns[1] + sc[1]) * ns[0] + sc[0]];
      double s = 0;
      for (int k = 0; k < nq_src; ++k)
        for (int j = 0; j < nq_src; ++j)
          for (int i = 0; i < nq_src; ++i)
            s += L[0][i] * L[1][j] * L[2][k] * log(src[cell * nqs3 + (k * nq_src + j) * nq_src + i]);
      dst[c * nqd3 + q] = exp(s);
    }
  free(cs); free(cd); free(lut);
}
