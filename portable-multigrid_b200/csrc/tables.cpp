// 1D quadrature rules and the tensor-product tables the kernels contract with.
//
// FE_Q(p) is the Lagrange basis on the p+1 Gauss-Lobatto points of [0,1]; the operator
// integrates with the (p+1)-point Gauss rule (QGauss<1>(fe_degree+1),
// include/operators/portable_laplace_operator_bk3.h:120).  The tables follow the layouts
// the reference's kernels read: shape_values[i*nq+q] and co_shape_gradients[n*nq+q]
// (include/kernels/bk3_kokkos_kernel.h:69, :339-461).  All values are computed in long
// double and rounded once.
#include <cmath>

#include "pmg_internal.hpp"

namespace pmg {
namespace {

using ld = long double;
constexpr ld kPi = 3.141592653589793238462643383279502884L;

// Legendre P_n(x) and P_n'(x) by the three-term recursion.
void legendre(int n, ld x, ld &P, ld &dP) {
  ld a = 1.0L, b = x;
  if (n == 0) {
    P = 1.0L;
    dP = 0.0L;
    return;
  }
  for (int k = 2; k <= n; ++k) {
    const ld c = ((2 * k - 1) * x * b - (k - 1) * a) / k;
    a = b;
    b = c;
  }
  P = b;
  dP = n * (x * b - a) / (x * x - 1.0L);
}

void gauss(int n, std::vector<ld> &x, std::vector<ld> &w) {
  x.assign(n, 0);
  w.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    ld t = std::cos(kPi * (i + 0.75L) / (n + 0.5L)), P, dP;
    for (int it = 0; it < 100; ++it) {
      legendre(n, t, P, dP);
      const ld dt = P / dP;
      t -= dt;
      if (std::fabs(dt) < 1e-19L) break;
    }
    legendre(n, t, P, dP);
    x[i] = 0.5L * (1.0L - t);
    w[i] = 1.0L / ((1.0L - t * t) * dP * dP);
  }
}

void gauss_lobatto(int n, std::vector<ld> &x) {
  x.assign(n, 0);
  const int m = n - 1;
  x[0] = 0.0L;
  x[n - 1] = 1.0L;
  for (int i = 1; i < n - 1; ++i) {
    ld t = std::cos(kPi * i / m), P, dP;
    for (int it = 0; it < 100; ++it) {
      legendre(m, t, P, dP);
      const ld d2P = (2.0L * t * dP - m * (m + 1.0L) * P) / (1.0L - t * t);
      const ld dt = dP / d2P;
      t -= dt;
      if (std::fabs(dt) < 1e-19L) break;
    }
    x[i] = 0.5L * (1.0L - t);
  }
}

ld lagrange(const std::vector<ld> &nodes, int i, ld x) {
  ld v = 1.0L;
  for (size_t j = 0; j < nodes.size(); ++j)
    if ((int)j != i) v *= (x - nodes[j]) / (nodes[i] - nodes[j]);
  return v;
}

ld lagrange_derivative(const std::vector<ld> &nodes, int i, ld x) {
  ld s = 0.0L;
  for (size_t m = 0; m < nodes.size(); ++m) {
    if ((int)m == i) continue;
    ld v = 1.0L / (nodes[i] - nodes[m]);
    for (size_t j = 0; j < nodes.size(); ++j)
      if ((int)j != i && j != m) v *= (x - nodes[j]) / (nodes[i] - nodes[j]);
    s += v;
  }
  return s;
}

} // namespace

Tables1D make_tables(int p, int nq) {
  Tables1D t;
  t.p = p;
  t.nq = nq;
  const int nm = p + 1;
  std::vector<ld> xg, wg, xl;
  gauss(nq, xg, wg);
  gauss_lobatto(nm, xl);
  t.S.resize(nm * nq);
  t.SD.resize(nm * nq);
  t.D.resize(nq * nq);
  t.W.resize(nq);
  t.xg.resize(nq);
  t.xl.resize(nm);
  for (int i = 0; i < nm; ++i)
    for (int q = 0; q < nq; ++q) {
      t.S[i * nq + q] = (double)lagrange(xl, i, xg[q]);
      t.SD[i * nq + q] = (double)lagrange_derivative(xl, i, xg[q]);
    }
  for (int n = 0; n < nq; ++n)
    for (int q = 0; q < nq; ++q) t.D[n * nq + q] = (double)lagrange_derivative(xg, n, xg[q]);
  for (int q = 0; q < nq; ++q) {
    t.W[q] = (double)wg[q];
    t.xg[q] = (double)xg[q];
  }
  for (int i = 0; i < nm; ++i) t.xl[i] = (double)xl[i];
  return t;
}

std::vector<double> lagrange_derivative_at(int p, double x) {
  std::vector<ld> xl;
  gauss_lobatto(p + 1, xl);
  std::vector<double> d(p + 1);
  for (int i = 0; i <= p; ++i) d[i] = (double)lagrange_derivative(xl, i, (ld)x);
  return d;
}

std::vector<double> gauss_lobatto_points(int n) {
  std::vector<ld> x;
  gauss_lobatto(n, x);
  return std::vector<double>(x.begin(), x.end());
}

// Interpolation of FE_Q(pc) at the FE_Q(pf) nodes: FETools::get_projection_matrix between
// nested Lagrange spaces, stored [i_c][j_f]
// (include/multigrid/portable_polynomial_transfer.h:1093-1108).
std::vector<double> p_transfer_matrix(int pc, int pf) {
  std::vector<ld> xc, xf;
  gauss_lobatto(pc + 1, xc);
  gauss_lobatto(pf + 1, xf);
  std::vector<double> P((pc + 1) * (pf + 1));
  for (int i = 0; i <= pc; ++i)
    for (int j = 0; j <= pf; ++j) P[i * (pf + 1) + j] = (double)lagrange(xc, i, xf[j]);
  return P;
}

// FE_Q(p) coarse basis at the nodes of both children of an isotropic refinement, fine
// nodes numbered 0..2p along the coarse cell (FE_Q<1>::get_prolongation_matrix(c) as
// assembled at include/multigrid/portable_geometric_transfer.h:1294-1330), [i_c][j_f].
std::vector<double> h_transfer_matrix(int p) {
  std::vector<ld> x;
  gauss_lobatto(p + 1, x);
  const int nf = 2 * p + 1;
  std::vector<double> P((p + 1) * nf);
  for (int i = 0; i <= p; ++i)
    for (int j = 0; j < nf; ++j) {
      const ld y = (j <= p) ? 0.5L * x[j] : 0.5L + 0.5L * x[j - p];
      P[i * nf + j] = (double)lagrange(x, i, y);
    }
  return P;
}

} // namespace pmg
