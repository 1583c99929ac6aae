// Level operator: setup of the index map and geometry on the device, vmult, diagonal,
// right-hand side assembly (LaplaceOperatorBK3, include/operators/portable_laplace_operator_bk3.h).
#include <algorithm>
#include <cmath>

#include "laplace_kernels.cuh"
#include "dg.hpp"
#include "fields.hpp"
#include "vector_ops.hpp"
#include "numbering.hpp"
#include "vmult_tc.hpp"
#include "pmg_internal.hpp"

namespace pmg {
namespace {

constexpr int kMaxNm = 8;   // nodes per direction (degree <= 6, +1 for nq = p+2 rules)
constexpr int kMaxNq = 8;

// Everything the per-cell geometry kernels need, passed by value (constant bank).
struct GeoParams {
  double lo[3], h[3];
  int deform;
  double amp;
  int nm, nq;
  int N, cpw, lanes; // slab layout of the owning operator (nm == nq == N for G output)
  double xl[kMaxNm];
  double S[kMaxNm * kMaxNq], SD[kMaxNm * kMaxNq], W[kMaxNq];
};

__device__ __forceinline__ void map_point(const GeoParams &g, const double xr[3], double xp[3]) {
  xp[0] = xr[0];
  xp[1] = xr[1];
  xp[2] = xr[2];
  if (g.deform == 1) {
    const double s = g.amp * sin(M_PI * xr[0]) * sin(M_PI * xr[1]) * sin(M_PI * xr[2]);
    xp[0] += s;
    xp[1] += s;
    xp[2] += s;
  }
}

__device__ __forceinline__ double coefficient(int kind, const double x[3]) {
  if (kind == PMG_COEFF_KAPPA)
    return 1.0 + 0.9 * sin(2 * M_PI * x[0]) * sin(2 * M_PI * x[1]) * sin(2 * M_PI * x[2]);
  return 1.0;
}

// One block per cell (grid-stride): mapping nodes in shared memory, then per quadrature
// point the Jacobian of the isoparametric Q_p map, its inverse and determinant.
// mode 0: write G = coef * |det J| w_q J^{-1} J^{-T} into the slab layout (full geometry);
// mode 1: write coef * (per-point factor) into the affine coefficient layout;
// mode 2: right-hand side, b_i += sum_q phi_i(x_q) f(x_q) |det J| w_q (atomic);
// mode 3: the quadrature points, out[cell][q][3];
// mode 4: coef * |det J| w_q into the affine coefficient layout (mass-matrix weights);
// mode 5: out[cell] = (sum_q (u_h(x_q) - u(x_q))^2 |det J| w_q)^(1/2) for the exact solution
//         u of f_kind 1 (sin(pi x) sin(pi y) sin(pi z)) or 2 (exp(x) sin(pi y) cos(pi z));
// mode 6: write J^{-1} (9 entries, row d = d xi_d / dx) and coef * |det J| w_q into the slab
//         layout of the inverse-Jacobian formulation, [group][x point][y point][10][lane];
// mode 7: out[dof][3] = the mapped position of every node (DoFs shared by cells receive the
//         same value from each of them).
template <typename T>
__global__ void cell_geometry_kernel(const GeoParams g, const int32_t *__restrict__ cell_xyz,
                                     int64_t n_cells, int mode, int coeff_kind,
                                     const double *__restrict__ coef_values,
                                     T *__restrict__ out, const uint32_t *__restrict__ idx_perm,
                                     int f_kind, const void *__restrict__ uvec = nullptr,
                                     const uint32_t *__restrict__ plain = nullptr, int u_f32 = 0) {
  __shared__ double X[3][kMaxNm * kMaxNm * kMaxNm];
  __shared__ double U[kMaxNm * kMaxNm * kMaxNm]; // mode 5: the cell's nodal values
  __shared__ double fq[kMaxNq * kMaxNq * kMaxNq];
  const int nm = g.nm, nq = g.nq, nm3 = nm * nm * nm, nq3 = nq * nq * nq;
  for (int64_t c = blockIdx.x; c < n_cells; c += gridDim.x) {
    const int cx = cell_xyz[3 * c], cy = cell_xyz[3 * c + 1], cz = cell_xyz[3 * c + 2];
    for (int l = threadIdx.x; l < nm3; l += blockDim.x) {
      const int i = l % nm, j = (l / nm) % nm, k = l / (nm * nm);
      const double xr[3] = {g.lo[0] + (cx + g.xl[i]) * g.h[0], g.lo[1] + (cy + g.xl[j]) * g.h[1],
                            g.lo[2] + (cz + g.xl[k]) * g.h[2]};
      double xp[3];
      map_point(g, xr, xp);
      if (mode == 7) {
        const uint32_t d = plain[c * nm3 + l];
        out[3 * int64_t(d)] = (T)xp[0];
        out[3 * int64_t(d) + 1] = (T)xp[1];
        out[3 * int64_t(d) + 2] = (T)xp[2];
        continue;
      }
      X[0][l] = xp[0];
      X[1][l] = xp[1];
      X[2][l] = xp[2];
      if (mode == 5) {
        const uint32_t d = plain[c * nm3 + l];
        U[l] = u_f32 ? (double)static_cast<const float *>(uvec)[d] : static_cast<const double *>(uvec)[d];
      }
    }
    if (mode == 7) continue; // uniform over the block: no shared memory was written
    __syncthreads();
    for (int q = threadIdx.x; q < nq3; q += blockDim.x) {
      const int q0 = q % nq, q1 = (q / nq) % nq, q2 = q / (nq * nq);
      double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, xq[3] = {0, 0, 0}, uh = 0.0;
      for (int k = 0; k < nm; ++k)
        for (int j = 0; j < nm; ++j) {
          const double sj = g.S[j * nq + q1], dj = g.SD[j * nq + q1];
          const double sk = g.S[k * nq + q2], dk = g.SD[k * nq + q2];
          for (int i = 0; i < nm; ++i) {
            const int l = (k * nm + j) * nm + i;
            const double si = g.S[i * nq + q0], di = g.SD[i * nq + q0];
            const double v = si * sj * sk, g0 = di * sj * sk, g1 = si * dj * sk, g2 = si * sj * dk;
            if (mode == 5) uh += U[l] * v;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const double xv = X[d][l];
              xq[d] += xv * v;
              J[3 * d + 0] += xv * g0;
              J[3 * d + 1] += xv * g1;
              J[3 * d + 2] += xv * g2;
            }
          }
        }
      const double A = J[4] * J[8] - J[5] * J[7], B = -(J[3] * J[8] - J[5] * J[6]),
                   C = J[3] * J[7] - J[4] * J[6];
      const double det = J[0] * A + J[1] * B + J[2] * C;
      const double r = 1.0 / det;
      const double inv[9] = {A * r,
                             -(J[1] * J[8] - J[2] * J[7]) * r,
                             (J[1] * J[5] - J[2] * J[4]) * r,
                             B * r,
                             (J[0] * J[8] - J[2] * J[6]) * r,
                             -(J[0] * J[5] - J[2] * J[3]) * r,
                             C * r,
                             -(J[0] * J[7] - J[1] * J[6]) * r,
                             (J[0] * J[4] - J[1] * J[3]) * r};
      const double wq = g.W[q0] * g.W[q1] * g.W[q2];
      double kap = coefficient(coeff_kind, xq);
      if (coef_values) kap *= coef_values[c * nq3 + q];
      const int64_t grp = c / g.cpw;
      const int e = (int)(c % g.cpw);
      // full geometry is column-major per group (x point outer) so that each x column of a
      // group is one contiguous chunk; the per-point coefficient stays row-major
      const int m = q0 * g.N + q1, m_row = q1 * g.N + q0, lane = e * g.N + q2;
      if (mode == 0) {
        const double f = fabs(det) * wq * kap;
        int comp = 0;
        for (int d1 = 0; d1 < 3; ++d1)
          for (int d2 = d1; d2 < 3; ++d2) {
            const double s = inv[3 * d1] * inv[3 * d2] + inv[3 * d1 + 1] * inv[3 * d2 + 1] +
                             inv[3 * d1 + 2] * inv[3 * d2 + 2];
            out[((grp * (g.N * g.N) + m) * 6 + comp) * g.lanes + lane] = (T)(f * s);
            ++comp;
          }
      } else if (mode == 6) {
        for (int comp = 0; comp < 9; ++comp)
          out[((grp * (g.N * g.N) + m) * 10 + comp) * g.lanes + lane] = (T)inv[comp];
        out[((grp * (g.N * g.N) + m) * 10 + 9) * g.lanes + lane] = (T)(fabs(det) * wq * kap);
      } else if (mode == 1) {
        out[(grp * (g.N * g.N) + m_row) * g.lanes + lane] = (T)kap;
      } else if (mode == 3) {
        for (int d = 0; d < 3; ++d) out[(c * nq3 + q) * 3 + d] = (T)xq[d];
      } else if (mode == 4) {
        out[(grp * (g.N * g.N) + m_row) * g.lanes + lane] = (T)(fabs(det) * wq * kap);
      } else if (mode == 5) {
        double ex = 0.0;
        if (f_kind == 1) ex = sin(M_PI * xq[0]) * sin(M_PI * xq[1]) * sin(M_PI * xq[2]);
        if (f_kind == 2) ex = exp(xq[0]) * sin(M_PI * xq[1]) * cos(M_PI * xq[2]);
        fq[q] = (uh - ex) * (uh - ex) * fabs(det) * wq;
      } else {
        double f = 1.0;
        if (f_kind == 1) f = 3.0 * M_PI * M_PI * sin(M_PI * xq[0]) * sin(M_PI * xq[1]) * sin(M_PI * xq[2]);
        if (f_kind == 2) f = (2.0 * M_PI * M_PI - 1.0) * exp(xq[0]) * sin(M_PI * xq[1]) * cos(M_PI * xq[2]);
        fq[q] = f * fabs(det) * wq;
      }
    }
    __syncthreads();
    if (mode == 5 && threadIdx.x == 0) { // fixed summation order: deterministic
      double e = 0.0;
      for (int q = 0; q < nq3; ++q) e += fq[q];
      out[c] = (T)sqrt(e);
    }
    if (mode == 2) {
      for (int l = threadIdx.x; l < nm3; l += blockDim.x) {
        const int i = l % nm, j = (l / nm) % nm, k = l / (nm * nm);
        double s = 0;
        for (int q2 = 0; q2 < nq; ++q2)
          for (int q1 = 0; q1 < nq; ++q1) {
            const double sjk = g.S[j * nq + q1] * g.S[k * nq + q2];
            for (int q0 = 0; q0 < nq; ++q0)
              s += g.S[i * nq + q0] * sjk * fq[(q2 * nq + q1) * nq + q0];
          }
        const int64_t grp = c / g.cpw;
        const int e = (int)(c % g.cpw);
        // Y-slab layout of the index map: [group][k*N + i][lane = e*N + j]
        const uint32_t id = idx_perm[(grp * (g.N * g.N) + k * g.N + i) * g.lanes + e * g.N + j];
        if (id != kInvalid) atomicAdd(out + id, (T)s);
      }
      __syncthreads();
    }
  }
}

template <typename T>
__global__ void invert_diagonal_kernel(T *__restrict__ d, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (d[i] != T(0)) ? T(1) / d[i] : T(1);
}

// dst_i = src_i on constrained DoFs (bit i of `bits`), 0 elsewhere
template <typename T>
__global__ void init_dst_kernel(T *__restrict__ dst, const T *__restrict__ src, const uint32_t *__restrict__ bits,
                                int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = __ldg(bits + (i >> 5));
    dst[i] = ((w >> (i & 31)) & 1u) ? src[i] : T(0);
  }
}

template <typename T>
__global__ void set_constrained_kernel(T *__restrict__ dst, const T *__restrict__ src,
                                       const uint32_t *__restrict__ list, int64_t n, T value) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[list[i]] = src ? src[list[i]] : value;
}

GeoParams make_geo_params(const pmg_operator &op, int nq) {
  GeoParams g{};
  const auto &b = op.mesh.box;
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = b.lo[d];
    g.h[d] = (b.hi[d] - b.lo[d]) / double(op.mesh.n[d]);
  }
  g.deform = b.deform;
  g.amp = b.amp;
  g.nm = op.nm;
  g.nq = nq;
  g.N = op.nm;
  g.cpw = op.cpw;
  g.lanes = op.lanes;
  const Tables1D t = make_tables(op.degree, nq);
  for (int i = 0; i < op.nm; ++i) g.xl[i] = t.xl[i];
  for (size_t a = 0; a < t.S.size(); ++a) {
    g.S[a] = t.S[a];
    g.SD[a] = t.SD[a];
  }
  for (int q = 0; q < nq; ++q) g.W[q] = t.W[q];
  return g;
}

int num_sms(int device) {
  int n = 0;
  PMG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
  return n;
}

typedef void (*slab_fn)(const SlabLaunch &);
slab_fn vmult_fn(int degree) {
  static const slab_fn f[] = {nullptr,         launch_vmult_p1, launch_vmult_p2, launch_vmult_p3,
                              launch_vmult_p4, launch_vmult_p5, launch_vmult_p6};
  return f[degree];
}
slab_fn diag_fn(int degree) {
  static const slab_fn f[] = {nullptr,        launch_diag_p1, launch_diag_p2, launch_diag_p3,
                              launch_diag_p4, launch_diag_p5, launch_diag_p6};
  return f[degree];
}
int occupancy(bool diag, int degree, int dtype, int geom) {
  typedef int (*occ_fn)(int, int);
  static const occ_fn fv[] = {nullptr,           occupancy_vmult_p1, occupancy_vmult_p2,
                              occupancy_vmult_p3, occupancy_vmult_p4, occupancy_vmult_p5,
                              occupancy_vmult_p6};
  static const occ_fn fd[] = {nullptr,          occupancy_diag_p1, occupancy_diag_p2,
                              occupancy_diag_p3, occupancy_diag_p4, occupancy_diag_p5,
                              occupancy_diag_p6};
  return (diag ? fd : fv)[degree](dtype, geom);
}

int geom_code(const pmg_operator &op) {
  if (op.geometry == PMG_GEOMETRY_FULL) return 0;
  if (op.geometry == PMG_GEOMETRY_INVJAC) return 3;
  return op.has_coeff_values ? 2 : 1;
}

SlabLaunch slab_launch(const pmg_operator &op, const Tables1D &t, cudaStream_t s) {
  SlabLaunch L{};
  L.idx = op.idx.as<uint32_t>();
  L.geo = op.geo.get();
  L.coef = op.coef.get();
  L.n_groups = op.n_groups;
  L.geom = geom_code(op);
  L.dtype = op.dtype;
  L.stream = s;
  L.S = t.S.data();
  L.SD = t.SD.data();
  L.D = t.D.data();
  L.W = t.W.data();
  return L;
}

// The index map with the sentinel, permuted into the Y-slab layout [group][k*N+i][e*N+j]
// (setup_dof_indices_per_color, bk3.h:360-437) from the device numbering: entries that are
// constrained DoFs, or the sentinel already, become the sentinel.
void build_slab_index(pmg_operator &op) {
  device_slab_index(op.dplain.as<uint32_t>(), op.dcons.as<uint8_t>(), op.n_cells, op.nm, op.cpw, op.lanes,
                    op.n_groups, op.sms, op.idx, nullptr);
}

// the constrained DoFs as a list and a bitmask (copy_constrained_values, bk3.h:230)
void build_constrained(pmg_operator &op) {
  device_constrained(op.dcons.as<uint8_t>(), op.n_dofs, op.sms, op.constrained_list, op.constrained_bits,
                     op.n_constrained, nullptr);
}

// persistent grids (as many warps as can be resident on this device) and the error flag
void finish_setup(pmg_operator &op) {
  PMG_CUDA(cudaDeviceSynchronize());
  const int sms = num_sms(op.device);
  const int gc = geom_code(op);
  const int occ = occupancy(false, op.degree, op.dtype, gc);
  op.warps_vmult = (int64_t)std::max(1, occ & 0xffff) * sms;
  op.warps_vmult_ring = (int64_t)std::max(1, occ >> 16) * sms;
  op.warps_diag = (int64_t)std::max(1, occupancy(true, op.degree, op.dtype, gc)) * sms;
  op.err_flag.allocate(sizeof(unsigned int));
  PMG_CUDA(cudaMemset(op.err_flag.get(), 0, sizeof(unsigned int)));
}

// Caller geometry (cell order of the caller, points lexicographic x fastest) into the slab
// layout [group][x point p][y point q][ncomp][lane = e*N + z point r]:
//   mode 0: in = G[C][6][nq^3] (rr, rs, rt, ss, st, tt);
//   mode 1: in = inv_jacobian[C][nq^3][3][3] (components 0..8), in2 = JxW[C][nq^3] (component 9).
// One thread per input value: reads are coalesced, writes land in lane-contiguous runs.
template <typename T>
__global__ void geometry_from_caller_kernel(const double *__restrict__ in, const double *__restrict__ in2,
                                            int mode, int64_t n_cells, int N, int cpw, int lanes,
                                            T *__restrict__ out) {
  const int N2 = N * N, N3 = N2 * N, ncomp = mode == 0 ? 6 : 10, nin = mode == 0 ? 6 : 9;
  const int64_t total = n_cells * N3 * (mode == 0 ? 6 : 10);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c;
    int comp, pt;
    double v;
    if (mode == 0) {
      c = t / (6 * N3);
      const int64_t r = t - c * 6 * N3;
      comp = (int)(r / N3);
      pt = (int)(r - (int64_t)comp * N3);
      v = in[t];
    } else if (t < n_cells * N3 * nin) {
      c = t / (N3 * nin);
      const int64_t r = t - c * N3 * nin;
      pt = (int)(r / nin);
      comp = (int)(r - (int64_t)pt * nin);
      v = in[t];
    } else {
      const int64_t u = t - n_cells * N3 * nin;
      c = u / N3;
      pt = (int)(u - c * N3);
      comp = 9;
      v = in2[u];
    }
    const int p = pt % N, q = (pt / N) % N, r = pt / N2;
    const int64_t grp = c / cpw;
    const int e = (int)(c - grp * cpw);
    out[((grp * N2 + p * N + q) * ncomp + comp) * lanes + e * N + r] = (T)v;
  }
}

} // namespace

void operator_setup_from_maps(pmg_operator &op, const pmg_operator_maps &m, const pmg_operator_params &prm) {
  PMG_REQUIRE(prm.degree >= 1 && prm.degree <= kMaxDegree, "degree must be in [1,6]");
  PMG_REQUIRE(prm.dtype == PMG_F64 || prm.dtype == PMG_F32, "dtype must be PMG_F64 or PMG_F32");
  PMG_REQUIRE(prm.kind == PMG_OP_LAPLACE, "operators from caller maps are continuous Laplace operators");
  PMG_REQUIRE(prm.coeff_kind == PMG_COEFF_NONE,
              "a coefficient of a caller-described operator is folded into its G or JxW");
  PMG_REQUIRE(m.n_cells >= 0 && m.n_dofs >= 0, "negative size");
  PMG_REQUIRE(m.n_dofs < (int64_t(1) << 32) - 1, "too many DoFs for 32-bit indices");
  PMG_REQUIRE(m.n_cells < (int64_t(1) << 31), "too many cells");
  PMG_REQUIRE(m.n_cells == 0 || m.dof_indices, "dof_indices is NULL");
  PMG_REQUIRE(m.n_constrained >= 0 && (m.n_constrained == 0 || m.constrained), "bad constrained list");
  PMG_REQUIRE(m.geometry == PMG_MAPS_G || m.geometry == PMG_MAPS_INVJAC, "geometry must be PMG_MAPS_G or PMG_MAPS_INVJAC");
  if (m.n_cells > 0) {
    if (m.geometry == PMG_MAPS_G) PMG_REQUIRE(m.G, "G is NULL");
    else PMG_REQUIRE(m.inv_jacobian && m.JxW, "inv_jacobian or JxW is NULL");
  }
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    (void)cudaGetLastError();
    fail(PMG_ENODEV, "no CUDA device available");
  }
  PMG_REQUIRE(prm.device >= 0 && prm.device < n_dev, "bad device ordinal");
  PMG_CUDA(cudaSetDevice(prm.device));
  op.device = prm.device;
  op.from_maps = true;
  op.kind = PMG_OP_LAPLACE;
  op.degree = prm.degree;
  op.nm = op.nq = prm.degree + 1;
  op.dtype = prm.dtype;
  op.coeff_kind = PMG_COEFF_NONE;
  op.geometry = m.geometry == PMG_MAPS_G ? PMG_GEOMETRY_FULL : PMG_GEOMETRY_INVJAC;
  op.has_coeff_values = false;
  op.n_cells = m.n_cells;
  op.n_dofs = m.n_dofs;
  op.mesh = BoxMesh{};
  op.mesh.n_cells = m.n_cells;
  const int N = op.nm, N2 = N * N, N3 = N2 * N;
  op.cpw = 32 / N;
  op.lanes = op.cpw * N;
  op.n_groups = (op.n_cells + op.cpw - 1) / op.cpw;
  op.sms = num_sms(op.device);
  // the caller's numbering: index map (sentinel = constrained) and identity rows
  op.num = Numbering{};
  op.num.p = op.degree;
  op.num.n_dofs = m.n_dofs;
  op.num.plain.assign(m.dof_indices, m.dof_indices + (size_t)m.n_cells * N3);
  op.num.constrained.assign((size_t)m.n_dofs, 0);
  for (int64_t i = 0; i < m.n_constrained; ++i) {
    const uint32_t d = m.constrained[i];
    if ((int64_t)d >= m.n_dofs)
      fail(PMG_EBOUNDS, "constrained DoF " + std::to_string(d) + " >= n_dofs " + std::to_string(m.n_dofs));
    op.num.constrained[d] = 1;
  }
  for (size_t e = 0; e < op.num.plain.size(); ++e) {
    uint32_t &d = op.num.plain[e];
    if (d == kInvalid) continue;
    if ((int64_t)d >= m.n_dofs)
      fail(PMG_EBOUNDS, "dof_indices[" + std::to_string(e) + "] = " + std::to_string(d) + " >= n_dofs " +
                            std::to_string(m.n_dofs));
    if (op.num.constrained[d]) d = kInvalid;
  }
  op.host_num_valid = true;
  op.dplain = upload(op.num.plain);
  op.dcons = upload(op.num.constrained);
  build_slab_index(op);
  build_constrained(op);
  // geometry: the caller's arrays, permuted into the slab layout on the device
  const size_t s = dtype_size(op.dtype);
  const bool ij = m.geometry == PMG_MAPS_INVJAC;
  const int ncomp = ij ? 10 : 6;
  op.geo.allocate(s * std::max<int64_t>(1, op.n_groups) * N2 * ncomp * op.lanes);
  PMG_CUDA(cudaMemset(op.geo.get(), 0, op.geo.bytes()));
  if (op.n_cells > 0) {
    const int64_t n_in = op.n_cells * N3 * (ij ? 9 : 6);
    DeviceBuffer in(sizeof(double) * n_in), in2;
    PMG_CUDA(cudaMemcpy(in.get(), ij ? m.inv_jacobian : m.G, sizeof(double) * n_in, cudaMemcpyHostToDevice));
    if (ij) {
      in2.allocate(sizeof(double) * op.n_cells * N3);
      PMG_CUDA(cudaMemcpy(in2.get(), m.JxW, sizeof(double) * op.n_cells * N3, cudaMemcpyHostToDevice));
    }
    const int grid = (int)std::min<int64_t>((op.n_cells * N3 * ncomp + 255) / 256, (int64_t)op.sms * 32);
    if (op.dtype == PMG_F64)
      geometry_from_caller_kernel<double><<<grid, 256>>>(in.as<double>(), in2.as<double>(), ij ? 1 : 0, op.n_cells,
                                                         N, op.cpw, op.lanes, op.geo.as<double>());
    else
      geometry_from_caller_kernel<float><<<grid, 256>>>(in.as<double>(), in2.as<double>(), ij ? 1 : 0, op.n_cells,
                                                        N, op.cpw, op.lanes, op.geo.as<float>());
    PMG_LAUNCH_CHECK();
    PMG_CUDA(cudaDeviceSynchronize()); // the input buffers are freed on return
  }
  finish_setup(op);
}

void operator_setup(pmg_operator &op, const pmg_mesh &mesh, const pmg_operator_params &prm) {
  PMG_REQUIRE(prm.degree >= 1 && prm.degree <= kMaxDegree, "degree must be in [1,6]");
  PMG_REQUIRE(prm.dtype == PMG_F64 || prm.dtype == PMG_F32, "dtype must be PMG_F64 or PMG_F32");
  PMG_REQUIRE(prm.coeff_kind >= 0 && prm.coeff_kind <= 2, "bad coeff_kind");
  PMG_REQUIRE(prm.kind == PMG_OP_LAPLACE || prm.kind == PMG_OP_DG_SIPG || prm.kind == PMG_OP_MASS,
              "bad operator kind");
  if (prm.kind == PMG_OP_DG_SIPG) {
    PMG_REQUIRE(mesh.m.box.deform == 0, "the DG operator needs an undeformed (axis-aligned) box");
    PMG_REQUIRE(prm.coeff_kind == PMG_COEFF_NONE, "the DG operator has no coefficient");
  }
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    (void)cudaGetLastError();
    fail(PMG_ENODEV, "no CUDA device available");
  }
  PMG_REQUIRE(prm.device >= 0 && prm.device < n_dev, "bad device ordinal");
  PMG_CUDA(cudaSetDevice(prm.device));
  op.device = prm.device;
  op.degree = prm.degree;
  op.nm = op.nq = prm.degree + 1;
  op.dtype = prm.dtype;
  op.coeff_kind = prm.coeff_kind;
  op.mesh = mesh.m;
  op.n_cells = mesh.m.n_cells;
  op.kind = prm.kind;
  int geometry = prm.geometry;
  if (geometry == PMG_GEOMETRY_AUTO || op.kind == PMG_OP_DG_SIPG)
    geometry = mesh.m.box.deform ? PMG_GEOMETRY_FULL : PMG_GEOMETRY_AFFINE;
  PMG_REQUIRE(geometry == PMG_GEOMETRY_FULL || geometry == PMG_GEOMETRY_AFFINE || geometry == PMG_GEOMETRY_INVJAC,
              "bad geometry");
  PMG_REQUIRE(!(geometry == PMG_GEOMETRY_AFFINE && mesh.m.box.deform), "affine geometry needs an undeformed box");
  op.geometry = geometry;
  op.has_coeff_values = (geometry == PMG_GEOMETRY_AFFINE && prm.coeff_kind != PMG_COEFF_NONE);

  const int N = op.nm, N2 = N * N, N3 = N2 * N;
  op.cpw = 32 / N;
  op.lanes = op.cpw * N;
  op.n_groups = (op.n_cells + op.cpw - 1) / op.cpw;

  // numbering (setup_dof_indices_per_color, bk3.h:360-437): first-visit order on the device
  // for continuous operators; cell by cell for DG
  op.sms = num_sms(op.device);
  op.cell_xyz = upload(mesh.m.cell_xyz);
  if (op.kind == PMG_OP_DG_SIPG) {
    op.num = make_numbering_dg(mesh.m, op.degree);
    op.host_num_valid = true;
    op.dplain = upload(op.num.plain);
    op.dcons = upload(op.num.constrained);
  } else {
    DeviceNumbering dn;
    device_numbering(mesh.m, op.degree, op.cell_xyz, op.sms, dn, nullptr);
    op.num = Numbering{};
    op.num.p = op.degree;
    op.num.n_dofs = dn.n_dofs;
    for (int d = 0; d < 3; ++d) op.num.L[d] = dn.L[d];
    op.dplain = std::move(dn.plain);
    op.dcons = std::move(dn.constrained);
    op.dlattice = std::move(dn.lattice);
    op.host_num_valid = false;
  }
  op.n_dofs = op.num.n_dofs;
  if (op.kind == PMG_OP_DG_SIPG) {
    op.dg = std::make_shared<DGHost>();
    dg_setup(*op.dg, mesh.m, op.degree, prm.penalty);
  }

  build_slab_index(op);
  build_constrained(op);
  // geometry (compute_G_tensors, bk3.h:456-515), computed on the device
  const size_t s = dtype_size(op.dtype);
  const DeviceBuffer &xyz = op.cell_xyz;
  // coefficient values (PMG_COEFF_VALUES): kept on the device in FP64 so that coarser levels
  // can interpolate them; no array given means the constant 1
  if (prm.coeff_kind == PMG_COEFF_VALUES) {
    op.coef_qp.allocate(sizeof(double) * std::max<int64_t>(1, op.n_cells * N3));
    if (prm.coeff_qp) {
      PMG_CUDA(cudaMemcpy(op.coef_qp.get(), prm.coeff_qp, sizeof(double) * op.n_cells * N3,
                          cudaMemcpyHostToDevice));
    } else {
      std::vector<double> ones((size_t)op.n_cells * N3, 1.0);
      if (!ones.empty())
        PMG_CUDA(cudaMemcpy(op.coef_qp.get(), ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  const double *coef_in = op.coef_qp.as<double>();
  const GeoParams gp = make_geo_params(op, op.nq);
  const int sms = num_sms(op.device);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(op.n_cells, (int64_t)sms * 16));
  if (op.kind == PMG_OP_MASS) {
    // mass matrix: the volume of an affine cell without a coefficient, else |det J| w_q
    // (times the coefficient) per quadrature point
    op.mass_geom = (geometry == PMG_GEOMETRY_AFFINE && prm.coeff_kind == PMG_COEFF_NONE) ? 1 : 0;
    op.has_coeff_values = false;
    if (op.mass_geom == 1) {
      double h[3];
      for (int d = 0; d < 3; ++d) h[d] = (mesh.m.box.hi[d] - mesh.m.box.lo[d]) / double(mesh.m.n[d]);
      const int64_t n_slots = op.n_groups * op.cpw;
      std::vector<double> v(n_slots * 8, 0.0);
      for (int64_t c = 0; c < op.n_cells; ++c) v[8 * c + 6] = h[0] * h[1] * h[2];
      if (op.dtype == PMG_F64) {
        op.geo = upload(v);
      } else {
        std::vector<float> f(v.begin(), v.end());
        op.geo = upload(f);
      }
    } else {
      op.coef.allocate(s * op.n_groups * N2 * op.lanes);
      PMG_CUDA(cudaMemset(op.coef.get(), 0, op.coef.bytes()));
      if (op.dtype == PMG_F64)
        cell_geometry_kernel<double><<<grid, 128>>>(gp, xyz.as<int32_t>(), op.n_cells, 4, prm.coeff_kind,
                                                    coef_in, op.coef.as<double>(), nullptr, 0);
      else
        cell_geometry_kernel<float><<<grid, 128>>>(gp, xyz.as<int32_t>(), op.n_cells, 4, prm.coeff_kind,
                                                   coef_in, op.coef.as<float>(), nullptr, 0);
      PMG_LAUNCH_CHECK();
    }
  } else if (geometry == PMG_GEOMETRY_FULL || geometry == PMG_GEOMETRY_INVJAC) {
    const bool ij = geometry == PMG_GEOMETRY_INVJAC;
    op.geo.allocate(s * op.n_groups * N2 * (ij ? 10 : 6) * op.lanes);
    PMG_CUDA(cudaMemset(op.geo.get(), 0, op.geo.bytes()));
    if (op.dtype == PMG_F64)
      cell_geometry_kernel<double><<<grid, 128>>>(gp, xyz.as<int32_t>(), op.n_cells, ij ? 6 : 0, prm.coeff_kind,
                                                  coef_in, op.geo.as<double>(), nullptr, 0);
    else
      cell_geometry_kernel<float><<<grid, 128>>>(gp, xyz.as<int32_t>(), op.n_cells, ij ? 6 : 0, prm.coeff_kind,
                                                 coef_in, op.geo.as<float>(), nullptr, 0);
    PMG_LAUNCH_CHECK();
  } else {
    // affine: C = |det J| J^{-1} J^{-T} / (w-independent) per cell; axis-aligned boxes give
    // J = diag(h) for every cell
    std::vector<double> c8(8, 0.0);
    double h[3];
    for (int d = 0; d < 3; ++d) h[d] = (mesh.m.box.hi[d] - mesh.m.box.lo[d]) / double(mesh.m.n[d]);
    const double vol = h[0] * h[1] * h[2];
    c8[0] = vol / (h[0] * h[0]);
    c8[3] = vol / (h[1] * h[1]);
    c8[5] = vol / (h[2] * h[2]);
    c8[6] = vol;
    const int64_t n_slots = op.n_groups * op.cpw;
    if (op.dtype == PMG_F64) {
      std::vector<double> v(n_slots * 8, 0.0);
      for (int64_t c = 0; c < op.n_cells; ++c) std::copy(c8.begin(), c8.end(), v.begin() + 8 * c);
      op.geo = upload(v);
    } else {
      std::vector<float> v(n_slots * 8, 0.0f);
      for (int64_t c = 0; c < op.n_cells; ++c)
        for (int a = 0; a < 8; ++a) v[8 * c + a] = (float)c8[a];
      op.geo = upload(v);
    }
    if (op.has_coeff_values) {
      op.coef.allocate(s * op.n_groups * N2 * op.lanes);
      PMG_CUDA(cudaMemset(op.coef.get(), 0, op.coef.bytes()));
      if (op.dtype == PMG_F64)
        cell_geometry_kernel<double><<<grid, 128>>>(gp, xyz.as<int32_t>(), op.n_cells, 1, prm.coeff_kind,
                                                    coef_in, op.coef.as<double>(), nullptr, 0);
      else
        cell_geometry_kernel<float><<<grid, 128>>>(gp, xyz.as<int32_t>(), op.n_cells, 1, prm.coeff_kind,
                                                   coef_in, op.coef.as<float>(), nullptr, 0);
      PMG_LAUNCH_CHECK();
    }
  }
  // the index lattice is only needed for building h-transfers: keep it
  finish_setup(op);
}

namespace {
// dst = 0 (bk3.h:134) with the identity rows of copy_constrained_values (bk3.h:230) written
// in the same pass: the cell kernels never touch constrained entries (index sentinel)
void vmult_init(const pmg_operator &op, void *dst, const void *src, cudaStream_t s) {
  const size_t bytes = dtype_size(op.dtype) * op.n_dofs;
  if (op.n_constrained > 0) {
    prof::Scope scope("vmult_init", s);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((op.n_dofs + 255) / 256, (int64_t)op.sms * 16));
    if (op.dtype == PMG_F64)
      init_dst_kernel<double><<<grid, 256, 0, s>>>(static_cast<double *>(dst), static_cast<const double *>(src),
                                                   op.constrained_bits.as<uint32_t>(), op.n_dofs);
    else
      init_dst_kernel<float><<<grid, 256, 0, s>>>(static_cast<float *>(dst), static_cast<const float *>(src),
                                                  op.constrained_bits.as<uint32_t>(), op.n_dofs);
    PMG_LAUNCH_CHECK();
  } else {
    PMG_CUDA(cudaMemsetAsync(dst, 0, bytes, s));
  }
}
} // namespace

// The Chebyshev step out = cur + f1 (cur - prev) + f2 invd (b - A cur) in one launch where the
// operator is a DG operator on 4x4x4 tiles (the fused tile kernel writes each entry of A cur
// once, so it applies the step there instead of storing A cur); false, with nothing launched,
// elsewhere.  out may be prev, not cur.
bool operator_vmult_chebyshev(const pmg_operator &op, void *out, const void *cur, const void *prev, const void *b,
                              const void *invd, double f1, double f2, cudaStream_t s) {
  if (!op.dg || op.n_cells == 0 || op.n_constrained > 0 || op.tensor_cores || out == cur) return false;
  if (!dg_fused_applies(*op.dg, op.degree, op.dtype, op.n_cells, op.sms)) return false;
  const DGChebStep c{prev, b, invd, f1, f2};
  prof::Scope scope("vmult_dg_tile", s);
  const bool ran = dg_apply_fused(*op.dg, op.degree, op.dtype, cur, out, op.n_cells, op.sms, s,
                                  &op.launch_units[PMG_KERNEL_DG_FACES], &op.launch_par[PMG_KERNEL_DG_FACES], &c);
  op.launch_units[PMG_KERNEL_VMULT_CELL] = op.launch_units[PMG_KERNEL_DG_FACES];
  op.launch_par[PMG_KERNEL_VMULT_CELL] = op.launch_par[PMG_KERNEL_DG_FACES];
  return ran;
}

void operator_vmult(const pmg_operator &op, void *dst, const void *src, cudaStream_t s, bool compute) {
  PMG_REQUIRE(dst && src, "null vector");
  PMG_REQUIRE(dst != src, "vmult needs distinct src and dst");
  if (compute && op.dg && op.n_cells > 0 && op.n_constrained == 0 && !op.tensor_cores) {
    // DG on 4x4x4 tiles: cell and face terms in one kernel that writes dst once; both launch
    // records describe it
    prof::Scope scope("vmult_dg_tile", s);
    if (dg_apply_fused(*op.dg, op.degree, op.dtype, src, dst, op.n_cells, op.sms, s,
                       &op.launch_units[PMG_KERNEL_DG_FACES], &op.launch_par[PMG_KERNEL_DG_FACES])) {
      op.launch_units[PMG_KERNEL_VMULT_CELL] = op.launch_units[PMG_KERNEL_DG_FACES];
      op.launch_par[PMG_KERNEL_VMULT_CELL] = op.launch_par[PMG_KERNEL_DG_FACES];
      return;
    }
  }
  vmult_init(op, dst, src, s);
  if (compute && op.n_cells > 0 && op.kind == PMG_OP_MASS) {
    prof::Scope scope("vmult_mass", s);
    mass_vmult_cells(op, src, dst, s);
  } else if (compute && op.n_cells > 0) {
    SlabLaunch L = slab_launch(op, cached_tables(op.degree), s);
    L.src = src;
    L.dst = dst;
    L.resident_warps = op.warps_vmult;
    L.resident_warps_ring = op.warps_vmult_ring;
    L.err = op.err_flag.as<unsigned int>();
    L.launched = &op.launch_par[PMG_KERNEL_VMULT_CELL];
    op.launch_units[PMG_KERNEL_VMULT_CELL] = op.n_groups;
    {
      prof::Scope scope("vmult_cell", s);
      if (op.tensor_cores) vmult_cells_tensor_cores(op, src, dst, s);
      else vmult_fn(op.degree)(L);
    }
    if (op.dg) {
      prof::Scope scope("vmult_dg_faces", s);
      dg_apply_faces(*op.dg, op.degree, op.dtype, src, dst, op.n_cells, op.sms, s,
                     &op.launch_units[PMG_KERNEL_DG_FACES], &op.launch_par[PMG_KERNEL_DG_FACES]);
    }
  }
}

// The cells [cell_begin, cell_end) of the operator's cell order added into dst (after
// vmult_init when init is set): the cell kernel on the warp groups that hold them, with the
// index map, geometry and coefficient pointers advanced to the first of those groups.
void operator_vmult_cells(const pmg_operator &op, void *dst, const void *src, int64_t cell_begin,
                          int64_t cell_end, bool init, cudaStream_t s) {
  PMG_REQUIRE(dst && src, "null vector");
  PMG_REQUIRE(dst != src, "vmult needs distinct src and dst");
  PMG_REQUIRE(op.kind == PMG_OP_LAPLACE && !op.dg, "cell ranges are applied by continuous Laplace operators");
  PMG_REQUIRE(op.tensor_cores == 0, "cell ranges are applied by the CUDA-core cell kernel");
  PMG_REQUIRE(0 <= cell_begin && cell_begin <= cell_end && cell_end <= op.n_cells, "cell range out of bounds");
  PMG_REQUIRE(cell_begin % op.cpw == 0 && (cell_end % op.cpw == 0 || cell_end == op.n_cells),
              "cell range bounds must be multiples of the cells per warp group (or the cell count)");
  if (init) vmult_init(op, dst, src, s);
  const int64_t g0 = cell_begin / op.cpw, g1 = (cell_end + op.cpw - 1) / op.cpw;
  if (g1 <= g0) return;
  const int N2 = op.nm * op.nm;
  const size_t sz = dtype_size(op.dtype);
  SlabLaunch L = slab_launch(op, cached_tables(op.degree), s);
  const int gc = geom_code(op);
  L.idx = op.idx.as<uint32_t>() + g0 * N2 * op.lanes;
  if (gc == 0 || gc == 3)
    L.geo = static_cast<const char *>(op.geo.get()) + sz * g0 * N2 * (gc == 3 ? 10 : 6) * op.lanes;
  else
    L.geo = static_cast<const char *>(op.geo.get()) + sz * g0 * op.cpw * 8;
  if (op.coef.get()) L.coef = static_cast<const char *>(op.coef.get()) + sz * g0 * N2 * op.lanes;
  L.n_groups = g1 - g0;
  L.src = src;
  L.dst = dst;
  L.resident_warps = op.warps_vmult;
  L.resident_warps_ring = op.warps_vmult_ring;
  L.err = op.err_flag.as<unsigned int>();
  L.launched = &op.launch_par[PMG_KERNEL_VMULT_CELL];
  op.launch_units[PMG_KERNEL_VMULT_CELL] = L.n_groups;
  prof::Scope scope("vmult_cell", s);
  vmult_fn(op.degree)(L);
}

void operator_compute_inverse_diagonal(pmg_operator &op, cudaStream_t s) {
  PMG_CUDA(cudaSetDevice(op.device));
  const size_t bytes = dtype_size(op.dtype) * op.n_dofs;
  if (op.inv_diag.bytes() != bytes) op.inv_diag.allocate(bytes);
  PMG_CUDA(cudaMemsetAsync(op.inv_diag.get(), 0, bytes, s));
  if (op.n_cells > 0 && op.kind == PMG_OP_MASS) {
    prof::Scope scope("diag_mass", s);
    mass_diagonal_cells(op, op.inv_diag.get(), s);
  } else if (op.n_cells > 0) {
    SlabLaunch L = slab_launch(op, cached_tables(op.degree), s);
    L.dst = op.inv_diag.get();
    L.resident_warps = op.warps_diag;
    L.err = op.err_flag.as<unsigned int>();
    prof::Scope scope("diag_cell", s);
    diag_fn(op.degree)(L);
  }
  if (op.dg) dg_add_face_diagonal(*op.dg, op.degree, op.dtype, op.inv_diag.get(), op.n_cells, op.sms, s);
  const int grid = (int)std::min<int64_t>(4096, (op.n_dofs + 255) / 256);
  if (op.dtype == PMG_F64) {
    invert_diagonal_kernel<double><<<grid, 256, 0, s>>>(op.inv_diag.as<double>(), op.n_dofs);
    if (op.n_constrained)
      set_constrained_kernel<double><<<64, 256, 0, s>>>(op.inv_diag.as<double>(), nullptr,
                                                        op.constrained_list.as<uint32_t>(), op.n_constrained, 1.0);
  } else {
    invert_diagonal_kernel<float><<<grid, 256, 0, s>>>(op.inv_diag.as<float>(), op.n_dofs);
    if (op.n_constrained)
      set_constrained_kernel<float><<<64, 256, 0, s>>>(op.inv_diag.as<float>(), nullptr,
                                                       op.constrained_list.as<uint32_t>(), op.n_constrained, 1.0f);
  }
  PMG_LAUNCH_CHECK();
  op.has_diag = true;
}

void operator_assemble_rhs(const pmg_operator &op, int f_kind, int nq, void *b, cudaStream_t s) {
  require_mesh(op, "the right-hand side");
  PMG_REQUIRE(f_kind >= 0 && f_kind <= 2, "f_kind must be 0, 1 or 2");
  if (nq <= 0) nq = op.nq;
  PMG_REQUIRE(nq >= 1 && nq <= kMaxNq, "nq must be in [1,8]");
  PMG_CUDA(cudaSetDevice(op.device));
  PMG_CUDA(cudaMemsetAsync(b, 0, dtype_size(op.dtype) * op.n_dofs, s));
  const DeviceBuffer &xyz = op.cell_xyz;
  const GeoParams gp = make_geo_params(op, nq);
  const int grid = (int)std::min<int64_t>(std::max<int64_t>(op.n_cells, 1), (int64_t)num_sms(op.device) * 16);
  if (op.dtype == PMG_F64)
    cell_geometry_kernel<double><<<grid, 128, 0, s>>>(gp, xyz.as<int32_t>(), op.n_cells, 2, 0, nullptr,
                                                      static_cast<double *>(b), op.idx.as<uint32_t>(), f_kind);
  else
    cell_geometry_kernel<float><<<grid, 128, 0, s>>>(gp, xyz.as<int32_t>(), op.n_cells, 2, 0, nullptr,
                                                     static_cast<float *>(b), op.idx.as<uint32_t>(), f_kind);
  PMG_LAUNCH_CHECK();
  if (op.dg && f_kind == 2) dg_add_boundary_rhs(*op.dg, op.mesh, op.degree, nq, op.dtype, b, s);
}

void operator_copy_geometry(const pmg_operator &op, double *host) {
  PMG_REQUIRE(op.geometry == PMG_GEOMETRY_FULL, "geometry copy needs the full geometry layout");
  const int N = op.nm, N2 = N * N, N3 = N2 * N;
  const size_t n = (size_t)op.n_groups * N2 * 6 * op.lanes;
  std::vector<double> g(n);
  if (op.dtype == PMG_F64) {
    PMG_CUDA(cudaMemcpy(g.data(), op.geo.get(), n * 8, cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> f(n);
    PMG_CUDA(cudaMemcpy(f.data(), op.geo.get(), n * 4, cudaMemcpyDeviceToHost));
    std::copy(f.begin(), f.end(), g.begin());
  }
  for (int64_t c = 0; c < op.n_cells; ++c) {
    const int64_t grp = c / op.cpw, e = c % op.cpw;
    for (int r = 0; r < N; ++r)
      for (int q = 0; q < N; ++q)
        for (int p = 0; p < N; ++p)
          for (int comp = 0; comp < 6; ++comp)
            host[(c * 6 + comp) * N3 + (r * N + q) * N + p] =
                g[((grp * N2 + p * N + q) * 6 + comp) * op.lanes + e * N + r];
  }
}

int64_t operator_bytes(const pmg_operator &op) {
  const int64_t s = (int64_t)dtype_size(op.dtype);
  const int64_t nm3 = (int64_t)op.nm * op.nm * op.nm, nq3 = (int64_t)op.nq * op.nq * op.nq;
  int64_t g = 0;
  if (op.kind == PMG_OP_MASS) g = op.mass_geom == 1 ? 1 : nq3;
  else if (op.geometry == PMG_GEOMETRY_FULL) g = 6 * nq3;
  else if (op.geometry == PMG_GEOMETRY_INVJAC) g = 10 * nq3;
  else g = 6 + (op.has_coeff_values ? nq3 : 0);
  return 2 * s * op.n_dofs + 4 * nm3 * op.n_cells + g * s * op.n_cells;
}

// Replace the coefficient values (PMG_COEFF_VALUES) and rebuild what depends on them: G
// (full geometry), the per-point factors (affine), or the mass weights.  The inverse
// diagonal is not recomputed here.
void operator_set_coefficient(pmg_operator &op, const double *values, bool on_device, cudaStream_t s) {
  require_mesh(op, "a coefficient update");
  PMG_REQUIRE(op.coeff_kind == PMG_COEFF_VALUES, "the operator was not created with PMG_COEFF_VALUES");
  PMG_REQUIRE(values, "null coefficient array");
  PMG_CUDA(cudaSetDevice(op.device));
  const int64_t n = op.n_cells * op.nq * op.nq * op.nq;
  if (values != op.coef_qp.as<double>())
    PMG_CUDA(cudaMemcpyAsync(op.coef_qp.get(), values, sizeof(double) * n,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  if (op.n_cells == 0) return;
  const GeoParams gp = make_geo_params(op, op.nq);
  const int grid = (int)std::min<int64_t>(op.n_cells, (int64_t)op.sms * 16);
  int mode = 0;
  void *out = nullptr;
  if (op.kind == PMG_OP_MASS) {
    mode = 4;
    out = op.coef.get();
  } else if (op.geometry == PMG_GEOMETRY_FULL || op.geometry == PMG_GEOMETRY_INVJAC) {
    mode = op.geometry == PMG_GEOMETRY_INVJAC ? 6 : 0;
    out = op.geo.get();
  } else {
    mode = 1;
    out = op.coef.get();
  }
  if (op.dtype == PMG_F64)
    cell_geometry_kernel<double><<<grid, 128, 0, s>>>(gp, op.cell_xyz.as<int32_t>(), op.n_cells, mode, op.coeff_kind,
                                                      op.coef_qp.as<double>(), static_cast<double *>(out), nullptr, 0);
  else
    cell_geometry_kernel<float><<<grid, 128, 0, s>>>(gp, op.cell_xyz.as<int32_t>(), op.n_cells, mode, op.coeff_kind,
                                                     op.coef_qp.as<double>(), static_cast<float *>(out), nullptr, 0);
  PMG_LAUNCH_CHECK();
}

// dst's coefficient := src's coefficient field at dst's quadrature points (nested boxes).
void operator_interpolate_coefficient(pmg_operator &dst, pmg_operator &src, cudaStream_t s) {
  require_mesh(dst, "coefficient interpolation");
  require_mesh(src, "coefficient interpolation");
  PMG_REQUIRE(dst.coeff_kind == PMG_COEFF_VALUES && src.coeff_kind == PMG_COEFF_VALUES,
              "both operators need PMG_COEFF_VALUES");
  PMG_REQUIRE(dst.device == src.device, "operators on different devices");
  PMG_CUDA(cudaSetDevice(dst.device));
  if (!src.cell_lut.get()) {
    std::vector<int32_t> lut((size_t)src.n_cells);
    for (int64_t c = 0; c < src.n_cells; ++c) {
      const int32_t *x = &src.mesh.cell_xyz[3 * c];
      lut[((int64_t)x[2] * src.mesh.n[1] + x[1]) * src.mesh.n[0] + x[0]] = (int32_t)c;
    }
    src.cell_lut = upload(lut);
  }
  if (dst.n_cells == 0) return;
  coefficient_interpolate(src, dst, dst.coef_qp.as<double>(), s);
  operator_set_coefficient(dst, dst.coef_qp.as<double>(), true, s);
}

void operator_quadrature_points(const pmg_operator &op, double *xq, cudaStream_t s) {
  require_mesh(op, "the quadrature points");
  PMG_REQUIRE(xq, "null output");
  PMG_CUDA(cudaSetDevice(op.device));
  if (op.n_cells == 0) return;
  const GeoParams gp = make_geo_params(op, op.nq);
  const int grid = (int)std::min<int64_t>(op.n_cells, (int64_t)op.sms * 16);
  cell_geometry_kernel<double><<<grid, 128, 0, s>>>(gp, op.cell_xyz.as<int32_t>(), op.n_cells, 3, 0, nullptr, xq,
                                                    nullptr, 0);
  PMG_LAUNCH_CHECK();
}

void operator_qp_form(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                      cudaStream_t s) {
  PMG_REQUIRE(op.kind == PMG_OP_LAPLACE, "the per-point form is defined for the continuous Laplace operator");
  PMG_REQUIRE(u && v && out, "null vector");
  PMG_CUDA(cudaSetDevice(op.device));
  if (op.n_cells == 0) return;
  prof::Scope scope("qp_form", s);
  qp_form_cells(op, u, v, alpha, out, s);
}

// ||u_h - u||_{L2} with an nq-point Gauss rule per direction; every DoF's value counts,
// Dirichlet ones included (the plain index map is uploaded for the call).
// xyz[dof][3] (device, FP64) = the mapped support point of every DoF, for boundary data
// (the points at which deal.II's VectorTools::interpolate_boundary_values evaluates the
// Dirichlet function, source/plain_solver/program.cc:125-131)
void operator_dof_coordinates(const pmg_operator &op, double *xyz, cudaStream_t s) {
  require_mesh(op, "the DoF coordinates");
  PMG_REQUIRE(xyz, "null output");
  PMG_CUDA(cudaSetDevice(op.device));
  if (op.n_cells == 0) return;
  const GeoParams gp = make_geo_params(op, op.nq);
  const int grid = (int)std::min<int64_t>(op.n_cells, (int64_t)op.sms * 16);
  cell_geometry_kernel<double><<<grid, 128, 0, s>>>(gp, op.cell_xyz.as<int32_t>(), op.n_cells, 7, 0, nullptr, xyz,
                                                    nullptr, 0, nullptr, op.dplain.as<uint32_t>(), 0);
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaStreamSynchronize(s));
}

const Numbering &host_numbering(const pmg_operator &op) {
  if (!op.host_num_valid) {
    PMG_CUDA(cudaSetDevice(op.device));
    const int64_t nm3 = (int64_t)op.nm * op.nm * op.nm;
    op.num.plain.resize((size_t)op.n_cells * nm3);
    op.num.constrained.resize((size_t)op.n_dofs);
    if (!op.num.plain.empty())
      PMG_CUDA(cudaMemcpy(op.num.plain.data(), op.dplain.get(), op.num.plain.size() * 4, cudaMemcpyDeviceToHost));
    if (!op.num.constrained.empty())
      PMG_CUDA(cudaMemcpy(op.num.constrained.data(), op.dcons.get(), op.num.constrained.size(),
                          cudaMemcpyDeviceToHost));
    if (op.dlattice.get()) {
      op.num.lattice.resize(op.dlattice.bytes() / 4);
      PMG_CUDA(cudaMemcpy(op.num.lattice.data(), op.dlattice.get(), op.dlattice.bytes(), cudaMemcpyDeviceToHost));
    }
    op.host_num_valid = true;
  }
  return op.num;
}

double operator_l2_error(const pmg_operator &op, const void *u, int exact_kind, int nq, cudaStream_t s) {
  require_mesh(op, "the error norm");
  PMG_REQUIRE(u, "null vector");
  PMG_REQUIRE(exact_kind == 1 || exact_kind == 2, "exact_kind must be 1 (sine) or 2 (exp-sine-cosine)");
  if (nq <= 0) nq = op.nq + 1;
  PMG_REQUIRE(nq >= 1 && nq <= kMaxNq, "nq must be in [1,8]");
  PMG_CUDA(cudaSetDevice(op.device));
  if (op.n_cells == 0) return 0.0;
  DeviceBuffer cell_err(sizeof(double) * op.n_cells);
  const GeoParams gp = make_geo_params(op, nq);
  const int grid = (int)std::min<int64_t>(op.n_cells, (int64_t)op.sms * 16);
  cell_geometry_kernel<double><<<grid, 128, 0, s>>>(gp, op.cell_xyz.as<int32_t>(), op.n_cells, 5, 0, nullptr,
                                                    cell_err.as<double>(), nullptr, exact_kind, u,
                                                    op.dplain.as<uint32_t>(), op.dtype == PMG_F32 ? 1 : 0);
  PMG_LAUNCH_CHECK();
  const double e2 = vec::dot(cell_err.get(), cell_err.get(), PMG_F64, op.n_cells, s); // synchronises
  return std::sqrt(e2);
}

} // namespace pmg
