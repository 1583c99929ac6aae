// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pmg/pmg.h"

namespace pmg {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kMaxDegree = 6; // OperatorDispatchFactory::max_degree

// ---------------------------------------------------------------------------------------
// errors: every failure throws pmg::Error; the C ABI turns it into a status + message
// ---------------------------------------------------------------------------------------
struct Error : std::runtime_error {
  pmg_status status;
  Error(pmg_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(pmg_status s, const std::string &m) { throw Error(s, m); }

inline void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError(); // clear a sticky-free error so later calls can proceed
    fail(e == cudaErrorMemoryAllocation ? PMG_ENOMEM : PMG_ECUDA,
         std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
             std::to_string(line) + ")");
  }
}
#define PMG_CUDA(call) ::pmg::cuda_check((call), #call, __FILE__, __LINE__)
#define PMG_LAUNCH_CHECK() ::pmg::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

#define PMG_REQUIRE(cond, msg)                                                              \
  do {                                                                                      \
    if (!(cond)) ::pmg::fail(PMG_EINVAL, std::string(msg));                                 \
  } while (0)

// ---------------------------------------------------------------------------------------
// kernel timing (profile.cu): an event pair per instrumented launch while enabled
// ---------------------------------------------------------------------------------------
namespace prof {
bool enabled();
void set_enabled(bool on);
void reset();
void query(const char *name, double *ms, int64_t *launches);
struct Scope {
  Scope(const char *name, cudaStream_t s);
  ~Scope();
  Scope(const Scope &) = delete;
  Scope &operator=(const Scope &) = delete;
  const char *name;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
};
} // namespace prof

// ---------------------------------------------------------------------------------------
// device memory owned by library objects
// ---------------------------------------------------------------------------------------
class DeviceBuffer {
public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { allocate(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
    o.ptr_ = nullptr;
    o.bytes_ = 0;
  }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
      release();
      ptr_ = o.ptr_;
      bytes_ = o.bytes_;
      o.ptr_ = nullptr;
      o.bytes_ = 0;
    }
    return *this;
  }
  void allocate(size_t bytes) {
    release();
    if (bytes == 0) return;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      fail(PMG_ENOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                           cudaGetErrorString(e));
    }
    ptr_ = p;
    bytes_ = bytes;
  }
  void release() {
    if (ptr_) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  template <typename T> T *as() const { return static_cast<T *>(ptr_); }
  void *get() const { return ptr_; }
  size_t bytes() const { return bytes_; }

private:
  void *ptr_ = nullptr;
  size_t bytes_ = 0;
};

template <typename T> DeviceBuffer upload(const std::vector<T> &h) {
  DeviceBuffer b(h.size() * sizeof(T));
  if (!h.empty()) PMG_CUDA(cudaMemcpy(b.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return b;
}

inline size_t dtype_size(int dtype) { return dtype == PMG_F64 ? 8 : 4; }

// ---------------------------------------------------------------------------------------
// 1D tables (tables.cpp)
// ---------------------------------------------------------------------------------------
struct Tables1D {
  int p = 0, nq = 0;
  std::vector<double> S;  // [nm][nq]  GLL Lagrange basis at Gauss points
  std::vector<double> SD; // [nm][nq]  its derivative
  std::vector<double> D;  // [nq][nq]  collocation derivative on the Gauss points
  std::vector<double> W;  // [nq]      Gauss weights on [0,1]
  std::vector<double> xg, xl;
};
Tables1D make_tables(int p, int nq);
std::vector<double> gauss_lobatto_points(int n);
std::vector<double> lagrange_derivative_at(int p, double x); // FE_Q(p) basis derivatives at x
std::vector<double> p_transfer_matrix(int pc, int pf);  // [nc][nf]
std::vector<double> h_transfer_matrix(int p);           // [p+1][2p+1]

// ---------------------------------------------------------------------------------------
// meshes and numbering (mesh.cpp)
// ---------------------------------------------------------------------------------------
struct BoxMesh {
  pmg_box box{};
  int64_t n[3] = {0, 0, 0};
  int64_t n_cells = 0;
  std::vector<int32_t> cell_xyz; // [C][3]
};

struct Numbering {
  int p = 0;
  int64_t n_dofs = 0;
  std::vector<uint32_t> plain;      // [C][nm^3] lexicographic, no sentinel
  std::vector<uint8_t> constrained; // [N]
  std::vector<uint32_t> lattice;    // node lattice (x fastest) -> dof
  int64_t L[3] = {0, 0, 0};         // lattice extents p*n+1
};

BoxMesh make_box(const pmg_box &b);
Numbering make_numbering_dg(const BoxMesh &m, int p); // dof = cell * (p+1)^3 + l

} // namespace pmg

// ---------------------------------------------------------------------------------------
// opaque handle types of the C ABI
// ---------------------------------------------------------------------------------------
struct pmg_mesh {
  pmg::BoxMesh m;
};

namespace pmg {
struct DGHost;
}

struct pmg_operator {
  int device = 0;
  bool from_maps = false;           // built from a caller's index map and geometry (no mesh)
  int tensor_cores = 0;             // cell kernel: 0 CUDA cores, 1 TF32 mma, 3 three TF32 products
  int kind = PMG_OP_LAPLACE;        // PMG_OP_LAPLACE, PMG_OP_DG_SIPG or PMG_OP_MASS
  std::shared_ptr<pmg::DGHost> dg;  // face data of a DG operator
  int degree = 1, nm = 2, nq = 2;
  int dtype = PMG_F64;
  int geometry = PMG_GEOMETRY_FULL; // resolved: FULL or AFFINE
  int coeff_kind = PMG_COEFF_NONE;
  bool has_coeff_values = false;    // affine: per-qp factors stored
  pmg::BoxMesh mesh;
  int64_t n_cells = 0, n_dofs = 0;
  int cpw = 1, lanes = 1;           // cells per warp group, active lanes per group
  int64_t n_groups = 0;
  // numbering on the device: plain [C][nm^3] (no sentinel; caller maps: the sentinel kept),
  // constrained flags [N], node lattice -> DoF (continuous box operators)
  pmg::DeviceBuffer dplain, dcons, dlattice;
  // host copy of the numbering, filled on first use (pmg::host_numbering); L and n_dofs always set
  mutable pmg::Numbering num;
  mutable bool host_num_valid = false;
  pmg::DeviceBuffer idx;            // permuted [group][nm^2][lanes] uint32
  pmg::DeviceBuffer geo;            // FULL: [group][nq^2][6][lanes]; AFFINE: [C][8]
  pmg::DeviceBuffer coef;           // AFFINE with coefficient: [group][nq^2][lanes];
                                    // MASS with mass_geom 0: |det J| w_q (times coefficient)
  int mass_geom = 0;                // MASS: 1 = affine volume in geo[cell][6], 0 = coef
  pmg::DeviceBuffer coef_qp;        // PMG_COEFF_VALUES: the values [C][nq^3] FP64
  pmg::DeviceBuffer cell_xyz;       // [C][3] int32 lattice coordinates of the cells
  pmg::DeviceBuffer cell_lut;       // lattice (x fastest) -> cell, int32 (built on demand)
  pmg::DeviceBuffer constrained_list; // uint32 [n_constrained]
  pmg::DeviceBuffer constrained_bits; // uint32 [(N + 31) / 32], bit i set: DoF i constrained
  int64_t n_constrained = 0;
  pmg::DeviceBuffer inv_diag;       // [N] dtype
  bool has_diag = false;
  int64_t warps_vmult = 0, warps_diag = 0; // resident warps of the cell kernels
  int64_t warps_vmult_ring = 0;             // ... of the geometry-ring vmult variant
  int sms = 0;                              // SM count of the device
  std::vector<pmg::DeviceBuffer> cg_work;   // CG work vectors kept between solves
  std::vector<pmg::DeviceBuffer> adj_work;  // adjoint-gradient work vectors
  pmg::DeviceBuffer err_flag;               // set by bounded device waits that give up
  // shape of the last launch of each grid-stride kernel (pmg_operator_last_launch): work
  // units (warp groups or cell batches) and the warps (or blocks) that shared them;
  // index PMG_KERNEL_VMULT_CELL .. PMG_KERNEL_QP_FORM
  mutable int64_t launch_units[4] = {0, 0, 0, 0};
  mutable int64_t launch_par[4] = {0, 0, 0, 0};
};

namespace pmg {
// operator.cu
void operator_setup(pmg_operator &op, const pmg_mesh &mesh, const pmg_operator_params &prm);
void operator_setup_from_maps(pmg_operator &op, const pmg_operator_maps &maps, const pmg_operator_params &prm);
// the operator's numbering on the host (copied from the device on first use)
const Numbering &host_numbering(const pmg_operator &op);
// fails with PMG_ESTATE for operators built from caller maps (no box mesh behind them)
inline void require_mesh(const pmg_operator &op, const char *what) {
  if (op.from_maps)
    fail(PMG_ESTATE, std::string(what) + " needs the library's box mesh; this operator was built from caller maps");
}
void operator_vmult(const pmg_operator &op, void *dst, const void *src, cudaStream_t s,
                    bool compute = true);
void operator_vmult_cells(const pmg_operator &op, void *dst, const void *src, int64_t cell_begin,
                          int64_t cell_end, bool init, cudaStream_t s);
bool operator_vmult_chebyshev(const pmg_operator &op, void *out, const void *cur, const void *prev, const void *b,
                              const void *invd, double f1, double f2, cudaStream_t s);
void operator_compute_inverse_diagonal(pmg_operator &op, cudaStream_t s);
void operator_assemble_rhs(const pmg_operator &op, int f_kind, int nq, void *b, cudaStream_t s);
void operator_copy_geometry(const pmg_operator &op, double *host);
int64_t operator_bytes(const pmg_operator &op);
void operator_set_coefficient(pmg_operator &op, const double *values, bool on_device, cudaStream_t s);
void operator_interpolate_coefficient(pmg_operator &dst, pmg_operator &src, cudaStream_t s);
void operator_quadrature_points(const pmg_operator &op, double *xq, cudaStream_t s);
double operator_l2_error(const pmg_operator &op, const void *u, int exact_kind, int nq, cudaStream_t s);
void operator_dof_coordinates(const pmg_operator &op, double *xyz, cudaStream_t s);
void operator_qp_form(const pmg_operator &op, const void *u, const void *v, double alpha, double *out,
                      cudaStream_t s);
} // namespace pmg
