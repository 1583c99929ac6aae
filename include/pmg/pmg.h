/*
 * pmg.h -- C ABI of the B200 matrix-free multigrid library (libpmg_b200.so).
 *
 * Every entry point is plain C: opaque handles, plain pointers and sizes, a pmg_status
 * return code (0 = success, negative = error, message via pmg_last_error).  Vectors are
 * device pointers owned by the caller; a `stream` argument is a cudaStream_t passed as
 * void* (NULL = the legacy default stream).  All work is ordered on that stream; only the
 * create functions, pmg_cg_solve and the Chebyshev eigenvalue estimate synchronise the host.
 * Handles are not thread safe; distinct handles may be used from distinct threads.
 *
 * The entry points replace the C++ virtual interfaces of the reference
 * (gshubhamk/portable-multigrid) for the matrix-free Laplace hot path; each declaration
 * names the interface member it stands in for.
 */
#ifndef PMG_PMG_H
#define PMG_PMG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pmg_status;
#define PMG_OK 0
#define PMG_EINVAL (-1)     /* bad argument or unsupported combination                 */
#define PMG_ENOMEM (-2)     /* device or host allocation failed                         */
#define PMG_ECUDA (-3)      /* a CUDA call failed                                       */
#define PMG_ENONFINITE (-4) /* a NaN or Inf appeared in a residual or a dot product     */
#define PMG_ENOCONV (-5)    /* iteration limit reached before the tolerance             */
#define PMG_EBOUNDS (-6)    /* an index map entry is out of range                       */
#define PMG_ESTATE (-7)     /* call made on an object in the wrong state                */
#define PMG_ENODEV (-8)     /* no CUDA device, or the library was built without one      */

typedef enum { PMG_F64 = 0, PMG_F32 = 1 } pmg_dtype;

typedef struct pmg_mesh pmg_mesh;
typedef struct pmg_operator pmg_operator;
typedef struct pmg_transfer pmg_transfer;
typedef struct pmg_chebyshev pmg_chebyshev;
typedef struct pmg_mg pmg_mg;

/* ---------------------------------------------------------------------------------- */
/* Errors and version                                                                 */
/* ---------------------------------------------------------------------------------- */

/* Copies the message of the last failed call on this host thread into buf (NUL
 * terminated, truncated to n bytes); returns the message length. */
size_t pmg_last_error(char *buf, size_t n);
/* Static name of a status code. */
const char *pmg_status_string(pmg_status status);
pmg_status pmg_version(int32_t *major, int32_t *minor);

/* ---------------------------------------------------------------------------------- */
/* Meshes                                                                             */
/* ---------------------------------------------------------------------------------- */

/* A box [lo,hi] of coarse[0]*coarse[1]*coarse[2] coarse hexahedra, each refined globally
 * `refine` times: GridGenerator::subdivided_hyper_rectangle + Triangulation::refine_global
 * as driven in tests/poisson_cube_bk3/program.cc:937-957.  Cells are ordered coarse cell by
 * coarse cell, Morton order inside each.  deform = 1 maps every Q_p mapping node by
 * x' = x + amp*sin(pi x)sin(pi y)sin(pi z) in each component.  dirichlet_mask bit f marks
 * face f (x-, x+, y-, y+, z-, z+) homogeneous Dirichlet (0x3F: all faces). */
typedef struct {
  int32_t coarse[3];
  int32_t refine;
  double lo[3];
  double hi[3];
  int32_t deform;
  double amp;
  int32_t dirichlet_mask;
} pmg_box;

pmg_status pmg_mesh_create_box(const pmg_box *box, pmg_mesh **mesh);
pmg_status pmg_mesh_destroy(pmg_mesh *mesh);
pmg_status pmg_mesh_n_cells(const pmg_mesh *mesh, int64_t *n_cells);
/* Integer coordinates (x, y, z) of every cell in the box's cell grid, in cell order, host
 * array xyz[n_cells][3]: the cell's lowest node sits at degree * (x, y, z) in the node lattice
 * (the child offsets a geometric transfer between refinements follows,
 * include/multigrid/portable_geometric_transfer.h:1095-1098). */
pmg_status pmg_mesh_cell_coordinates(const pmg_mesh *mesh, int32_t *xyz);

/* ---------------------------------------------------------------------------------- */
/* Level operators: Portable::LaplaceOperatorBase<3,Number>                           */
/* (include/base/portable_laplace_operator_base.h:17-61)                              */
/* ---------------------------------------------------------------------------------- */

#define PMG_GEOMETRY_AUTO 0   /* per-cell constants on undeformed boxes, else per point */
#define PMG_GEOMETRY_FULL 1   /* symmetric tensor G per quadrature point, 6*nq^3/cell   */
#define PMG_GEOMETRY_AFFINE 2 /* 6 constants per cell, times w_q and the coefficient   */
/* J^{-1} (9 values) and JxW per quadrature point, 10*nq^3/cell: the deal.II-style
 * formulation of include/operators/portable_laplace_operator.h:136-245 with
 * include/kernels/portable_local_laplace_operator.h:329-347 (inverse Jacobian applied twice
 * per point); any box, PMG_COEFF_NONE / _KAPPA / _VALUES folded into JxW */
#define PMG_GEOMETRY_INVJAC 3

#define PMG_COEFF_NONE 0   /* -lap u                                                   */
#define PMG_COEFF_KAPPA 1  /* kappa = 1 + 0.9 sin(2 pi x) sin(2 pi y) sin(2 pi z)      */
#define PMG_COEFF_VALUES 2 /* caller-supplied values per quadrature point [C][nq^3],
                              cell order of the mesh, points lexicographic (x fastest) on
                              the (degree+1)-point Gauss rule; NULL coeff_qp means 1      */

#define PMG_OP_LAPLACE 0 /* continuous FE_Q Laplace (LaplaceOperatorBK3)                 */
#define PMG_OP_DG_SIPG 1 /* discontinuous FE_DGQ symmetric interior penalty Laplace
                            (LaplaceOperatorDG, include/operators/portable_laplace_operator_dg.h);
                            axis-aligned undeformed boxes, no coefficient, Dirichlet data
                            enter weakly through the boundary faces                       */
#define PMG_OP_MASS 2    /* continuous FE_Q mass matrix (phi_i, kappa phi_j) with identity
                            rows on constrained DoFs; no counterpart in the reference (the
                            adjoint misfit J = 1/2 (u - u_d)^T M (u - u_d))               */

typedef struct {
  int32_t degree;          /* FE_Q / FE_DGQ degree 1..6 (OperatorDispatchFactory::max_degree) */
  int32_t dtype;           /* pmg_dtype: arithmetic and vector type                     */
  int32_t geometry;        /* PMG_GEOMETRY_*                                            */
  int32_t coeff_kind;      /* PMG_COEFF_*                                               */
  const double *coeff_qp;  /* host array [C][(degree+1)^3] for PMG_COEFF_VALUES or NULL */
  int32_t device;          /* CUDA device ordinal                                       */
  int32_t kind;            /* PMG_OP_*                                                  */
  double penalty;          /* DG: sigma = penalty/h; <= 0 selects the reference's p(p+1)
                              (portable_laplace_operator_dg.h:147-151)                     */
} pmg_operator_params;

/* LaplaceOperatorBK3 constructor + setup_dof_indices_per_color + compute_G_tensors
 * (include/operators/portable_laplace_operator_bk3.h:104-126, :360-437, :456-515). */
pmg_status pmg_operator_create(const pmg_mesh *mesh, const pmg_operator_params *params,
                               pmg_operator **op);
pmg_status pmg_operator_destroy(pmg_operator *op);

/* An operator on the caller's own discretisation, as LaplaceOperatorBK3 takes it from
 * deal.II's MatrixFree: setup_dof_indices_per_color (bk3.h:360-437) gives the cell -> DoF map
 * in lexicographic cell-local order with the sentinel on constrained DoFs, and
 * compute_G_tensors (bk3.h:456-515) forms G from MatrixFree's inv_jacobian and JxW.  All arrays
 * are host arrays, read during the call; the library regroups the cells (consecutive caller
 * cells share a warp, so a locality-preserving cell order reads HBM best) and permutes the
 * maps and geometry into its device layouts.
 *   dof_indices   [n_cells][(degree+1)^3] uint32, node (i,j,k) of a cell at (k*nm+j)*nm+i,
 *                 entries < n_dofs or 0xFFFFFFFF (constrained: no contribution);
 *   constrained   the DoFs whose rows are the identity (copy_constrained_values, bk3.h:230);
 *                 map entries naming one of them are treated as the sentinel;
 *   PMG_MAPS_G:   G [n_cells][6][(degree+1)^3] = JxW J^{-1} J^{-T} in the order rr, rs, rt, ss,
 *                 st, tt at the (degree+1)-point Gauss points (x fastest), coefficient folded in;
 *   PMG_MAPS_INVJAC: inv_jacobian [n_cells][(degree+1)^3][3][3] with [d][e] = d xi_d / d x_e
 *                 (MatrixFree's inverse Jacobian, portable_local_laplace_operator.h:329-347) and
 *                 JxW [n_cells][(degree+1)^3]: the deal.II-style formulation.
 * params: degree, dtype and device are used; kind must be PMG_OP_LAPLACE and coeff_kind
 * PMG_COEFF_NONE.  An entry >= n_dofs fails with PMG_EBOUNDS.  Such an operator has no box
 * mesh: the calls that evaluate data on the mesh (right-hand side, error norm, coordinates,
 * quadrature points, coefficients) and pmg_transfer_create fail with PMG_ESTATE; transfers
 * to and from it come from pmg_transfer_create_from_maps. */
#define PMG_INVALID_INDEX 0xFFFFFFFFu /* the constrained-DoF sentinel of an index map */
#define PMG_MAPS_G 0
#define PMG_MAPS_INVJAC 1
typedef struct {
  int64_t n_cells;
  int64_t n_dofs;
  const uint32_t *dof_indices;
  const uint32_t *constrained;
  int64_t n_constrained;
  int32_t geometry; /* PMG_MAPS_G or PMG_MAPS_INVJAC */
  const double *G;
  const double *inv_jacobian;
  const double *JxW;
} pmg_operator_maps;
pmg_status pmg_operator_create_from_maps(const pmg_operator_maps *maps, const pmg_operator_params *params,
                                         pmg_operator **op);
/* m() / n() (bk3.h:570-582). */
pmg_status pmg_operator_m(const pmg_operator *op, int64_t *m);
pmg_status pmg_operator_n(const pmg_operator *op, int64_t *n);
pmg_status pmg_operator_n_cells(const pmg_operator *op, int64_t *n_cells);
pmg_status pmg_operator_degree(const pmg_operator *op, int32_t *degree, int32_t *dtype);
/* vmult(dst, src): dst = A src with identity rows on constrained DoFs (bk3.h:128-231).
 * dst is overwritten; dst and src must not overlap. */
pmg_status pmg_operator_vmult(const pmg_operator *op, void *dst, const void *src, void *stream);
/* Tvmult == vmult (bk3.h:440-453). */
pmg_status pmg_operator_tvmult(const pmg_operator *op, void *dst, const void *src, void *stream);
/* vmult_dummy(dst, src, ghost_exchange_on, computation_on) (bk3.h:233-357): with one GPU
 * there is no ghost exchange; computation_on = 0 only zeroes dst and copies the
 * constrained values. */
pmg_status pmg_operator_vmult_dummy(const pmg_operator *op, void *dst, const void *src,
                                    int32_t ghost_exchange_on, int32_t computation_on,
                                    void *stream);
/* The cells [cell_begin, cell_end) of a continuous Laplace operator added into dst:
 * dst += A_K src summed over those cells K (in the operator's cell order: the caller's for
 * operators from maps, the mesh's otherwise).  init != 0 first sets dst as vmult does (zero,
 * with the identity rows of the constrained DoFs), so that
 *   vmult_cells(dst, src, 0, c, 1); vmult_cells(dst, src, c, n_cells, 0)
 * equals vmult(dst, src) up to the order of the floating-point additions.  This is the split
 * of the reference's colour loop (bk3.h:187-227): the cells that read no ghost DoFs are
 * computed while the ghost update is in flight, the others after it.  cell_begin and
 * cell_end are multiples of pmg_operator_cells_per_group (cell_end may also be n_cells);
 * PMG_EINVAL for DG, mass and tensor-core operators. */
pmg_status pmg_operator_vmult_cells(const pmg_operator *op, void *dst, const void *src, int64_t cell_begin,
                                    int64_t cell_end, int32_t init, void *stream);
/* Cells per warp group of the cell kernel: floor(32 / (degree + 1)). */
pmg_status pmg_operator_cells_per_group(const pmg_operator *op, int32_t *cells);
/* compute_diagonal() (bk3.h:533-561): inverse of diag(A), 1 on constrained rows. */
pmg_status pmg_operator_compute_diagonal(pmg_operator *op, void *stream);
/* get_matrix_diagonal_inverse() (bk3.h:563-568): device pointer owned by the operator,
 * valid until the operator is destroyed; PMG_ESTATE before compute_diagonal. */
pmg_status pmg_operator_get_inverse_diagonal(const pmg_operator *op, const void **inv_diag);
/* Copies the inverse diagonal into a caller-owned device vector (ordered on stream). */
pmg_status pmg_operator_copy_inverse_diagonal(const pmg_operator *op, void *dst, void *stream);
/* el(row, col) (bk3.h:584-595): 1/inv_diag(row); only row == col is defined. */
pmg_status pmg_operator_el(const pmg_operator *op, int64_t row, int64_t col, double *value);
/* Algorithmic bytes of one vmult: 2*s*N + 4*nm^3*C + geometry bytes. */
pmg_status pmg_operator_bytes_per_vmult(const pmg_operator *op, int64_t *bytes);
/* Right-hand side b_i = (phi_i, f) with an nq-point Gauss rule, zero on constrained DoFs
 * (tests/poisson_cube_bk3/program.cc:517-566): f_kind 0: f = 1;
 * f_kind 1: f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z);
 * f_kind 2: u = exp(x) sin(pi y) cos(pi z), f = (2 pi^2 - 1) u, and for DG operators the
 * weakly imposed Dirichlet data (g, 2 sigma phi_i - d_n phi_i) on Dirichlet faces.
 * b has the operator's dtype. */
pmg_status pmg_operator_assemble_rhs(const pmg_operator *op, int32_t f_kind, int32_t nq,
                                     void *b, void *stream);
/* Inspection, host copies in the reference layouts: the dof index map with the
 * 0xFFFFFFFF sentinel [C][nm^3] (bk3.h:397-433), the constrained flags [N], and the
 * geometry tensor [C][6][nq^3] in the order rr,rs,rt,ss,st,tt (bk3.h:477-510; full
 * geometry only). */
pmg_status pmg_operator_copy_dof_indices(const pmg_operator *op, uint32_t *host);
pmg_status pmg_operator_copy_constrained(const pmg_operator *op, uint8_t *host);
pmg_status pmg_operator_copy_geometry(const pmg_operator *op, double *host);

/* The tensor-core variant of the cell kernel for FP32 operators with affine geometry (the
 * BF16/TF32 contraction variant; the reference contracts on CUDA cores only): mode 1 applies
 * the twelve 1D contractions of every cell as TF32 mma.sync products (10-bit mantissas, FP32
 * accumulation, about 1e-3 relative), mode 3 as three TF32 products per contraction (hi*hi +
 * hi*lo + lo*hi, about FP32 accuracy), mode 0 returns to the CUDA-core kernel.  PMG_EINVAL for
 * FP64, DG, mass or non-affine operators. */
pmg_status pmg_operator_set_tensor_cores(pmg_operator *op, int32_t mode);

/* Node-lattice coordinates (i, j, k) of every DoF of a continuous operator on a box mesh,
 * host array ijk[N][3] (x fastest in the lattice of degree * cells + 1 points per direction):
 * the support points a partitioned mesh matches across ranks (the ghost DoFs of
 * portable_laplace_operator_bk3.h:187-227).  PMG_ESTATE for DG and caller-map operators. */
pmg_status pmg_operator_dof_lattice(const pmg_operator *op, int32_t *ijk);

/* Shape of the last launch of one of the operator's grid-stride kernels (inspection; the
 * reference launches one Kokkos team per cell batch and has no counterpart): *units = the
 * work units (warp groups of cells; cell batches or 4x4x4 cell tiles for the DG face
 * kernels) and *parallel = the warps (blocks for the DG face kernels) of the grid that shared
 * them, so a launch with units >= 2 * parallel gave every warp two or more units.  Where a DG
 * vmult runs as one fused tile kernel (cell and face terms), both the VMULT_CELL and the
 * DG_FACES records describe that launch.  Zero before the first launch. */
#define PMG_KERNEL_VMULT_CELL 0 /* the cell kernel of vmult                              */
#define PMG_KERNEL_DG_FACES 1   /* the face kernel of a DG vmult                         */
#define PMG_KERNEL_MASS 2       /* the cell kernel of a mass-matrix vmult                */
#define PMG_KERNEL_QP_FORM 3    /* the kernel of pmg_operator_qp_form                    */
pmg_status pmg_operator_last_launch(const pmg_operator *op, int32_t kernel, int64_t *units,
                                    int64_t *parallel);

/* Coefficient fields and per-point forms (the adjoint path; no counterpart in the reference).
 * set_coefficient: new PMG_COEFF_VALUES values [C][nq^3] (FP64; on_device selects a device
 * or a host pointer), rebuilding G / the per-point factors / the mass weights on the stream.
 * The inverse diagonal keeps describing the old values until pmg_operator_compute_diagonal. */
pmg_status pmg_operator_set_coefficient(pmg_operator *op, const double *coeff_qp, int32_t on_device,
                                        void *stream);
/* dst's coefficient := src's coefficient field at dst's quadrature points: both on the same box,
 * src refined at least as often; log(coefficient) is interpolated by the tensor Lagrange
 * polynomial through src's Gauss points of the containing cell, so values stay positive. */
pmg_status pmg_operator_interpolate_coefficient(pmg_operator *dst, pmg_operator *src, void *stream);
/* ||u_h - u||_{L2(Omega)} of the FE function with DoF values u (the operator's dtype, every DoF
 * counted, Dirichlet ones included) against the exact solution of the manufactured problems of
 * pmg_operator_assemble_rhs: exact_kind 1: u = sin(pi x) sin(pi y) sin(pi z) (f_kind 1),
 * exact_kind 2: u = exp(x) sin(pi y) cos(pi z) (f_kind 2); an nq-point Gauss rule per direction
 * (nq <= 0: degree + 2), evaluated on the GPU with a deterministic sum.  Replaces the host
 * FEValues error loop of tests/poisson_cube_bk3/program.cc.  Synchronises. */
pmg_status pmg_operator_l2_error(const pmg_operator *op, const void *u, int32_t exact_kind, int32_t nq,
                                 double *error, void *stream);
/* Support point of every DoF, device array xyz[n_dofs][3] (FP64): where Dirichlet data is
 * evaluated, as deal.II's VectorTools::interpolate_boundary_values does for the constraints
 * (source/plain_solver/program.cc:125-131, homogeneous there).  With it inhomogeneous data is
 * imposed by lifting: u_D = g at the Dirichlet DoFs (0 elsewhere), b0 = b - A0 u_D on the free
 * rows (A0 the operator of the same mesh without Dirichlet DoFs), solve A u0 = b0, u = u0 + u_D.
 * Synchronises. */
pmg_status pmg_operator_dof_coordinates(const pmg_operator *op, double *xyz, void *stream);
/* Quadrature points of the operator's Gauss rule, device array xq[C][nq^3][3] (FP64). */
pmg_status pmg_operator_quadrature_points(const pmg_operator *op, double *xq, void *stream);
/* out[c][q] = alpha * grad u(x_q)^T kappa_q |det J| w_q J^{-1} J^{-T} grad v(x_q) in reference
 * gradients, i.e. the integrand of a(u, v) per quadrature point (FP64 device array [C][nq^3];
 * u and v have the operator's dtype, constrained entries read as 0).  For kappa = exp(m):
 * d(u^T A v)/dm_q = out with alpha = 1. */
pmg_status pmg_operator_qp_form(const pmg_operator *op, const void *u, const void *v, double alpha,
                                double *out, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Transfers: Portable::MGTransferBase<3,number>                                      */
/* (include/base/portable_mg_transfer_base.h:16-37)                                   */
/* ---------------------------------------------------------------------------------- */

/* reinit(mf_coarse, mf_fine, constraints_coarse, constraints_fine): a polynomial transfer
 * (PolynomialTransfer, include/multigrid/portable_polynomial_transfer.h:1044-1361) when
 * both operators live on the same mesh with degree_coarse < degree_fine, a geometric one
 * (GeometricTransfer, include/multigrid/portable_geometric_transfer.h:944-1486) when the
 * degrees agree and the fine mesh is the coarse box refined once more, and the DG <-> CG
 * transfer (ContinuousTransfer, include/multigrid/portable_continuous_transfer.h:110-319)
 * when the fine operator is DG and the coarse one continuous of the same degree on the same
 * mesh.  Both operators must have the same dtype. */
pmg_status pmg_transfer_create(const pmg_operator *coarse, const pmg_operator *fine,
                               pmg_transfer **transfer);
/* reinit(mf_coarse, mf_fine, constraints_coarse, constraints_fine) from the caller's own maps
 * (the index arrays PolynomialTransfer / GeometricTransfer / ContinuousTransfer build from
 * MatrixFree and the constraints: portable_polynomial_transfer.h:1116-1245,
 * portable_geometric_transfer.h:1294-1330, portable_continuous_transfer.h:339-485).  One
 * patch is a cell of the fine mesh (polynomial, DG <-> CG) or of the coarse mesh (geometric):
 *   kind            PMG_TRANSFER_POLYNOMIAL: nc = degree_c+1, nf = degree_f+1, degree_c < degree_f,
 *                   the 1D matrix interpolates FE_Q(degree_c) at FE_Q(degree_f)'s nodes;
 *                   PMG_TRANSFER_GEOMETRIC: equal degrees p, nc = p+1, nf = 2p+1 (the patch's
 *                   two children per direction share their middle nodes), the 1D matrix
 *                   interpolates at the children's nodes;
 *                   PMG_TRANSFER_DG_CG: equal degrees, fine = FE_DGQ, identity per entry;
 *   coarse_indices  [n_patches][nc^3] lexicographic, 0xFFFFFFFF for constrained coarse DoFs;
 *   fine_indices    [n_patches][nf^3] lexicographic, every fine DoF of the patch;
 *   weights         [n_patches][nf^3] or NULL: NULL gives the reference's 1 / (number of
 *                   patches holding the fine DoF), 0 on the fine operator's constrained DoFs.
 * Host arrays, read during the call; entries out of range fail with PMG_EBOUNDS.  The
 * operators may come from a mesh or from caller maps; they fix n_dofs, dtype and device. */
#define PMG_TRANSFER_POLYNOMIAL 0
#define PMG_TRANSFER_GEOMETRIC 1
#define PMG_TRANSFER_DG_CG 2
typedef struct {
  int32_t kind;
  int64_t n_patches;
  const uint32_t *coarse_indices;
  const uint32_t *fine_indices;
  const double *weights;
} pmg_transfer_maps;
pmg_status pmg_transfer_create_from_maps(const pmg_operator *coarse, const pmg_operator *fine,
                                         const pmg_transfer_maps *maps, pmg_transfer **transfer);
pmg_status pmg_transfer_destroy(pmg_transfer *transfer);
/* prolongate_and_add(dst_fine, src_coarse) */
pmg_status pmg_transfer_prolongate_and_add(const pmg_transfer *transfer, void *dst_fine,
                                           const void *src_coarse, void *stream);
/* restrict_and_add(dst_coarse, src_fine) */
pmg_status pmg_transfer_restrict_and_add(const pmg_transfer *transfer, void *dst_coarse,
                                         const void *src_fine, void *stream);
/* Shape of the last launch (inspection, no reference counterpart): *units = patches (the
 * DG <-> CG transfer: entries; the runtime-size kernel: patch batches) and *parallel = the
 * warps (threads; blocks) of the grid that shared them.  Zero before the first launch. */
pmg_status pmg_transfer_last_launch(const pmg_transfer *transfer, int64_t *units, int64_t *parallel);

/* ---------------------------------------------------------------------------------- */
/* Smoother: deal.II PreconditionChebyshev<LaplaceOperatorBase, Vector> as configured at */
/* tests/poisson_cube_bk3/program.cc:474-515                                          */
/* ---------------------------------------------------------------------------------- */

typedef struct {
  int32_t degree;              /* <= 0: chosen so the Chebyshev bound reaches range   */
  double smoothing_range;      /* > 1: lambda_max/range; < 1: target reduction        */
  int32_t eig_cg_n_iterations; /* CG steps of the eigenvalue estimate                 */
} pmg_chebyshev_params;

/* initialize(matrix, data) with the operator's inverse diagonal as preconditioner
 * (computed here if needed); the eigenvalue estimate runs on the first use or in
 * pmg_chebyshev_estimate. */
pmg_status pmg_chebyshev_create(pmg_operator *op, const pmg_chebyshev_params *params,
                                pmg_chebyshev **smoother);
pmg_status pmg_chebyshev_destroy(pmg_chebyshev *smoother);
pmg_status pmg_chebyshev_estimate(pmg_chebyshev *smoother, void *stream);
/* vmult(dst, src): degree-1 matrix-vector products from a zero initial guess. */
pmg_status pmg_chebyshev_vmult(pmg_chebyshev *smoother, void *dst, const void *src,
                               void *stream);
/* step(dst, src): degree products starting from dst. */
pmg_status pmg_chebyshev_step(pmg_chebyshev *smoother, void *dst, const void *src,
                              void *stream);
pmg_status pmg_chebyshev_info(const pmg_chebyshev *smoother, double *min_eigenvalue,
                              double *max_eigenvalue, int32_t *degree, int32_t *cg_iterations);

/* ---------------------------------------------------------------------------------- */
/* V-cycle: VCycleMultigridBase::vmult (include/base/portable_v_cycle_multigrid_base.h:   */
/* 18-27), MultigridSolver::vmult / v_cycle (tests/common/portable_multigrid_solver.h:    */
/* 171-271)                                                                           */
/* ---------------------------------------------------------------------------------- */

/* levels[0] is the coarsest; transfers[l] connects levels l-1 and l (transfers[0] is
 * ignored); smoothers[l] smooths level l (smoothers[0] is the coarse solver).  The
 * objects are borrowed and must outlive the multigrid handle. */
pmg_status pmg_mg_create(int32_t n_levels, pmg_operator *const *levels,
                         pmg_transfer *const *transfers, pmg_chebyshev *const *smoothers,
                         pmg_mg **mg);
pmg_status pmg_mg_destroy(pmg_mg *mg);
/* dst = V-cycle(src); src and dst have dtype vec_dtype, converted on entry and exit when
 * it differs from the finest level's dtype. */
pmg_status pmg_mg_vmult(pmg_mg *mg, void *dst, const void *src, int32_t vec_dtype,
                        void *stream);

/* ---------------------------------------------------------------------------------- */
/* Conjugate gradients: MultigridSolver::solve_cg (portable_multigrid_solver.h:147-169)  */
/* with deal.II SolverCG + ReductionControl                                           */
/* ---------------------------------------------------------------------------------- */

typedef struct {
  int32_t iterations;
  int32_t converged;
  double initial_residual;
  double final_residual;
  double reduction_per_step; /* (final/initial)^(1/iterations), as the reference reports */
} pmg_cg_info;

/* Solves A x = b (A FP64) by preconditioned CG from the given x, stopping when
 * ||r|| <= max(abs_tol, reduce*||r_0||) or after max_iterations (PMG_ENOCONV).
 * precond: NULL = the operator's Jacobi preconditioner (computed if needed), else a
 * multigrid V-cycle. */
pmg_status pmg_cg_solve(pmg_operator *A, pmg_mg *precond, void *x, const void *b,
                        double reduce, double abs_tol, int32_t max_iterations,
                        pmg_cg_info *info, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Adjoint gradient of J(m) = 1/2 ||u(m) - u_d||^2_{L2} for -div(exp(m) grad u) = f     */
/* (no counterpart in the reference)                                                  */
/* ---------------------------------------------------------------------------------- */

/* New coefficient values on a whole hierarchy: A (may be NULL) and the finest level take
 * coeff_qp, every coarser level interpolates the one above it
 * (pmg_operator_interpolate_coefficient); then every level's inverse diagonal and smoother
 * eigenvalue estimate are recomputed.  Every level needs PMG_COEFF_VALUES.  Synchronises. */
pmg_status pmg_mg_set_coefficient(pmg_mg *mg, pmg_operator *A, const double *coeff_qp,
                                  int32_t on_device, void *stream);
/* Given the forward solution u of A u = b (A FP64 with coefficient exp(m), M the FP64 mass
 * operator of the same space): J = 1/2 (u-u_d)^T M (u-u_d), the adjoint solve
 * A lambda = M (u - u_d) by CG with the multigrid preconditioner (NULL: Jacobi) from
 * lambda = 0, and g_qp[c][q] = dJ/dm_q = -exp(m_q) grad lambda^T G grad u (FP64 device
 * array [C][nq^3]).  info describes the adjoint solve.  Synchronises. */
pmg_status pmg_adjoint_gradient(pmg_operator *A, const pmg_operator *M, pmg_mg *precond, const void *u,
                                const void *u_d, void *lambda, double *g_qp, double *J, double reduce,
                                double abs_tol, int32_t max_iterations, pmg_cg_info *info,
                                void *stream);

/* ---------------------------------------------------------------------------------- */
/* Vector kernels on the path: LinearAlgebra::distributed::Vector operator* (the CG dot  */
/* products) and copy_locally_owned_data_from across precisions                        */
/* (tests/common/portable_multigrid_solver.h:185, :191)                                */
/* ---------------------------------------------------------------------------------- */

/* *result = sum_i a_i b_i over n entries of dtype, accumulated in FP64 with a fixed
 * reduction order (deterministic); synchronises the stream to return the value.  The
 * reductions of the library (this dot, the fused CG and Jacobi updates inside pmg_cg_solve,
 * the Chebyshev estimate) share one partial-sum buffer per device: they must not run
 * concurrently on one device from different host threads or unordered streams. */
pmg_status pmg_vector_dot(const void *a, const void *b, int32_t dtype, int64_t n, double *result,
                          void *stream);
/* The dot product of pmg_vector_dot for callers that cannot allocate device memory at the
 * point of the call (their allocator owns the device budget, or they cannot afford the
 * synchronisation cudaMalloc/cudaFree may imply).  No counterpart in the reference.
 * Allocates nothing: its scratch is a fixed 32 KB array in the library's device image,
 * held on every GPU that loads the library until exit.  *result_dev (a caller-owned device
 * double) receives the FP64-accumulated sum, ordered on stream, without a host
 * synchronisation.  The reduction order is fixed for a given n and device (deterministic)
 * but differs from pmg_vector_dot's, so the two may differ in the last bits.  n is limited
 * to 268,435,456 entries (PMG_EINVAL beyond).  The first call on a device looks up the
 * scratch address and should come before any stream capture; the address is kept for the
 * life of the process, which assumes the device's primary context is never reset
 * (cudaDeviceReset) and that calls run in it.  Calls that overlap on the GPU share the
 * scratch and race. */
pmg_status pmg_vector_dot_noalloc(const void *a, const void *b, int32_t dtype, int64_t n,
                                  double *result_dev, void *stream);
/* Vector updates of the CG and Chebyshev iterations (LinearAlgebra::distributed::Vector add /
 * sadd / scale, used by SolverCG), n entries of dtype, ordered on stream:
 * axpy: y += alpha x;  xpay: y = x + alpha y;  pointwise_mult: z = d .* r. */
pmg_status pmg_vector_axpy(void *y, const void *x, double alpha, int32_t dtype, int64_t n, void *stream);
pmg_status pmg_vector_xpay(void *y, const void *x, double alpha, int32_t dtype, int64_t n, void *stream);
pmg_status pmg_vector_pointwise_mult(void *z, const void *d, const void *r, int32_t dtype, int64_t n,
                                     void *stream);
/* One Chebyshev step of PreconditionChebyshev (deal.II), fused: out = cur + f1 (cur - prev) +
 * f2 inv_diag .* (src - Ax), prev == NULL meaning zero; out may alias prev. */
pmg_status pmg_vector_chebyshev_step(void *out, const void *cur, const void *prev, const void *src,
                                     const void *Ax, const void *inv_diag, double f1, double f2, int32_t dtype,
                                     int64_t n, void *stream);
/* dst (dt_dst) = src (dt_src), n entries, converting between FP64 and FP32. */
pmg_status pmg_vector_copy(void *dst, int32_t dt_dst, const void *src, int32_t dt_src, int64_t n,
                           void *stream);

/* ---------------------------------------------------------------------------------- */
/* Kernel timing (no reference counterpart; the reference times with deal.II Timer)   */
/* ---------------------------------------------------------------------------------- */

/* While enabled, every instrumented kernel launch records a CUDA event pair on its own
 * stream.  Labels: "vmult_cell", "vmult_constrained", "diag_cell", "transfer_prolongate",
 * "transfer_restrict". */
pmg_status pmg_profile_enable(int32_t on);
pmg_status pmg_profile_reset(void);
/* Waits for the recorded events of `kernel` and returns their summed device time and the
 * number of launches since the last reset. */
pmg_status pmg_profile_query(const char *kernel, double *total_ms, int64_t *launches);

/* Same-run peaks for roofline fractions (no reference counterpart): a device-to-device copy
 * over two buffers of copy_bytes each (256 MiB .. 16 GiB, larger than L2; copy_gbs counts
 * bytes read plus written) and FP64 / FP32 FMA throughput (2 flops per FMA, no memory
 * traffic).  Allocates 2 x copy_bytes for the duration of the call and synchronises. */
typedef struct pmg_peaks {
  double copy_gbs;
  double fp64_fma_tflops;
  double fp32_fma_tflops;
  int64_t copy_bytes;
  int32_t sm_count;
} pmg_peaks;
pmg_status pmg_measure_peaks(int32_t device, int64_t copy_bytes, pmg_peaks *out);

#ifdef __cplusplus
}
#endif

#endif /* PMG_PMG_H */
