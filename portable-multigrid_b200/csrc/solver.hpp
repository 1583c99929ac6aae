// Smoother, multigrid and CG objects (solver.cu).
#pragma once

#include <vector>

#include "pmg_internal.hpp"

struct pmg_chebyshev {
  pmg_operator *op = nullptr; // borrowed: may be gone when the smoother is destroyed
  int device = 0;             // the operator's device, kept for the destructor
  int degree = 0;
  int requested_degree = 0; // <= 0: the degree is chosen by every eigenvalue estimate
  int generation = 0;       // incremented by every eigenvalue estimate
  double range = 15.0;
  int eig_its = 10;
  bool estimated = false;
  double theta = 1, delta = 0, min_ev = 1, max_ev = 1;
  int cg_its = 0;
  pmg::DeviceBuffer xo, Ax;
  std::vector<pmg::DeviceBuffer> est_work; // eigenvalue-estimate vectors kept once re-estimated
};

struct pmg_mg {
  int device = 0; // the finest level's device, kept for the destructor (the levels are borrowed)
  std::vector<pmg_operator *> levels;
  std::vector<pmg_transfer *> transfers;
  std::vector<pmg_chebyshev *> smoothers;
  std::vector<pmg::DeviceBuffer> sol, def, t;
  // The V-cycle below the finest level's input and output buffers is a fixed sequence of
  // launches on fixed buffers: it is captured once into a CUDA graph and replayed.
  cudaGraphExec_t graph = nullptr;
  bool graph_enabled = true;
  std::vector<int> graph_generations; // smoother estimates the graph was captured with
  ~pmg_mg() {
    if (graph) cudaGraphExecDestroy(graph);
  }
};

namespace pmg {
void chebyshev_setup(pmg_chebyshev &c, pmg_operator &op, const pmg_chebyshev_params &prm);
void chebyshev_estimate(pmg_chebyshev &c, cudaStream_t s);
void chebyshev_apply(pmg_chebyshev &c, void *dst, const void *src, bool from_zero, cudaStream_t s);
void mg_setup(pmg_mg &mg, int n_levels, pmg_operator *const *levels, pmg_transfer *const *transfers,
              pmg_chebyshev *const *smoothers);
void mg_vmult(pmg_mg &mg, void *dst, const void *src, int vec_dtype, cudaStream_t s);
void cg_solve(pmg_operator &A, pmg_mg *mg, void *x, const void *b, double reduce, double abs_tol,
              int max_it, pmg_cg_info &info, cudaStream_t s);
void mg_set_coefficient(pmg_mg &mg, pmg_operator *A, const double *values, bool on_device, cudaStream_t s);
void adjoint_gradient(pmg_operator &A, const pmg_operator &M, pmg_mg *mg, const void *u, const void *u_d,
                      void *lambda, double *g_qp, double &J, double reduce, double abs_tol, int max_it,
                      pmg_cg_info &info, cudaStream_t s);
} // namespace pmg
