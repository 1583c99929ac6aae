// DG-SIPG face terms (dg.cu).
#pragma once

#include <vector>

#include "pmg_internal.hpp"

namespace pmg {

struct DGHost {
  std::vector<double> M1, K1, dphi0, dphi1; // 1D GLL mass and stiffness matrices, basis derivatives at 0 and 1
  double h[3] = {0, 0, 0};
  double c_pen = 0;  // sigma = c_pen / h on every face (uniform boxes)
  int dirichlet = 0; // face mask
  bool tiles64 = false; // every 64 consecutive cells form a 4x4x4 cube (refine >= 2)
  DeviceBuffer nbr;  // int32 [cell][6] neighbour cells, -1 on the boundary
};

void dg_setup(DGHost &h, const BoxMesh &mesh, int degree, double c_pen);
// units / blocks (if set) receive the cell batches and the blocks of the face-kernel launch
void dg_apply_faces(const DGHost &h, int degree, int dtype, const void *src, void *dst, int64_t n_cells,
                    int sms, cudaStream_t s, int64_t *units = nullptr, int64_t *blocks = nullptr);
// A Chebyshev step that the fused kernel applies instead of storing A x (x = src):
// out = x + f1 (x - prev) + f2 invd (b - A x), prev null: zero; out (dst) may be prev, not src
struct DGChebStep {
  const void *prev, *b, *invd;
  double f1, f2;
};
// The whole DG vmult (cell stiffness and face terms) in one tile kernel where it applies
// (degrees 1 and 3, the box refined at least twice, the tiles filling the device twice or
// PMG_DG_FACE=2; PMG_DG_FUSE=0 turns it off): dst = A src, written once, or with cheb the
// Chebyshev step from it.  Returns false, with nothing launched, where it does not apply.
bool dg_apply_fused(const DGHost &h, int degree, int dtype, const void *src, void *dst, int64_t n_cells, int sms,
                    cudaStream_t s, int64_t *units = nullptr, int64_t *blocks = nullptr,
                    const DGChebStep *cheb = nullptr);
// whether dg_apply_fused would launch for this operator (nothing launched)
bool dg_fused_applies(const DGHost &h, int degree, int dtype, int64_t n_cells, int sms);
void dg_add_face_diagonal(const DGHost &h, int degree, int dtype, void *diag, int64_t n_cells, int sms,
                          cudaStream_t s);
void dg_add_boundary_rhs(const DGHost &h, const BoxMesh &mesh, int degree, int nq, int dtype, void *b,
                         cudaStream_t s);

} // namespace pmg
