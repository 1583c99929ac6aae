// Structured box meshes (host side, setup only) and the FE_DGQ numbering on them.
//
// The reference takes its meshes from GridGenerator::subdivided_hyper_rectangle refined
// globally on a p4est triangulation (tests/poisson_cube_bk3/program.cc:937-957,
// :263-278) and its numbering from deal.II's DoFHandler.  Here the box is generated
// directly: coarse cells lexicographically, each refined cell set in Morton order (the
// order p4est gives globally refined trees).  The FE_Q numbering along that order is built on
// the device (numbering.cu).
#include <algorithm>

#include "pmg_internal.hpp"

namespace pmg {

BoxMesh make_box(const pmg_box &b) {
  PMG_REQUIRE(b.refine >= 0 && b.refine <= 12, "refine must be in [0,12]");
  for (int d = 0; d < 3; ++d) {
    PMG_REQUIRE(b.coarse[d] >= 1, "coarse subdivisions must be >= 1");
    PMG_REQUIRE(b.hi[d] > b.lo[d], "box must have hi > lo");
  }
  PMG_REQUIRE(b.deform == 0 || b.deform == 1, "deform must be 0 or 1");
  BoxMesh m;
  m.box = b;
  for (int d = 0; d < 3; ++d) m.n[d] = (int64_t)b.coarse[d] << b.refine;
  m.n_cells = m.n[0] * m.n[1] * m.n[2];
  PMG_REQUIRE(m.n_cells < (int64_t(1) << 31), "too many cells");
  m.cell_xyz.resize(3 * m.n_cells);
  const int L = b.refine;
  const int64_t per_tree = int64_t(1) << (3 * L);
  int64_t c = 0;
  for (int tz = 0; tz < b.coarse[2]; ++tz)
    for (int ty = 0; ty < b.coarse[1]; ++ty)
      for (int tx = 0; tx < b.coarse[0]; ++tx)
        for (int64_t code = 0; code < per_tree; ++code, ++c) {
          int32_t xyz[3] = {0, 0, 0};
          for (int bit = 0; bit < L; ++bit)
            for (int d = 0; d < 3; ++d) xyz[d] |= int32_t((code >> (3 * bit + d)) & 1) << bit;
          m.cell_xyz[3 * c + 0] = (tx << L) + xyz[0];
          m.cell_xyz[3 * c + 1] = (ty << L) + xyz[1];
          m.cell_xyz[3 * c + 2] = (tz << L) + xyz[2];
        }
  return m;
}

// FE_DGQ(p): every cell owns its (p+1)^3 DoFs, numbered cell by cell in lexicographic order
// (deal.II numbers FE_DGQ DoFs the same way); nothing is constrained, Dirichlet data enter
// weakly through the face terms.
Numbering make_numbering_dg(const BoxMesh &m, int p) {
  Numbering nb;
  nb.p = p;
  const int64_t nm3 = int64_t(p + 1) * (p + 1) * (p + 1);
  PMG_REQUIRE(m.n_cells * nm3 < (int64_t(1) << 32) - 1, "too many DoFs for 32-bit indices");
  nb.n_dofs = m.n_cells * nm3;
  nb.plain.resize(nb.n_dofs);
  for (int64_t i = 0; i < nb.n_dofs; ++i) nb.plain[i] = (uint32_t)i;
  nb.constrained.assign(nb.n_dofs, 0);
  return nb;
}

} // namespace pmg
