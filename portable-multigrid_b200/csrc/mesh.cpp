// Structured box meshes and the FE_Q(p) DoF numbering on them (host side, setup only).
//
// The reference takes its meshes from GridGenerator::subdivided_hyper_rectangle refined
// globally on a p4est triangulation (tests/poisson_cube_bk3/program.cc:937-957,
// :263-278) and its numbering from deal.II's DoFHandler.  Here the box is generated
// directly: coarse cells lexicographically, each refined cell set in Morton order (the
// order p4est gives globally refined trees), and DoFs numbered in order of first visit
// along that cell order with each cell's nodes in lexicographic order, so that the DoFs a
// batch of consecutive cells touches are close together in memory.
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

Numbering make_numbering(const BoxMesh &m, int p, bool keep_lattice) {
  Numbering nb;
  nb.p = p;
  const int nm = p + 1, nm3 = nm * nm * nm;
  for (int d = 0; d < 3; ++d) nb.L[d] = p * m.n[d] + 1;
  const int64_t n_lat = nb.L[0] * nb.L[1] * nb.L[2];
  PMG_REQUIRE(n_lat < (int64_t(1) << 32) - 1, "too many DoFs for 32-bit indices");
  nb.lattice.assign(n_lat, kInvalid);
  nb.plain.resize(m.n_cells * nm3);
  std::vector<uint8_t> cons;
  cons.reserve(n_lat);
  const int mask = m.box.dirichlet_mask;
  uint32_t next = 0;
  for (int64_t c = 0; c < m.n_cells; ++c) {
    const int64_t bx = int64_t(p) * m.cell_xyz[3 * c], by = int64_t(p) * m.cell_xyz[3 * c + 1],
                  bz = int64_t(p) * m.cell_xyz[3 * c + 2];
    uint32_t *out = nb.plain.data() + c * nm3;
    for (int k = 0; k < nm; ++k)
      for (int j = 0; j < nm; ++j) {
        const int64_t row = ((bz + k) * nb.L[1] + (by + j)) * nb.L[0] + bx;
        for (int i = 0; i < nm; ++i) {
          uint32_t &slot = nb.lattice[row + i];
          if (slot == kInvalid) {
            slot = next++;
            const int64_t gx = bx + i, gy = by + j, gz = bz + k;
            const bool on = ((mask & 1) && gx == 0) || ((mask & 2) && gx == nb.L[0] - 1) ||
                            ((mask & 4) && gy == 0) || ((mask & 8) && gy == nb.L[1] - 1) ||
                            ((mask & 16) && gz == 0) || ((mask & 32) && gz == nb.L[2] - 1);
            cons.push_back(on ? 1 : 0);
          }
          out[(k * nm + j) * nm + i] = slot;
        }
      }
  }
  nb.n_dofs = next;
  nb.constrained = std::move(cons);
  if (!keep_lattice) std::vector<uint32_t>().swap(nb.lattice);
  return nb;
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
