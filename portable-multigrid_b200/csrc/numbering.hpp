// Device-side setup: DoF numbering of box meshes, constrained lists, slab index maps (numbering.cu).
#pragma once

#include "pmg_internal.hpp"

namespace pmg {

// first-visit numbering of FE_Q(p) on a box mesh, on the device: plain [C][nm^3] (no
// sentinel), lattice [L2][L1][L0] -> DoF, constrained [N] flags
struct DeviceNumbering {
  int p = 0;
  int64_t n_dofs = 0;
  int64_t L[3] = {0, 0, 0};
  DeviceBuffer plain, lattice, constrained;
};

void device_numbering(const BoxMesh &m, int p, const DeviceBuffer &cell_xyz, int sms, DeviceNumbering &out,
                      cudaStream_t s);
// out[i] = sum_{j < i} in[j] (uint32, deterministic); synchronises s
void exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, cudaStream_t s);
// the DoFs whose flag is set, ascending, and the bitmask of them; synchronises s
void device_constrained(const uint8_t *cons, int64_t n, int sms, DeviceBuffer &list, DeviceBuffer &bits,
                        int64_t &n_constrained, cudaStream_t s);
// the slab layout [group][k*N+i][e*N+j] of an index map, sentinel on constrained DoFs
void device_slab_index(const uint32_t *plain, const uint8_t *cons, int64_t n_cells, int N, int cpw, int lanes,
                       int64_t n_groups, int sms, DeviceBuffer &idx, cudaStream_t s);

} // namespace pmg
