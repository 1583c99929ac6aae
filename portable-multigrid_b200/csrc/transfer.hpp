// Multigrid transfer objects (transfer.cu).
#pragma once

#include <vector>

#include "pmg_internal.hpp"

struct pmg_transfer {
  int device = 0;
  int dtype = PMG_F64;
  int kind = 0; // 0 polynomial, 1 geometric, 2 DG <-> CG
  int nc = 0, nf = 0;
  int64_t n_patches = 0, n_coarse = 0, n_fine = 0;
  pmg::DeviceBuffer P1d, coarse_idx, fine_idx, weights;
  std::vector<double> P_host; // the 1D matrix [nc][nf], passed to the kernels by value
  int ppb = 1, grid = 1;
  size_t smem = 0;
  int sms = 0;               // SM count of the device
  bool patch_kernels = true; // warp-per-patch kernels for the compiled (nc, nf) pairs
  // last launch (pmg_transfer_last_launch): patches (or entries) and the warps (or threads)
  // of the grid that shared them
  mutable int64_t launch_units = 0, launch_par = 0;
};

namespace pmg {
void transfer_setup(pmg_transfer &t, const pmg_operator &coarse, const pmg_operator &fine);
void transfer_setup_from_maps(pmg_transfer &t, const pmg_operator &coarse, const pmg_operator &fine,
                              const pmg_transfer_maps &maps);
// dir 0: dst_fine += P src_coarse;  dir 1: dst_coarse += P^T src_fine
void transfer_apply(const pmg_transfer &t, int dir, void *dst, const void *src, cudaStream_t s);
} // namespace pmg
