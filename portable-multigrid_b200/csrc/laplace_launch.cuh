// Launchers of the slab kernels for one polynomial degree.  Included by laplace_p<d>.cu
// with PMG_DEGREE defined, so each degree compiles as its own translation unit.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <set>
#include <utility>

#include "laplace_kernels.cuh"
#include "pmg_internal.hpp"

#ifndef PMG_DEGREE
#error "define PMG_DEGREE before including laplace_launch.cuh"
#endif

#define PMG_CAT2(a, b) a##b
#define PMG_CAT(a, b) PMG_CAT2(a, b)

namespace pmg {
namespace {

constexpr int kN = PMG_DEGREE + 1;
constexpr int kWarpsPerBlock = 4;

template <typename T> kern::Tab<kN, T> make_tab(const SlabLaunch &L) {
  kern::Tab<kN, T> t;
  for (int a = 0; a < kN * kN; ++a) {
    t.S[a] = (T)L.S[a];
    t.SD[a] = (T)L.SD[a];
    t.D[a] = (T)L.D[a];
  }
  for (int a = 0; a < kN; ++a) t.W[a] = (T)L.W[a];
  kern::fill_even_odd(t, L.S, L.SD);
  return t;
}

template <typename T> kern::Tab2<kN, T> make_tab2(const SlabLaunch &L) {
  kern::Tab2<kN, T> t;
  for (int a = 0; a < kN * kN; ++a) {
    t.S2[a] = (T)(L.S[a] * L.S[a]);
    t.SS[a] = (T)(L.S[a] * L.SD[a]);
    t.D2[a] = (T)(L.SD[a] * L.SD[a]);
  }
  for (int a = 0; a < kN; ++a) t.W[a] = (T)L.W[a];
  return t;
}

// warps per block of vmult_slab_kernel: one for the ring variant; for the direct variant four,
// unless a warp needs more than 24 KB of shared memory (FP64 at N >= 6), where blocks of four
// would leave most of an SM's shared memory unused (one 132-220 KB block per SM)
template <typename T, bool SMEM_G, int PIPE> constexpr int vmult_wpb() {
  return (SMEM_G || kern::SlabSmem<kN, T, SMEM_G, PIPE>::PER_WARP > 24 * 1024) ? 1 : kWarpsPerBlock;
}
template <typename T, bool SMEM_G, int PIPE> constexpr size_t vmult_smem() {
  return size_t(vmult_wpb<T, SMEM_G, PIPE>()) * kern::SlabSmem<kN, T, SMEM_G, PIPE>::PER_WARP;
}
template <typename T> constexpr size_t diag_smem() {
  return size_t(kWarpsPerBlock) * 3 * kern::Layout<kN>::CPW * kern::Layout<kN>::N3 * sizeof(T);
}

// cudaFuncSetAttribute for the dynamic shared memory, once per device and kernel
template <typename K> void allow_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<int, const void *>> done;
  int dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, reinterpret_cast<const void *>(kernel));
  if (done.count(key)) return;
  PMG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done.insert(key);
}

// Full geometry streams through the shared-memory column ring (TMA) where that measured faster
// on B200 (deformed-cube sweeps at 64^3/128^3): FP64 degrees 1-5 and FP32 degrees 2, 3, 5, 6
// (FP32 Q5 64^3 621 -> 563 us, Q6 1236 -> 1135 us once the ring no longer prefetched into L2);
// FP32 degrees 1 and 4 (whose unrolled forms hide the latency at 8 warps/SM: Q4 128^3 2158
// against 2427 us with the ring) and FP64 degree 6 (2372 against 2488 us) load it directly.
// PMG_VMULT_STAGE=0 / 1 forces direct loads / the ring (a tuning switch; both are compiled).
inline int stage_override() {
  static const int v = [] {
    const char *e = std::getenv("PMG_VMULT_STAGE");
    return e ? std::atoi(e) : -1;
  }();
  return v;
}
template <typename T> bool use_ring() {
  const int o = stage_override();
  if (o == 0 || o == 1) return o == 1;
  return sizeof(T) == 8 ? kN != 7 : (kN != 2 && kN != 5);
}
// gather pipeline (PIPE template parameter); PMG_VMULT_PIPE=0/1/2/3 overrides
inline int pipe_override() {
  static const int v = [] {
    const char *e = std::getenv("PMG_VMULT_PIPE");
    return e ? std::atoi(e) : -1;
  }();
  return v;
}
// Defaults from B200 sweeps (cell kernel time, 48^3..128^3 meshes), for the FP64 ring variant
// without the L2 prefetch: the register pipeline (3) at N = 4 (deformed cube 128^3: Q3 1895 ->
// 1758-1798 us); none at N = 5 (Q4: 3734-3764 us against 3803-3837 us with the register
// pipeline, which was ahead, 4255 -> 4042 us, while the ring variant still prefetched); the
// shared-memory index pipeline (1) at N = 3 (Q2 677 -> 657 us) and N >= 6 (Q5 +18 %; the
// register pipeline there: 1186 -> 1428 us); and the index pipeline for the FP32 Q6 affine
// kernel (+9 %; register pipeline 356 -> 435 us); none elsewhere (FP32 full geometry Q4 with
// the register pipeline 2160 -> 2307 us, with the index pipeline 2415 us; Q4/Q5 affine and
// FP64 Q6 affine lose 15-35 % with the index pipeline).
template <typename T, int GEOM, bool SG> int use_pipe() {
  const int o = pipe_override();
  if (o >= 0 && o <= 3) return o;
  if (SG) return sizeof(T) == 8 ? ((kN >= 6 || kN == 3) ? 1 : (kN == 4 ? 3 : 0)) : 0;
  if ((GEOM == 1 || GEOM == 2) && kN == 7 && sizeof(T) == 4) return 1;
  return 0;
}


// Block shape of a vmult variant on the current device: warps per block and resident warps
// per SM.  The direct variant keeps vmult_wpb(); the ring variant, whose warps share nothing,
// takes the block size (1..8 warps) that fits the most warps per SM -- the per-block
// shared-memory reservation can leave room for one more warp in one large block than in
// one-warp blocks (Q4 FP64: 7 against 6).  PMG_RING_WPB=1..8 fixes it (a tuning switch).
struct VmultShape {
  int wpb = 1, warps_per_sm = 1;
};
inline int ring_wpb_override() {
  static const int v = [] {
    const char *e = std::getenv("PMG_RING_WPB");
    return e ? std::atoi(e) : 0;
  }();
  return v;
}
template <typename T, int GEOM, bool SG, int PIPE> VmultShape vmult_shape() {
  static std::mutex mu;
  static std::map<int, VmultShape> cache; // device -> shape
  int dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  auto k = kern::vmult_slab_kernel<kN, T, GEOM, SG, PIPE>;
  constexpr size_t per_warp = kern::SlabSmem<kN, T, SG, PIPE>::PER_WARP;
  VmultShape best;
  if (!SG) {
    best.wpb = vmult_wpb<T, SG, PIPE>();
    PMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(best.wpb * per_warp)));
    int nb = 0;
    PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * best.wpb, best.wpb * per_warp));
    best.warps_per_sm = std::max(1, nb * best.wpb);
  } else {
    int max_smem = 0;
    PMG_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const int hi = (int)std::min<size_t>(8, std::max<size_t>(1, (size_t)max_smem / per_warp));
    PMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(hi * per_warp)));
    const int o = ring_wpb_override();
    best.warps_per_sm = 0;
    for (int w = 1; w <= hi; ++w) {
      if (o >= 1 && o <= hi && w != o) continue;
      int nb = 0;
      PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * w, w * per_warp));
      if (nb * w > best.warps_per_sm) {
        best.wpb = w;
        best.warps_per_sm = nb * w;
      }
    }
    best.warps_per_sm = std::max(1, best.warps_per_sm);
  }
  cache.emplace(dev, best);
  return best;
}

template <typename T, int GEOM, bool SG, int PIPE> void vmult_launch(const SlabLaunch &L) {
  auto k = kern::vmult_slab_kernel<kN, T, GEOM, SG, PIPE>;
  const VmultShape sh = vmult_shape<T, GEOM, SG, PIPE>();
  int sms = 0, dev = 0;
  PMG_CUDA(cudaGetDevice(&dev));
  PMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t want = (L.n_groups + sh.wpb - 1) / sh.wpb;
  const int64_t resident_blocks = (int64_t)sh.warps_per_sm * sms / sh.wpb;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, resident_blocks));
  const size_t smem = (size_t)sh.wpb * kern::SlabSmem<kN, T, SG, PIPE>::PER_WARP;
  k<<<grid, 32 * sh.wpb, smem, L.stream>>>(
      make_tab<T>(L), static_cast<const T *>(L.src), static_cast<T *>(L.dst), L.idx,
      static_cast<const T *>(L.geo), static_cast<const T *>(L.coef), L.n_groups, L.err);
  PMG_LAUNCH_CHECK();
  if (L.launched) *L.launched = (int64_t)grid * sh.wpb;
}

// The src-staging pipeline (PIPE 2) is built for the direct-load variant only: together with
// the geometry column ring it raised "an illegal instruction was encountered" on B200
// (Q1 FP64, deformed 4^3 mesh) for a cause not found, so that combination is not compiled.
template <typename T, int GEOM, bool SG> void vmult_pipe(const SlabLaunch &L) {
  const int pp = use_pipe<T, GEOM, SG>();
  if constexpr (!SG) {
    if (pp == 2) {
      vmult_launch<T, GEOM, SG, 2>(L);
      return;
    }
  }
  if (pp == 3) vmult_launch<T, GEOM, SG, 3>(L);
  else if (pp >= 1) vmult_launch<T, GEOM, SG, 1>(L);
  else vmult_launch<T, GEOM, SG, 0>(L);
}

template <typename T, int GEOM> void vmult_geom(const SlabLaunch &L) {
  if constexpr (GEOM == 0) {
    if (use_ring<T>()) {
      vmult_pipe<T, GEOM, true>(L);
      return;
    }
  }
  vmult_pipe<T, GEOM, false>(L);
}

template <typename T, int GEOM> void diag_geom(const SlabLaunch &L) {
  auto k = kern::diag_slab_kernel<kN, T, GEOM>;
  allow_smem(k, diag_smem<T>());
  const int64_t want = (L.n_groups + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, L.resident_warps / kWarpsPerBlock));
  k<<<grid, 32 * kWarpsPerBlock, diag_smem<T>(), L.stream>>>(
      make_tab2<T>(L), static_cast<T *>(L.dst), L.idx, static_cast<const T *>(L.geo),
      static_cast<const T *>(L.coef), L.n_groups);
  PMG_LAUNCH_CHECK();
}

template <typename T> void vmult_type(const SlabLaunch &L) {
  if (L.geom == 0) vmult_geom<T, 0>(L);
  else if (L.geom == 1) vmult_geom<T, 1>(L);
  else if (L.geom == 3) vmult_geom<T, 3>(L);
  else vmult_geom<T, 2>(L);
}

template <typename T> void diag_type(const SlabLaunch &L) {
  if (L.geom == 0) diag_geom<T, 0>(L);
  else if (L.geom == 1) diag_geom<T, 1>(L);
  else if (L.geom == 3) diag_geom<T, 3>(L);
  else diag_geom<T, 2>(L);
}

template <typename T, int GEOM, bool SG, int PIPE> int occ_vmult_variant() {
  return vmult_shape<T, GEOM, SG, PIPE>().warps_per_sm; // resident warps per SM
}
// resident warps per SM of the direct variant (low 16 bits) and of the ring variant (high)
template <typename T, int GEOM> int occ_vmult() {
  const int direct = occ_vmult_variant<T, GEOM, false, 0>();
  int ring = direct;
  if constexpr (GEOM == 0) ring = occ_vmult_variant<T, GEOM, true, 0>();
  return direct | (ring << 16);
}
template <typename T, int GEOM> int occ_diag() {
  auto k = kern::diag_slab_kernel<kN, T, GEOM>;
  allow_smem(k, diag_smem<T>());
  int nb = 0;
  PMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * kWarpsPerBlock, diag_smem<T>()));
  return nb * kWarpsPerBlock; // resident warps per SM
}

template <typename T> int occ_vmult_geom(int geom) {
  switch (geom) {
  case 0: return occ_vmult<T, 0>();
  case 1: return occ_vmult<T, 1>();
  case 3: return occ_vmult<T, 3>();
  default: return occ_vmult<T, 2>();
  }
}
template <typename T> int occ_diag_geom(int geom) {
  switch (geom) {
  case 0: return occ_diag<T, 0>();
  case 1: return occ_diag<T, 1>();
  case 3: return occ_diag<T, 3>();
  default: return occ_diag<T, 2>();
  }
}

} // namespace

void PMG_CAT(launch_vmult_p, PMG_DEGREE)(const SlabLaunch &L) {
  if (L.dtype == PMG_F64) vmult_type<double>(L);
  else vmult_type<float>(L);
}

void PMG_CAT(launch_diag_p, PMG_DEGREE)(const SlabLaunch &L) {
  if (L.dtype == PMG_F64) diag_type<double>(L);
  else diag_type<float>(L);
}

int PMG_CAT(occupancy_vmult_p, PMG_DEGREE)(int dtype, int geom) {
  return dtype == PMG_F64 ? occ_vmult_geom<double>(geom) : occ_vmult_geom<float>(geom);
}

int PMG_CAT(occupancy_diag_p, PMG_DEGREE)(int dtype, int geom) {
  return dtype == PMG_F64 ? occ_diag_geom<double>(geom) : occ_diag_geom<float>(geom);
}

} // namespace pmg
