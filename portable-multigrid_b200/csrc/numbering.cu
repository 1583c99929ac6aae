// DoF numbering, index maps and transfer maps built on the device (setup).
//
// The numbering visits the cells in the box's order (coarse cells lexicographically, Morton
// order inside each) and the nodes of a cell in lexicographic order, and numbers every node
// when it is first visited, so that the DoFs a batch of consecutive cells touches are close
// together in memory.  In parallel: node X's
// number is the rank of (first cell containing X, X's local index in that cell) among all
// nodes, so with cnt[c] = the nodes first visited by cell c, an exclusive scan of cnt gives
// each cell the first number of its new nodes, and the cell numbers them in local order.
// The reference builds its index maps on the host from deal.II's DoFHandler
// (include/operators/portable_laplace_operator_bk3.h:360-437) and its transfer maps and
// weights in host loops (include/multigrid/portable_polynomial_transfer.h:1116-1361).
#include <algorithm>

#include "numbering.hpp"

namespace pmg {
namespace {

constexpr int kScanBlock = 1024;

struct BoxDims {
  int64_t n[3];     // cells per direction
  int64_t L[3];     // lattice points per direction (p n + 1)
  int32_t coarse[3];
  int refine, p, nm;
  int mask;         // Dirichlet faces
};

// index of cell (cx, cy, cz) in the box's cell order
__device__ __forceinline__ int64_t cell_index(const BoxDims &b, int64_t cx, int64_t cy, int64_t cz) {
  const int L = b.refine;
  const int64_t tile = ((cz >> L) * b.coarse[1] + (cy >> L)) * b.coarse[0] + (cx >> L);
  const int64_t m = (int64_t(1) << L) - 1;
  const int64_t x = cx & m, y = cy & m, z = cz & m;
  int64_t code = 0;
  for (int bit = 0; bit < L; ++bit)
    code |= (((x >> bit) & 1) << (3 * bit)) | (((y >> bit) & 1) << (3 * bit + 1)) | (((z >> bit) & 1) << (3 * bit + 2));
  return (tile << (3 * L)) + code;
}

// the first cell (in cell order) that contains lattice point g
__device__ __forceinline__ int64_t first_cell(const BoxDims &b, const int64_t g[3]) {
  int64_t lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    const int64_t q = g[d] / b.p;
    hi[d] = q < b.n[d] - 1 ? q : b.n[d] - 1;
    lo[d] = (g[d] % b.p == 0 && g[d] > 0) ? q - 1 : q;
    if (lo[d] > hi[d]) lo[d] = hi[d];
  }
  int64_t best = INT64_MAX;
  for (int64_t z = lo[2]; z <= hi[2]; ++z)
    for (int64_t y = lo[1]; y <= hi[1]; ++y)
      for (int64_t x = lo[0]; x <= hi[0]; ++x) {
        const int64_t c = cell_index(b, x, y, z);
        best = c < best ? c : best;
      }
  return best;
}

__device__ __forceinline__ bool on_dirichlet(const BoxDims &b, const int64_t g[3]) {
  return ((b.mask & 1) && g[0] == 0) || ((b.mask & 2) && g[0] == b.L[0] - 1) || ((b.mask & 4) && g[1] == 0) ||
         ((b.mask & 8) && g[1] == b.L[1] - 1) || ((b.mask & 16) && g[2] == 0) || ((b.mask & 32) && g[2] == b.L[2] - 1);
}

// cnt[c] = the nodes cell c visits first
__global__ void count_new_nodes_kernel(const BoxDims b, const int32_t *__restrict__ cell_xyz, int64_t n_cells,
                                       uint32_t *__restrict__ cnt) {
  const int nm = b.nm;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t base[3] = {int64_t(b.p) * cell_xyz[3 * c], int64_t(b.p) * cell_xyz[3 * c + 1],
                             int64_t(b.p) * cell_xyz[3 * c + 2]};
    uint32_t k_new = 0;
    for (int k = 0; k < nm; ++k)
      for (int j = 0; j < nm; ++j)
        for (int i = 0; i < nm; ++i) {
          const int64_t g[3] = {base[0] + i, base[1] + j, base[2] + k};
          k_new += first_cell(b, g) == c;
        }
    cnt[c] = k_new;
  }
}

// cell c numbers its new nodes from off[c] on, in local order; lattice, plain (for its new
// nodes) and the constrained flags are written
__global__ void assign_numbers_kernel(const BoxDims b, const int32_t *__restrict__ cell_xyz, int64_t n_cells,
                                      const uint32_t *__restrict__ off, uint32_t *__restrict__ lattice,
                                      uint8_t *__restrict__ cons) {
  const int nm = b.nm;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n_cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t base[3] = {int64_t(b.p) * cell_xyz[3 * c], int64_t(b.p) * cell_xyz[3 * c + 1],
                             int64_t(b.p) * cell_xyz[3 * c + 2]};
    uint32_t r = off[c];
    for (int k = 0; k < nm; ++k)
      for (int j = 0; j < nm; ++j)
        for (int i = 0; i < nm; ++i) {
          const int64_t g[3] = {base[0] + i, base[1] + j, base[2] + k};
          if (first_cell(b, g) != c) continue;
          lattice[(g[2] * b.L[1] + g[1]) * b.L[0] + g[0]] = r;
          cons[r] = on_dirichlet(b, g) ? 1 : 0;
          ++r;
        }
  }
}

// plain[c][l] = the number of node l of cell c
__global__ void gather_plain_kernel(const BoxDims b, const int32_t *__restrict__ cell_xyz, int64_t n_cells,
                                    const uint32_t *__restrict__ lattice, uint32_t *__restrict__ plain) {
  const int nm = b.nm, nm3 = nm * nm * nm;
  const int64_t total = n_cells * nm3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / nm3;
    const int l = (int)(t - c * nm3);
    const int i = l % nm, j = (l / nm) % nm, k = l / (nm * nm);
    const int64_t gx = int64_t(b.p) * cell_xyz[3 * c] + i, gy = int64_t(b.p) * cell_xyz[3 * c + 1] + j,
                  gz = int64_t(b.p) * cell_xyz[3 * c + 2] + k;
    plain[t] = lattice[(gz * b.L[1] + gy) * b.L[0] + gx];
  }
}

// ---- deterministic exclusive scan of uint32 counts (three passes) ----
__global__ void scan_block_sums_kernel(const uint32_t *__restrict__ in, int64_t n, uint32_t *__restrict__ sums) {
  __shared__ uint32_t s[kScanBlock];
  const int64_t i = int64_t(blockIdx.x) * kScanBlock + threadIdx.x;
  s[threadIdx.x] = i < n ? in[i] : 0u;
  __syncthreads();
  for (int w = kScanBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = s[0];
}

// exclusive scan of the block sums in one block, chunk by chunk
__global__ void scan_sums_kernel(uint32_t *__restrict__ sums, int64_t n_blocks) {
  __shared__ uint32_t s[kScanBlock];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n_blocks; base += kScanBlock) {
    const int64_t i = base + threadIdx.x;
    const uint32_t v = i < n_blocks ? sums[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) { // inclusive Hillis-Steele
      const uint32_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
      __syncthreads();
      s[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < n_blocks) sums[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry += s[kScanBlock - 1];
    __syncthreads();
  }
}

__global__ void scan_apply_kernel(const uint32_t *__restrict__ in, int64_t n, const uint32_t *__restrict__ sums,
                                  uint32_t *__restrict__ out) {
  __shared__ uint32_t s[kScanBlock];
  const int64_t i = int64_t(blockIdx.x) * kScanBlock + threadIdx.x;
  const uint32_t v = i < n ? in[i] : 0u;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < kScanBlock; off <<= 1) {
    const uint32_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
    __syncthreads();
    s[threadIdx.x] += add;
    __syncthreads();
  }
  if (i < n) out[i] = sums[blockIdx.x] + s[threadIdx.x] - v;
}

__global__ void flags_to_u32_kernel(const uint8_t *__restrict__ f, int64_t n, uint32_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = f[i] ? 1u : 0u;
}

// list[pos[i]] = i where f[i] (pos: exclusive scan of the flags), and the bitmask
__global__ void compact_flags_kernel(const uint8_t *__restrict__ f, const uint32_t *__restrict__ pos, int64_t n,
                                     uint32_t *__restrict__ list, uint32_t *__restrict__ bits) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (f[i]) {
      list[pos[i]] = (uint32_t)i;
      atomicOr(bits + (i >> 5), 1u << (i & 31));
    }
}

// the slab layout of the index map: [group][k*N+i][e*N+j], sentinel on constrained DoFs
__global__ void slab_index_kernel(const uint32_t *__restrict__ plain, const uint8_t *__restrict__ cons,
                                  int64_t n_cells, int N, int cpw, int lanes, uint32_t *__restrict__ idx) {
  const int N2 = N * N, N3 = N2 * N;
  const int64_t total = n_cells * N3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / N3;
    const int l = (int)(t - c * N3);
    const int i = l % N, j = (l / N) % N, k = l / N2;
    const uint32_t d = plain[t];
    const int64_t grp = c / cpw;
    const int e = (int)(c - grp * cpw);
    idx[(grp * N2 + k * N + i) * lanes + e * N + j] = (d == kInvalid || cons[d]) ? kInvalid : d;
  }
}

int grid_for(int64_t n, int sms, int threads = 256) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, (int64_t)sms * 32));
}

} // namespace

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  const int64_t n_blocks = (n + kScanBlock - 1) / kScanBlock;
  DeviceBuffer sums(sizeof(uint32_t) * n_blocks);
  scan_block_sums_kernel<<<(unsigned)n_blocks, kScanBlock, 0, s>>>(in, n, sums.as<uint32_t>());
  PMG_LAUNCH_CHECK();
  scan_sums_kernel<<<1, kScanBlock, 0, s>>>(sums.as<uint32_t>(), n_blocks);
  PMG_LAUNCH_CHECK();
  scan_apply_kernel<<<(unsigned)n_blocks, kScanBlock, 0, s>>>(in, n, sums.as<uint32_t>(), out);
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaStreamSynchronize(s)); // sums is freed on return
}

void device_numbering(const BoxMesh &m, int p, const DeviceBuffer &cell_xyz, int sms, DeviceNumbering &out,
                      cudaStream_t s) {
  BoxDims b{};
  for (int d = 0; d < 3; ++d) {
    b.n[d] = m.n[d];
    b.L[d] = p * m.n[d] + 1;
    b.coarse[d] = m.box.coarse[d];
  }
  b.refine = m.box.refine;
  b.p = p;
  b.nm = p + 1;
  b.mask = m.box.dirichlet_mask;
  const int64_t C = m.n_cells, nm3 = int64_t(p + 1) * (p + 1) * (p + 1);
  const int64_t n_lat = b.L[0] * b.L[1] * b.L[2];
  PMG_REQUIRE(n_lat < (int64_t(1) << 32) - 1, "too many DoFs for 32-bit indices");
  out.p = p;
  out.n_dofs = n_lat; // every lattice point is a DoF of a box mesh
  for (int d = 0; d < 3; ++d) out.L[d] = b.L[d];
  out.lattice.allocate(sizeof(uint32_t) * n_lat);
  out.plain.allocate(sizeof(uint32_t) * std::max<int64_t>(1, C * nm3));
  out.constrained.allocate(std::max<int64_t>(1, n_lat));
  if (C == 0) return;
  DeviceBuffer cnt(sizeof(uint32_t) * C), off(sizeof(uint32_t) * C);
  count_new_nodes_kernel<<<grid_for(C, sms, 128), 128, 0, s>>>(b, cell_xyz.as<int32_t>(), C, cnt.as<uint32_t>());
  PMG_LAUNCH_CHECK();
  exclusive_scan_u32(cnt.as<uint32_t>(), off.as<uint32_t>(), C, s);
  assign_numbers_kernel<<<grid_for(C, sms, 128), 128, 0, s>>>(b, cell_xyz.as<int32_t>(), C, off.as<uint32_t>(),
                                                              out.lattice.as<uint32_t>(), out.constrained.as<uint8_t>());
  PMG_LAUNCH_CHECK();
  gather_plain_kernel<<<grid_for(C * nm3, sms), 256, 0, s>>>(b, cell_xyz.as<int32_t>(), C, out.lattice.as<uint32_t>(),
                                                             out.plain.as<uint32_t>());
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaStreamSynchronize(s)); // cnt and off are freed on return
}

void device_constrained(const uint8_t *cons, int64_t n, int sms, DeviceBuffer &list, DeviceBuffer &bits,
                        int64_t &n_constrained, cudaStream_t s) {
  bits.allocate(sizeof(uint32_t) * std::max<int64_t>(1, (n + 31) / 32));
  PMG_CUDA(cudaMemsetAsync(bits.get(), 0, bits.bytes(), s));
  n_constrained = 0;
  if (n == 0) {
    list.allocate(sizeof(uint32_t));
    return;
  }
  DeviceBuffer f32(sizeof(uint32_t) * n), pos(sizeof(uint32_t) * n);
  flags_to_u32_kernel<<<grid_for(n, sms), 256, 0, s>>>(cons, n, f32.as<uint32_t>());
  PMG_LAUNCH_CHECK();
  exclusive_scan_u32(f32.as<uint32_t>(), pos.as<uint32_t>(), n, s);
  uint32_t last_pos = 0, last_flag = 0;
  PMG_CUDA(cudaMemcpy(&last_pos, pos.as<uint32_t>() + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  PMG_CUDA(cudaMemcpy(&last_flag, f32.as<uint32_t>() + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  n_constrained = int64_t(last_pos) + last_flag;
  list.allocate(sizeof(uint32_t) * std::max<int64_t>(1, n_constrained));
  compact_flags_kernel<<<grid_for(n, sms), 256, 0, s>>>(cons, pos.as<uint32_t>(), n, list.as<uint32_t>(),
                                                         bits.as<uint32_t>());
  PMG_LAUNCH_CHECK();
  PMG_CUDA(cudaStreamSynchronize(s));
}

void device_slab_index(const uint32_t *plain, const uint8_t *cons, int64_t n_cells, int N, int cpw, int lanes,
                       int64_t n_groups, int sms, DeviceBuffer &idx, cudaStream_t s) {
  const int64_t n_idx = n_groups * N * N * lanes;
  idx.allocate(sizeof(uint32_t) * std::max<int64_t>(1, n_idx));
  PMG_CUDA(cudaMemsetAsync(idx.get(), 0xFF, idx.bytes(), s));
  const int64_t total = n_cells * N * N * N;
  if (total > 0) {
    slab_index_kernel<<<grid_for(total, sms), 256, 0, s>>>(plain, cons, n_cells, N, cpw, lanes, idx.as<uint32_t>());
    PMG_LAUNCH_CHECK();
  }
}

} // namespace pmg
