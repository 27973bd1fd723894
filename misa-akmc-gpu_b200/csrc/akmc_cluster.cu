// akmc_cluster.cu -- Cu cluster statistics of a job's resident lattice.
//
// The isolated-Cu count of MEventHook::onStepFinished (profiles/m_event_hook.cpp:17-55: a Cu
// atom none of whose 8 first neighbours is Cu) and the Cu cluster-size histogram by 1nn
// connectivity, on the device, so that a run can sample them every few rounds without
// copying the lattice out.
//
//   k_cu_collect  one pass over the occupancy bytes (16 per thread, vector loads): every Cu
//                 site is appended to a list and starts as its own root.  The only pass over
//                 the whole lattice: HBM-bound.
//   k_cu_union    per listed site (one per thread), its 8 first neighbours are read once: no
//                 Cu among them makes it isolated, and each Cu bond to a higher site id is
//                 merged into one set (lock-free union-find: the larger root is hooked under
//                 the smaller with a CAS, finds halve their paths).
//   k_cu_size     per listed site, +1 on its root's size.
//   k_cu_hist     per root, +1 on the bin of its size (min(size, bins - 1)).
// The partition, hence every count, does not depend on the order the threads run in.
#include <algorithm>
#include <cstdint>

#include "akmc_device.h"

namespace akmc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kCuCode = AKMC_CU;
constexpr int kFindLimit = 1 << 24;   // a find walks at most the set's size; the bound only guards
constexpr int kUnionLimit = 1 << 20;  // CAS retries; each failure means another hook succeeded

__device__ __forceinline__ int64_t nn1_site(int64_t s, int b, int sx, int sy, int sz) {
  const int X = static_cast<int>(s % sx);
  const int64_t t = s / sx;
  const int y = static_cast<int>(t % sy), z = static_cast<int>(t / sy);
  const int p = X & 1;
  int gx = X + ((b & 4) ? 1 : -1);
  int gy = y + ((b >> 1) & 1) - 1 + p;
  int gz = z + (b & 1) - 1 + p;
  gx = gx < 0 ? gx + sx : (gx >= sx ? gx - sx : gx);
  gy = gy < 0 ? gy + sy : (gy >= sy ? gy - sy : gy);
  gz = gz < 0 ? gz + sz : (gz >= sz ? gz - sz : gz);
  return gx + static_cast<int64_t>(sx) * (gy + static_cast<int64_t>(sy) * gz);
}

// Mask with bit 7 of every byte of w that equals the Cu code (exact per byte: no borrow
// crosses a byte boundary).
__device__ __forceinline__ uint32_t cu_bytes(uint32_t w) {
  const uint32_t x = w ^ (0x01010101u * kCuCode);
  return ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu);
}

// Thread t of the grid reads 16 sites of one row (the lattice's halo layout: rows of pitch px,
// the row's sites from entry kHaloL on); the warp takes list slots with one atomic.
__global__ void k_cu_collect(const uint8_t* __restrict__ occ, int64_t ns, int sx, int px, int32_t* list,
                             unsigned int* n_list, int32_t* parent, int32_t* size) {
  const int lane = threadIdx.x & 31;
  const int vpr = (sx + 15) / 16;  // vectors per row
  const int64_t nvec = (ns / sx) * vpr;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w0 = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x - lane); w0 < nvec;
       w0 += warps * 32) {
    const int64_t i = w0 + lane;
    uint32_t m[4] = {0, 0, 0, 0};
    int64_t s0 = 0;
    if (i < nvec) {
      const int64_t row = i / vpr;
      const int k = static_cast<int>(i - row * vpr);
      s0 = row * sx + 16 * k;
      const uint4 w = __ldg(reinterpret_cast<const uint4*>(occ + row * px + kHaloL + 16 * k));
      m[0] = cu_bytes(w.x);
      m[1] = cu_bytes(w.y);
      m[2] = cu_bytes(w.z);
      m[3] = cu_bytes(w.w);
      const int valid = sx - 16 * k;  // the row's last vector reaches into its halo
      if (valid < 16)
        for (int q = 0; q < 4; ++q) {
          const int keep = min(max(valid - 4 * q, 0), 4);
          m[q] &= keep == 4 ? 0xffffffffu : ((1u << (8 * keep)) - 1u);
        }
    }
    const int cnt = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
    int pre = cnt;  // inclusive prefix over the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(kFull, pre, d);
      if (lane >= d) pre += o;
    }
    unsigned int base = 0;
    if (lane == 31 && pre) base = atomicAdd(n_list, static_cast<unsigned int>(pre));
    base = __shfl_sync(kFull, base, 31) + static_cast<unsigned int>(pre - cnt);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint32_t z = m[k];
      while (z) {
        const int64_t s = s0 + k * 4 + ((__ffs(static_cast<int>(z)) - 1) >> 3);
        z &= z - 1;
        parent[s] = static_cast<int32_t>(s);
        size[s] = 0;
        list[base++] = static_cast<int32_t>(s);
      }
    }
  }
}

__device__ __forceinline__ int32_t find_root(int32_t* parent, int32_t x, unsigned int* status) {
  for (int it = 0; it < kFindLimit; ++it) {
    const int32_t p = __ldcg(parent + x);
    if (p == x) return x;
    const int32_t gp = __ldcg(parent + p);
    if (gp != p) atomicCAS(parent + x, p, gp);  // path halving; losing the race is harmless
    x = gp;
  }
  atomicOr(status, kErrTimeout);
  return x;
}

__global__ void k_cu_union(const uint8_t* __restrict__ occ, int sx, int sy, int sz, int px, const int32_t* list,
                           const unsigned int* n_list, int32_t* parent, unsigned long long* iso,
                           unsigned int* status) {
  const int lane = threadIdx.x & 31;
  const int64_t n = *n_list;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  // warp-uniform trip count, so that the warp can sum its isolated atoms
  for (int64_t w0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x - lane; w0 < n; w0 += step) {
    const int64_t i = w0 + lane;
    const int32_t s = i < n ? list[i] : -1;
    unsigned cu = 0;  // bit b: first neighbour b is Cu
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (s >= 0 && __ldg(occ + lattice_index(static_cast<int32_t>(nn1_site(s, b, sx, sy, sz)), sx, px)) == kCuCode)
        cu |= 1u << b;
    const int isolated = __reduce_add_sync(kFull, s >= 0 && cu == 0 ? 1 : 0);
    if (lane == 0 && isolated) atomicAdd(iso, static_cast<unsigned long long>(isolated));
#pragma unroll 1
    for (int b = 0; b < 8; ++b) {
      if (!((cu >> b) & 1u)) continue;
      const int64_t r = nn1_site(s, b, sx, sy, sz);
      if (r <= s) continue;
      int32_t a = s, c = static_cast<int32_t>(r);
      int it = 0;
      for (; it < kUnionLimit; ++it) {
        a = find_root(parent, a, status);
        c = find_root(parent, c, status);
        if (a == c) break;
        if (a < c) {
          const int32_t t = a;
          a = c;
          c = t;
        }
        if (atomicCAS(parent + a, a, c) == a) break;  // root a now hangs under c
      }
      if (it == kUnionLimit) atomicOr(status, kErrTimeout);
    }
  }
}

__global__ void k_cu_size(const int32_t* list, const unsigned int* n_list, int32_t* parent, int32_t* size,
                          unsigned int* status) {
  const int64_t n = *n_list;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    atomicAdd(size + find_root(parent, list[i], status), 1);
}

__global__ void k_cu_hist(const int32_t* list, const unsigned int* n_list, const int32_t* parent,
                          const int32_t* size, unsigned long long* hist, int bins) {
  extern __shared__ unsigned long long h_s[];
  for (int k = threadIdx.x; k < bins; k += blockDim.x) h_s[k] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t n = *n_list;
  // warp-uniform trip count; lanes with the same bin add once through their leader (most
  // clusters are single atoms: one shared bin would otherwise take every atomic)
  for (int64_t w0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x - lane; w0 < n;
       w0 += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = w0 + lane;
    int bin = -1;
    if (i < n) {
      const int32_t s = list[i];
      if (parent[s] == s) bin = min(size[s], bins - 1);
    }
    const unsigned same = __match_any_sync(kFull, bin);
    if (bin >= 0 && lane == __ffs(static_cast<int>(same)) - 1) atomicAdd(h_s + bin, static_cast<unsigned long long>(__popc(same)));
  }
  __syncthreads();
  for (int k = threadIdx.x; k < bins; k += blockDim.x)
    if (h_s[k]) atomicAdd(hist + k, h_s[k]);
}

}  // namespace

int launch_cluster_stats(const ClusterArgs& c, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(c.n_list, 0, sizeof(unsigned int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.iso, 0, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.hist, 0, sizeof(unsigned long long) * c.bins, st);
  if (e != cudaSuccess) return static_cast<int>(e);
  const int64_t nvec = (c.ns / c.sx) * ((c.sx + 15) / 16);
  int grid = static_cast<int>(std::min<int64_t>((nvec + 255) / 256, 148 * 16));
  if (grid < 1) grid = 1;
  k_cu_collect<<<grid, 256, 0, st>>>(c.occ, c.ns, c.sx, c.px, c.list, c.n_list, c.parent, c.size);
  const int g2 = 148 * 8;
  k_cu_union<<<g2, 256, 0, st>>>(c.occ, c.sx, c.sy, c.sz, c.px, c.list, c.n_list, c.parent, c.iso, c.status);
  k_cu_size<<<g2, 256, 0, st>>>(c.list, c.n_list, c.parent, c.size, c.status);
  k_cu_hist<<<g2, 256, sizeof(unsigned long long) * c.bins, st>>>(c.list, c.n_list, c.parent, c.size, c.hist,
                                                                   c.bins);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace akmc
