// Batched layered circuits: thousands of small parameterised circuits of
// uneven width, each layer one 2x2 gate per qubit followed by an optional
// entangler ladder (CX or CZ on (q, q+1) for q = 0..n-2, in that order), run
// to <Z_q> for every qubit of every circuit in ONE persistent launch that is
// captured in a CUDA graph and replayed.
//
// There is no batched path in the reference: each circuit there is a run of
// apply_ops (src/simulator.rs:122-147) on its own StateVector, followed by
// probability_one per qubit (src/measure.rs:43-65). This file computes the
// same quantities, <Z_q> = total - 2 * P(q = 1) with sums in f64, for a whole
// batch at once.
//
// Work distribution: circuits are sorted by cost (largest first) and handed
// out through an atomic counter, so one launch of (SMs x resident CTAs)
// persistent CTAs keeps every SM busy until the batch drains.
//
// A circuit of n <= L qubits lives in shared memory for its whole run (L =
// tile qubits, 12-14, chosen by the autotuner). A wider circuit lives in a
// per-CTA slot in HBM and each layer is two tile passes: pass A over tiles of
// the low L qubits, pass B over tiles of the high n-L qubits plus the low
// r = 2L - n qubits (so rows of 2^r contiguous amplitudes stay coalesced).
//
// Gates are applied in registers, four qubits at a time: a thread loads the
// 16 amplitudes of a subcube, applies the four 2x2 gates, then the part of
// the entangler ladder that lands in those qubits (the ladder's gate into the
// group's first qubit is controlled by a bit outside the subcube, which is
// constant for it, so it becomes a conditional register swap; the ladder
// gates inside the group are register renames). Ladder order is preserved:
// groups run in ascending qubit order and a ladder gate only touches the
// qubits of its own and the previous group.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "batch.hpp"

namespace qvdg {

namespace {

constexpr int kVec = 16;  // >= max tile qubits + 1 (reduction vector)

// Shared-memory position of tile element e: bits 5-7 are folded into bits
// 1-3 so that gate groups above the lowest four bits reach all banks; bit 0
// is kept, so element pairs 2v, 2v+1 stay one 16-byte slot (cp.async).
__device__ __forceinline__ uint32_t swz(uint32_t e) { return e ^ ((e >> 4) & 14u); }

struct TileMap {
  int kind;   // 0: local = global (in-shared circuits and pass A), 1: pass B
  int r;      // pass B: low bits kept in the tile
  int L;      // tile qubits
  uint32_t tile;
  __device__ __forceinline__ uint32_t global(uint32_t e) const {
    if (kind == 0) return (tile << L) | e;
    const uint32_t low = e & ((1u << r) - 1u);
    return low | (tile << r) | ((e >> r) << L);
  }
};

__device__ __forceinline__ float2 cfma2(float2 m0, float2 x0, float2 m1, float2 x1) {
  float2 o;
  o.x = fmaf(m0.x, x0.x, fmaf(-m0.y, x0.y, fmaf(m1.x, x1.x, -m1.y * x1.y)));
  o.y = fmaf(m0.x, x0.y, fmaf(m0.y, x0.x, fmaf(m1.x, x1.y, m1.y * x1.x)));
  return o;
}

// The part of the entangler ladder that lands in the group's G qubits
// (local bits q..q+G-1 of subcube `base`, global qubit of bit q = qglob).
template <int G>
__device__ __forceinline__ void ladder(float2 (&a)[1 << G], int entangler, int qglob, const TileMap& map,
                                       uint32_t base) {
  constexpr int S = 1 << G;
  if (entangler != QVDG_ENTANGLE_NONE) {
    const bool ctrl = qglob > 0 && ((map.global(base) >> (qglob - 1)) & 1u);
    if (entangler == QVDG_ENTANGLE_CX_LADDER) {
      // cx(qglob-1, qglob): flip local bit 0 where the outside control is 1.
#pragma unroll
      for (int j = 0; j < S; j += 2) {
        const float2 t0 = a[j], t1 = a[j + 1];
        a[j] = ctrl ? t1 : t0;
        a[j + 1] = ctrl ? t0 : t1;
      }
      // cx(q+g, q+g+1) inside the group, in ladder order.
#pragma unroll
      for (int g = 0; g + 1 < G; ++g) {
#pragma unroll
        for (int j = 0; j < S; ++j) {
          if (!(j & (1 << g)) || (j & (2 << g))) continue;
          const float2 t = a[j];
          a[j] = a[j | (2 << g)];
          a[j | (2 << g)] = t;
        }
      }
    } else {
#pragma unroll
      for (int j = 1; j < S; j += 2)
        if (ctrl) a[j] = make_float2(-a[j].x, -a[j].y);
#pragma unroll
      for (int g = 0; g + 1 < G; ++g) {
#pragma unroll
        for (int j = 0; j < S; ++j)
          if ((j & (1 << g)) && (j & (2 << g))) a[j] = make_float2(-a[j].x, -a[j].y);
      }
    }
  }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// The same for a phased circuit: each qubit's gate is diag(p) R diag(q)
// with R real, so a group applies its right phases (one complex multiply per
// element from the table `right`, the product of the group's q), the real
// rotations (half the multiply-adds of a complex 2x2) and its left phases.
template <int G>
__device__ void apply_group_phased(float2* __restrict__ tile, int nb, int q, const float2* __restrict__ mats,
                                   const float2* __restrict__ left, const float2* __restrict__ right, uint32_t form,
                                   int entangler, int qglob, const TileMap& map) {
  constexpr int S = 1 << G;
  const uint32_t subcubes = 1u << (nb - G);
  const uint32_t low_mask = (1u << q) - 1u;
  for (uint32_t b = threadIdx.x; b < subcubes; b += blockDim.x) {
    const uint32_t base = ((b & ~low_mask) << G) | (b & low_mask);
    float2 a[S];
#pragma unroll
    for (int j = 0; j < S; ++j) a[j] = tile[swz(base | (uint32_t(j) << q))];
    if (form & kBatchRight)
#pragma unroll
      for (int j = 0; j < S; ++j) a[j] = cmul(a[j], right[j]);
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const float2 r0 = mats[kBatchGateSlots * (q + g) + 0], r1 = mats[kBatchGateSlots * (q + g) + 1];
#pragma unroll
      for (int j = 0; j < S; ++j) {
        if (j & (1 << g)) continue;
        const float2 x0 = a[j], x1 = a[j | (1 << g)];
        a[j] = make_float2(fmaf(r0.x, x0.x, r0.y * x1.x), fmaf(r0.x, x0.y, r0.y * x1.y));
        a[j | (1 << g)] = make_float2(fmaf(r1.x, x0.x, r1.y * x1.x), fmaf(r1.x, x0.y, r1.y * x1.y));
      }
    }
    if (form & kBatchLeft)
#pragma unroll
      for (int j = 0; j < S; ++j) a[j] = cmul(a[j], left[j]);
    ladder<G>(a, entangler, qglob, map, base);
#pragma unroll
    for (int j = 0; j < S; ++j) tile[swz(base | (uint32_t(j) << q))] = a[j];
  }
}

// Apply the gates of local qubits q..q+G-1 (and their ladder part) to every
// subcube of the 2^nb-element tile. `mats` holds a gate record per local
// qubit (m00, m01, m10, m11 first). `qglob` = global qubit of local bit q.
template <int G>
__device__ void apply_group(float2* __restrict__ tile, int nb, int q, const float2* __restrict__ mats,
                            int entangler, int qglob, const TileMap& map) {
  constexpr int S = 1 << G;
  const uint32_t subcubes = 1u << (nb - G);
  const uint32_t low_mask = (1u << q) - 1u;
  for (uint32_t b = threadIdx.x; b < subcubes; b += blockDim.x) {
    const uint32_t base = ((b & ~low_mask) << G) | (b & low_mask);
    float2 a[S];
#pragma unroll
    for (int j = 0; j < S; ++j) a[j] = tile[swz(base | (uint32_t(j) << q))];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const float2 m00 = mats[kBatchGateSlots * (q + g) + 0], m01 = mats[kBatchGateSlots * (q + g) + 1];
      const float2 m10 = mats[kBatchGateSlots * (q + g) + 2], m11 = mats[kBatchGateSlots * (q + g) + 3];
#pragma unroll
      for (int j = 0; j < S; ++j) {
        if (j & (1 << g)) continue;
        const float2 x0 = a[j], x1 = a[j | (1 << g)];
        a[j] = cfma2(m00, x0, m01, x1);
        a[j | (1 << g)] = cfma2(m10, x0, m11, x1);
      }
    }
    ladder<G>(a, entangler, qglob, map, base);
#pragma unroll
    for (int j = 0; j < S; ++j) tile[swz(base | (uint32_t(j) << q))] = a[j];
  }
}

// Gates of local qubits [q0, q1) in register groups of up to four qubits,
// ascending, the range split as evenly as possible (13 qubits: 4 + 3 + 3 +
// 3); each group costs one shared-memory round trip of the tile (groups of
// five spill registers at 512 threads). For a phased circuit the groups'
// phase tables (products of the members' left and right phases over the 2^G
// elements of a subcube) go to `tabs` first.
constexpr int kMaxGroup = 4;

template <bool PHASED>
__device__ __forceinline__ void apply_one(int G, float2* tile, int nb, int q, const float2* mats, const float2* l,
                                          const float2* r, uint32_t form, int entangler, int qg, const TileMap& map) {
  if constexpr (PHASED) {
    switch (G) {
      case 4: return apply_group_phased<4>(tile, nb, q, mats, l, r, form, entangler, qg, map);
      case 3: return apply_group_phased<3>(tile, nb, q, mats, l, r, form, entangler, qg, map);
      case 2: return apply_group_phased<2>(tile, nb, q, mats, l, r, form, entangler, qg, map);
      default: return apply_group_phased<1>(tile, nb, q, mats, l, r, form, entangler, qg, map);
    }
  } else {
    switch (G) {
      case 4: return apply_group<4>(tile, nb, q, mats, entangler, qg, map);
      case 3: return apply_group<3>(tile, nb, q, mats, entangler, qg, map);
      case 2: return apply_group<2>(tile, nb, q, mats, entangler, qg, map);
      default: return apply_group<1>(tile, nb, q, mats, entangler, qg, map);
    }
  }
}

__device__ void apply_range(float2* tile, int nb, int q0, int q1, const float2* mats, uint32_t form, int entangler,
                            int qglob0, const TileMap& map, float2 (*tabs)[1 << kMaxGroup]) {
  const int m = q1 - q0;
  if (m <= 0) return;
  const bool phased = (form & kBatchPhased) != 0;
  const int groups = (m + kMaxGroup - 1) / kMaxGroup, small = m / groups, extra = m % groups;
  auto start = [&](int gi) { return q0 + gi * small + min(gi, extra); };
  auto size = [&](int gi) { return small + (gi < extra ? 1 : 0); };
  if (phased) {
    for (int i = threadIdx.x; i < groups << kMaxGroup; i += blockDim.x) {
      const int gi = i >> kMaxGroup, j = i & ((1 << kMaxGroup) - 1), q = start(gi), G = size(gi);
      if (j >= (1 << G)) continue;
      float2 l = make_float2(1.f, 0.f), r = make_float2(1.f, 0.f);
      for (int b = 0; b < G; ++b) {
        const float2* rec = mats + kBatchGateSlots * (q + b);
        const int bit = (j >> b) & 1;
        l = cmul(l, rec[2 + bit]);
        r = cmul(r, rec[4 + bit]);
      }
      tabs[2 * gi][j] = l;
      tabs[2 * gi + 1][j] = r;
    }
    __syncthreads();
  }
  for (int gi = 0; gi < groups; ++gi) {
    const int q = start(gi), qg = qglob0 + (q - q0);
    if (phased)
      apply_one<true>(size(gi), tile, nb, q, mats, tabs[2 * gi], tabs[2 * gi + 1], form, entangler, qg, map);
    else
      apply_one<false>(size(gi), tile, nb, q, mats, nullptr, nullptr, form, entangler, qg, map);
    __syncthreads();
  }
}

// Deterministic block sum of kVec doubles per thread into out[0..kVec)
// (valid in every thread after the call).
__device__ void block_sum_vec(double (&v)[kVec], double* red /* [32 * kVec] */, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < kVec; ++i) {
    double x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    v[i] = x;
  }
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < kVec; ++i) red[warp * kVec + i] = v[i];
  __syncthreads();
  if (threadIdx.x < kVec) {
    double t = 0.0;
    for (int w = 0; w < warps; ++w) t += red[w * kVec + threadIdx.x];
    out[threadIdx.x] = t;
  }
  __syncthreads();
}

// Adds the tile's probability sums to the CTA's per-qubit accumulators
// acc[0] = total, acc[1 + q] = sum over global index bit q set. Thread i
// visits elements i, i + T, i + 2T, ...: the local bits below log2(T) are
// fixed per thread and the others vary.
__device__ void reduce_tile(const float2* tile, int nb, const TileMap& map, int n, double* red, double* tmp,
                            double* acc) {
  double v[kVec];
#pragma unroll
  for (int i = 0; i < kVec; ++i) v[i] = 0.0;
  const uint32_t count = 1u << nb;
  const int tbits = 31 - __clz(blockDim.x);
  for (uint32_t e = threadIdx.x; e < count; e += blockDim.x) {
    const float2 a = tile[swz(e)];
    const double p = __dadd_rn(__dmul_rn(double(a.x), double(a.x)), __dmul_rn(double(a.y), double(a.y)));
    v[0] += p;
#pragma unroll
    for (int bit = 0; bit < kVec - 1; ++bit)
      if (bit >= tbits && bit < nb && ((e >> bit) & 1u)) v[1 + bit] += p;
  }
#pragma unroll
  for (int bit = 0; bit < kVec - 1; ++bit)
    if (bit < tbits && bit < nb && ((threadIdx.x >> bit) & 1u)) v[1 + bit] = v[0];
  block_sum_vec(v, red, tmp);
  if (threadIdx.x == 0) {
    // Local bit -> global qubit; the tile's fixed bits take the whole total.
    const uint32_t g0 = map.global(0);
    uint32_t local_global = 0;
    for (int bit = 0; bit < nb; ++bit) {
      const uint32_t gq = 31 - __clz(map.global(1u << bit) ^ g0);
      local_global |= 1u << gq;
      acc[1 + gq] += tmp[1 + bit];
    }
    for (int q = 0; q < n; ++q)
      if (!((local_global >> q) & 1u) && ((g0 >> q) & 1u)) acc[1 + q] += tmp[0];
    acc[0] += tmp[0];
  }
  __syncthreads();
}

// Tile <-> slot copies in 16-byte units (element pairs 2u, 2u+1: adjacent in
// the slot because every tile keeps global bit 0, and one aligned slot in
// shared memory because swz keeps bit 0).
__device__ __forceinline__ float4 get_pair(const float2* tile, uint32_t e) {
  return *reinterpret_cast<const float4*>(tile + swz(e));
}

// The tile's 16-byte copies issued asynchronously (cp.async) into `tile`,
// as one commit group.
__device__ void issue_tile(float2* tile, const float2* __restrict__ slot, const TileMap& map) {
  const uint32_t units = 1u << (map.L - 1);
  for (uint32_t u = threadIdx.x; u < units; u += blockDim.x) {
    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(tile + swz(2 * u)));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(slot + map.global(2 * u)) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void commit_empty() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ void store_tile(const float2* tile, float2* __restrict__ slot, const TileMap& map) {
  const uint32_t units = 1u << (map.L - 1);
  for (uint32_t u = threadIdx.x; u < units; u += blockDim.x)
    __stcs(reinterpret_cast<float4*>(slot + map.global(2 * u)), get_pair(tile, 2 * u));
}

__device__ void load_mats(float2* smem_mats, const float2* gates, int first_global, int count, int local0) {
  for (int i = threadIdx.x; i < kBatchGateSlots * count; i += blockDim.x)
    smem_mats[kBatchGateSlots * local0 + i] = gates[kBatchGateSlots * first_global + i];
}

__global__ void __launch_bounds__(512) k_batch(const BatchCircuit* __restrict__ circuits,
                                               const uint32_t* __restrict__ order, uint32_t count,
                                               const float2* __restrict__ gates, float2* __restrict__ slots,
                                               uint64_t slot_elems, double* __restrict__ out,
                                               uint32_t* __restrict__ queue, int L) {
  extern __shared__ float2 tile[];
  __shared__ float2 mats[kBatchGateSlots * kBatchMaxQubits];
  __shared__ float2 tabs[8][1 << kMaxGroup];  // phase tables of up to four groups (left, right)
  __shared__ double red[32 * kVec];
  __shared__ double tmp[kVec];
  __shared__ double acc[1 + kBatchMaxQubits];
  __shared__ uint32_t item;
  float2* slot = slots + uint64_t(blockIdx.x) * slot_elems;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t it = item;
    if (it >= count) break;
    const BatchCircuit c = circuits[order[it]];
    const int n = int(c.num_qubits);
    if (threadIdx.x <= kBatchMaxQubits) acc[threadIdx.x] = 0.0;
    if (n <= L) {
      // Whole state in shared memory.
      const uint32_t size = 1u << n;
      for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) tile[swz(e)] = make_float2(e == 0 ? 1.f : 0.f, 0.f);
      const TileMap map{0, 0, L, 0};
      for (uint32_t l = 0; l < c.num_layers; ++l) {
        __syncthreads();
        load_mats(mats, gates + kBatchGateSlots * c.gates, int(l) * n, n, 0);
        __syncthreads();
        apply_range(tile, n, 0, n, mats, c.form, int(c.entangler), 0, map, tabs);
      }
      __syncthreads();
      reduce_tile(tile, n, map, n, red, tmp, acc);
    } else {
      // Two tile passes per layer over the slot in HBM, on tiles of
      // Lw = L - 1 qubits: the CTA's shared tile holds two of them, so the
      // next tile's copies fly (cp.async) while the current one is computed.
      const int Lw = L - 1;
      const int r = 2 * Lw - n;
      const uint32_t tiles = 1u << (n - Lw);
      const uint32_t tsize = 1u << Lw;
      float2* buf[2] = {tile, tile + tsize};
      for (uint32_t l = 0; l < c.num_layers; ++l) {
        const bool last = l + 1 == c.num_layers;
        __syncthreads();
        load_mats(mats, gates + kBatchGateSlots * c.gates, int(l) * n, n, 0);
        __syncthreads();
        // pass A: low Lw qubits
        if (l > 0) issue_tile(buf[0], slot, TileMap{0, 0, Lw, 0});
        for (uint32_t t = 0; t < tiles; ++t) {
          const TileMap map{0, 0, Lw, t};
          float2* cur = (t & 1u) ? buf[1] : buf[0];
          if (l == 0) {
            for (uint32_t e = threadIdx.x; e < tsize; e += blockDim.x)
              cur[swz(e)] = make_float2((t == 0 && e == 0) ? 1.f : 0.f, 0.f);
          } else {
            if (t + 1 < tiles)
              issue_tile((t & 1u) ? buf[0] : buf[1], slot, TileMap{0, 0, Lw, t + 1});
            else
              commit_empty();
            wait_prev();
          }
          __syncthreads();
          apply_range(cur, Lw, 0, Lw, mats, c.form, int(c.entangler), 0, map, tabs);
          store_tile(cur, slot, map);
          __threadfence_block();
          __syncthreads();
        }
        // pass B: high n-Lw qubits (reads what pass A stored, after the barrier)
        issue_tile(buf[0], slot, TileMap{1, r, Lw, 0});
        for (uint32_t t = 0; t < tiles; ++t) {
          const TileMap map{1, r, Lw, t};
          float2* cur = (t & 1u) ? buf[1] : buf[0];
          if (t + 1 < tiles)
            issue_tile((t & 1u) ? buf[0] : buf[1], slot, TileMap{1, r, Lw, t + 1});
          else
            commit_empty();
          wait_prev();
          __syncthreads();
          // Local bits r..Lw-1 are global qubits Lw..n-1 (matrices at local index).
          apply_range(cur, Lw, r, Lw, mats + kBatchGateSlots * (Lw - r), c.form, int(c.entangler), Lw, map, tabs);
          if (last) {
            reduce_tile(cur, Lw, map, n, red, tmp, acc);
          } else {
            store_tile(cur, slot, map);
            __threadfence_block();
            __syncthreads();
          }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
    }
    if (threadIdx.x < uint32_t(n)) out[c.out + threadIdx.x] = acc[0] - 2.0 * acc[1 + threadIdx.x];
    __syncthreads();
  }
}

}  // namespace

int batch_kernel_occupancy(int threads, int tile_qubits) {
  int blocks = 0;
  const size_t smem = sizeof(float2) << tile_qubits;
  // Allow the largest tile once, so that launches (also under stream
  // capture) need no attribute change.
  if (cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(float2) << 14)) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_batch, cudaFuncAttributePreferredSharedMemoryCarveout,
                           int(cudaSharedmemCarveoutMaxShared)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_batch, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return blocks;
}

void launch_batch(const BatchLaunch& b, cudaStream_t stream) {
  const size_t smem = sizeof(float2) << b.tile_qubits;
  QVDG_CUDA(cudaMemsetAsync(b.queue, 0, sizeof(uint32_t), stream));
  k_batch<<<b.ctas, b.threads, smem, stream>>>(b.circuits, b.order, b.count, b.gates, b.slots, b.slot_elems, b.out,
                                               b.queue, b.tile_qubits);
  QVDG_LAUNCH_CHECK();
}

}  // namespace qvdg
