// Stable LSD radix sort of 64-bit keys (8-bit digits, 8 passes).
//
// Used by the sampler to sort its targets (the reference sorts them with
// rayon's par_sort_unstable_by(f64::total_cmp), src/measure.rs:125-126; the
// keys here are the doubles' total-order bit patterns, so equal keys are
// equal doubles and stability does not change the result).
//
// Per pass: per-tile digit histograms, one exclusive scan over them in
// digit-major order, then a stable scatter in which each warp ranks equal
// digits with __match_any_sync and warps are combined through shared memory.

#include <cuda_runtime.h>

#include "engine.hpp"

namespace qvdg {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTile = 4096;  // keys per tile
constexpr int kRounds = kTile / kThreads;

__global__ void __launch_bounds__(kThreads) k_hist(const uint64_t* __restrict__ keys, size_t n, int shift,
                                                   uint32_t* __restrict__ hist, uint32_t tiles) {
  __shared__ uint32_t counts[256];
  counts[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = size_t(blockIdx.x) * kTile;
  for (int r = 0; r < kRounds; ++r) {
    const size_t i = base + size_t(r) * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&counts[(keys[i] >> shift) & 255], 1u);
  }
  __syncthreads();
  hist[size_t(threadIdx.x) * tiles + blockIdx.x] = counts[threadIdx.x];
}

// Exclusive scan of `count` values in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan(uint32_t* __restrict__ v, size_t count) {
  __shared__ uint32_t part[1024];
  const size_t per = (count + 1023) / 1024;
  const size_t first = size_t(threadIdx.x) * per;
  uint32_t sum = 0;
  for (size_t i = first; i < first + per && i < count; ++i) sum += v[i];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const uint32_t add = threadIdx.x >= unsigned(o) ? part[threadIdx.x - o] : 0u;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - sum;  // exclusive prefix of this segment
  for (size_t i = first; i < first + per && i < count; ++i) {
    const uint32_t x = v[i];
    v[i] = run;
    run += x;
  }
}

__global__ void __launch_bounds__(kThreads) k_scatter(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                                      size_t n, int shift, const uint32_t* __restrict__ hist,
                                                      uint32_t tiles) {
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcount[kWarps][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base[threadIdx.x] = hist[size_t(threadIdx.x) * tiles + blockIdx.x];
  const size_t tile = size_t(blockIdx.x) * kTile;
  const unsigned lt = (1u << lane) - 1u;
  for (int r = 0; r < kRounds; ++r) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) wcount[w][threadIdx.x] = 0;
    __syncthreads();
    const size_t i = tile + size_t(r) * kThreads + threadIdx.x;
    const bool valid = i < n;
    const uint64_t key = valid ? in[i] : 0;
    const uint32_t d = valid ? uint32_t((key >> shift) & 255) : 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lt);
    if (valid && rank == 0) wcount[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t off = base[d] + rank;
      for (int w = 0; w < warp; ++w) off += wcount[w][d];
      out[off] = key;
    }
    __syncthreads();
    uint32_t add = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) add += wcount[w][threadIdx.x];
    base[threadIdx.x] += add;
    __syncthreads();
  }
}

}  // namespace

void radix_sort_u64(uint64_t* keys, uint64_t* tmp, size_t count, DeviceScratch& work, cudaStream_t stream) {
  if (count <= 1) return;
  if (count > size_t(0xFFFFFFFFu)) throw Error(1, "too many keys to sort");
  const uint32_t tiles = uint32_t((count + kTile - 1) / kTile);
  uint32_t* hist = static_cast<uint32_t*>(work.get(size_t(256) * tiles * sizeof(uint32_t)));
  uint64_t* src = keys;
  uint64_t* dst = tmp;
  for (int shift = 0; shift < 64; shift += 8) {
    k_hist<<<tiles, kThreads, 0, stream>>>(src, count, shift, hist, tiles);
    QVDG_LAUNCH_CHECK();
    k_scan<<<1, 1024, 0, stream>>>(hist, size_t(256) * tiles);
    QVDG_LAUNCH_CHECK();
    k_scatter<<<tiles, kThreads, 0, stream>>>(src, dst, count, shift, hist, tiles);
    QVDG_LAUNCH_CHECK();
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  // Eight passes: the sorted keys are back in `keys`.
}

}  // namespace qvdg
