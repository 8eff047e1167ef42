// Gate application on a shared-memory tile (CUDA cores), shared by the
// staged kernels. A tile holds 2^L amplitudes indexed by tile-local bits.
#pragma once

#include "common.cuh"
#include "stage_kernel.hpp"

namespace qvdg {

__device__ __forceinline__ uint32_t insert_zeros32(uint32_t x, const uint8_t* pos, int count) {
  for (int i = 0; i < count; ++i) {
    const uint32_t p = pos[i];
    x = ((x >> p) << (p + 1)) | (x & ((1u << p) - 1u));
  }
  return x;
}

// Tile-local offset of group member h (matrix index bit j -> tgt[j]).
template <int K>
__device__ __forceinline__ uint32_t member(uint32_t h, const uint8_t* tgt) {
  uint32_t o = 0;
#pragma unroll
  for (int j = 0; j < K; ++j) o |= ((h >> j) & 1u) << tgt[j];
  return o;
}

// Dense gate with K <= 4: one thread per group, the group in registers,
// matrix entries read as warp-wide broadcasts.
template <typename T, int K>
__device__ __forceinline__ void tile_dense(cplx_t<T>* tile, int L, const TileGate& g,
                                           const cplx_t<T>* __restrict__ m) {
  constexpr int D = 1 << K;
  uint8_t tgt[K];
#pragma unroll
  for (int j = 0; j < K; ++j) tgt[j] = g.tgt[j];
  uint32_t off[D];
#pragma unroll
  for (int h = 0; h < D; ++h) off[h] = member<K>(h, tgt);
  const uint32_t groups = 1u << (L - g.nfixed);
  for (uint32_t gi = threadIdx.x; gi < groups; gi += blockDim.x) {
    const uint32_t b = insert_zeros32(gi, g.fixed, g.nfixed) | g.lcv;
    cplx_t<T> x[D];
#pragma unroll
    for (int h = 0; h < D; ++h) x[h] = tile[b | off[h]];
#pragma unroll 1
    for (int r = 0; r < D; ++r) {
      cplx_t<T> acc = make_c<T>(T(0), T(0));
#pragma unroll
      for (int c = 0; c < D; ++c) cmac<T>(acc, __ldg(&m[r * D + c]), x[c]);
      tile[b | off[r]] = acc;
    }
  }
}

// Dense gate with K = 5, 6: D threads per group, one output row each; the
// matrix is stored transposed so a warp's row entries are contiguous.
template <typename T, int K>
__device__ __forceinline__ void tile_dense_rows(cplx_t<T>* tile, int L, const TileGate& g,
                                                const cplx_t<T>* __restrict__ mt) {
  constexpr int D = 1 << K;
  const uint32_t groups = 1u << (L - g.nfixed);
  const uint32_t per_wave = blockDim.x / D;
  const uint32_t r = threadIdx.x % D, slot = threadIdx.x / D;
  const uint32_t out_off = member<K>(r, g.tgt);
  for (uint32_t g0 = 0; g0 < groups; g0 += per_wave) {
    const uint32_t gi = g0 + slot;
    const bool active = gi < groups;
    cplx_t<T> acc = make_c<T>(T(0), T(0));
    uint32_t b = 0;
    if (active) {
      b = insert_zeros32(gi, g.fixed, g.nfixed) | g.lcv;
#pragma unroll 8
      for (int c = 0; c < D; ++c) cmac<T>(acc, __ldg(&mt[c * D + r]), tile[b | member<K>(c, g.tgt)]);
    }
    __syncthreads();
    if (active) tile[b | out_off] = acc;
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ void tile_diag(cplx_t<T>* tile, int L, const TileGate& g, const cplx_t<T>* __restrict__ d,
                                          uint64_t base) {
  uint32_t dglob = 0;
  for (int j = 0; j < g.k; ++j)
    if (g.tgt[j] & 0x80) dglob |= uint32_t((base >> (g.tgt[j] & 0x7f)) & 1) << j;
  const uint32_t count = 1u << (L - g.nfixed);
  for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) {
    const uint32_t e = insert_zeros32(i, g.fixed, g.nfixed) | g.lcv;
    uint32_t idx = dglob;
    for (int j = 0; j < g.k; ++j)
      if (!(g.tgt[j] & 0x80)) idx |= ((e >> g.tgt[j]) & 1u) << j;
    tile[e] = cmul<T>(__ldg(&d[idx]), tile[e]);
  }
}

}  // namespace qvdg
