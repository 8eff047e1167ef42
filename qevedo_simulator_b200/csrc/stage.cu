// Staged tile kernel: a CTA loads a tile of 2^L amplitudes (the low B
// physical bits plus L - B chosen bits) into shared memory with 16-byte
// coalesced loads, applies the stage's whole gate program in place, and
// stores it back. CTAs are persistent over tiles. The tile is the GPU form of
// the reference's region (src/blocking.rs:228-302): one pass over HBM per
// stage instead of one per gate.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "program.hpp"
#include "stage.hpp"
#include "stage_kernel.hpp"

namespace qvdg {

namespace {

constexpr int kStageThreads = 256;

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

template <typename T>
__global__ void __launch_bounds__(kStageThreads) k_stage(cplx_t<T>* __restrict__ psi, const TileGeom geo,
                                                         const TileGate* __restrict__ gates,
                                                         const cplx_t<T>* __restrict__ mats) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint8_t tile_bits[48];
  if (threadIdx.x < 48) tile_bits[threadIdx.x] = geo.tile_bits[threadIdx.x];
  __syncthreads();  // every thread reads tile_bits below
  const int L = geo.L, B = geo.B;
  cplx_t<T>* tile = reinterpret_cast<cplx_t<T>*>(smem);
  uint64_t* hi = reinterpret_cast<uint64_t*>(smem + (sizeof(cplx_t<T>) << L));
  const int nhi = 1 << (L - B);
  for (int r = threadIdx.x; r < nhi; r += blockDim.x) {
    uint64_t a = 0;
    for (int j = 0; j < L - B; ++j)
      if ((r >> j) & 1) a |= uint64_t(1) << tile_bits[B + j];
    hi[r] = a;
  }
  __syncthreads();
  const uint32_t n_el = 1u << L;
  const uint32_t lowmask = (1u << B) - 1u;
  // 16-byte accesses: two complex64 per access when runs have >= 2 amplitudes.
  const bool pairs = sizeof(T) == 4 && B >= 1;
  for (uint64_t t = blockIdx.x; t < geo.num_tiles; t += gridDim.x) {
    const uint64_t base = insert_zeros(t, tile_bits, L);
    if (pairs) {
      for (uint32_t e = threadIdx.x * 2; e < n_el; e += blockDim.x * 2) {
        const uint64_t a = base | hi[e >> B] | (e & lowmask);
        *reinterpret_cast<float4*>(&tile[e]) = *reinterpret_cast<const float4*>(&psi[a]);
      }
    } else {
      for (uint32_t e = threadIdx.x; e < n_el; e += blockDim.x) tile[e] = psi[base | hi[e >> B] | (e & lowmask)];
    }
    __syncthreads();
    for (int gi = 0; gi < geo.num_gates; ++gi) {
      const TileGate& g = gates[gi];
      if ((base & g.gcm) != g.gcv) continue;  // global controls: same for the whole tile
      const cplx_t<T>* m = mats + g.mat;
      if (g.kind == 1) {
        tile_diag<T>(tile, L, g, m, base);
      } else {
        switch (g.k) {
          case 1: tile_dense<T, 1>(tile, L, g, m); break;
          case 2: tile_dense<T, 2>(tile, L, g, m); break;
          case 3: tile_dense<T, 3>(tile, L, g, m); break;
          case 4: tile_dense<T, 4>(tile, L, g, m); break;
          case 5: tile_dense_rows<T, 5>(tile, L, g, m); break;
          default: tile_dense_rows<T, 6>(tile, L, g, m); break;
        }
      }
      __syncthreads();
    }
    if (pairs) {
      for (uint32_t e = threadIdx.x * 2; e < n_el; e += blockDim.x * 2) {
        const uint64_t a = base | hi[e >> B] | (e & lowmask);
        *reinterpret_cast<float4*>(&psi[a]) = *reinterpret_cast<const float4*>(&tile[e]);
      }
    } else {
      for (uint32_t e = threadIdx.x; e < n_el; e += blockDim.x) psi[base | hi[e >> B] | (e & lowmask)] = tile[e];
    }
    __syncthreads();
  }
}

template <typename T>
void stage_launch(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  const int L = lp.geo.L, B = lp.geo.B;
  const size_t smem = (sizeof(cplx_t<T>) << L) + (sizeof(uint64_t) << (L - B));
  static size_t configured = 0;
  if (smem > configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_stage<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    configured = smem;
  }
  const size_t per_sm = std::max<size_t>(1, std::min<size_t>(8, (220 * 1024) / smem));
  const uint64_t grid = std::min<uint64_t>(lp.geo.num_tiles, uint64_t(s.sms) * per_sm);
  k_stage<T><<<unsigned(grid), kStageThreads, smem, s.stream>>>(
      static_cast<cplx_t<T>*>(s.amp), lp.geo, dev.gates + lp.gate_offset, static_cast<const cplx_t<T>*>(dev.mats));
  QVDG_LAUNCH_CHECK();
}

}  // namespace

LoweredPass lower_pass(const Target& s, const PlannedPass& p, const StageConfig& cfg, StageUpload& up) {
  LoweredPass lp;
  lp.staged = p.staged;
  if (!p.staged) {
    const HOp& op = p.ops[0];
    PlainGate& g = lp.plain;
    g.diagonal = op.diagonal;
    for (uint32_t q : op.targets) g.targets.push_back(s.layout[q]);
    for (auto& c : op.controls) g.controls.push_back({s.layout[c.first], c.second});
    if (g.diagonal) {
      if (op.targets.size() > QVDG_MAX_DIAGONAL_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "diagonal gates on more than 10 qubits are not supported");
      g.matrix_offset = up.push_matrix(op.matrix.diagonal_entries());
    } else {
      if (op.targets.size() > QVDG_MAX_GATE_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "dense gates on more than 6 qubits are not supported");
      g.matrix_offset = up.push_matrix(op.matrix.a);
    }
    return lp;
  }
  TileGeom& geo = lp.geo;
  geo.L = int(p.tile_bits.size());
  geo.B = int(cfg.low_bits);
  geo.num_tiles = uint64_t(1) << (s.n - uint32_t(geo.L));
  for (size_t j = 0; j < p.tile_bits.size(); ++j) geo.tile_bits[j] = uint8_t(p.tile_bits[j]);
  std::vector<int> local(s.n, -1);
  for (size_t j = 0; j < p.tile_bits.size(); ++j) local[p.tile_bits[j]] = int(j);
  lp.gate_offset = up.gates.size();
  for (const HOp& op : p.ops) {
    TileGate g{};
    std::vector<uint8_t> fixed;
    for (auto& c : op.controls) {
      const uint32_t ph = s.layout[c.first];
      if (local[ph] >= 0) {
        g.lcm |= 1u << local[ph];
        if (c.second) g.lcv |= 1u << local[ph];
        fixed.push_back(uint8_t(local[ph]));
      } else {
        g.gcm |= uint64_t(1) << ph;
        if (c.second) g.gcv |= uint64_t(1) << ph;
      }
    }
    g.k = uint8_t(op.targets.size());
    if (op.diagonal) {
      if (op.targets.size() > QVDG_MAX_DIAGONAL_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "diagonal gates on more than 10 qubits are not supported");
      g.kind = 1;
      for (size_t j = 0; j < op.targets.size(); ++j) {
        const uint32_t ph = s.layout[op.targets[j]];
        g.tgt[j] = local[ph] >= 0 ? uint8_t(local[ph]) : uint8_t(0x80 | ph);
      }
      g.mat = uint32_t(up.push_matrix(op.matrix.diagonal_entries()));
    } else {
      if (op.targets.size() > QVDG_MAX_GATE_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "dense gates on more than 6 qubits are not supported");
      g.kind = 0;
      for (size_t j = 0; j < op.targets.size(); ++j) {
        const int l = local[s.layout[op.targets[j]]];
        if (l < 0) throw Error(QVDG_ERR_INVALID, "internal: dense stage gate with a global target");
        g.tgt[j] = uint8_t(l);
        fixed.push_back(uint8_t(l));
      }
      if (op.targets.size() >= 5) {
        // transposed for the row-parallel kernel
        const size_t D = op.matrix.dim;
        std::vector<C> t(D * D);
        for (size_t r = 0; r < D; ++r)
          for (size_t c = 0; c < D; ++c) t[c * D + r] = op.matrix.at(r, c);
        g.mat = uint32_t(up.push_matrix(t));
      } else {
        g.mat = uint32_t(up.push_matrix(op.matrix.a));
      }
    }
    std::sort(fixed.begin(), fixed.end());
    g.nfixed = uint8_t(fixed.size());
    for (size_t i = 0; i < fixed.size(); ++i) g.fixed[i] = fixed[i];
    up.gates.push_back(g);
  }
  geo.num_gates = int(up.gates.size() - lp.gate_offset);
  return lp;
}

void launch_pass(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  if (!lp.staged) {
    launch_plain_gate(s, lp.plain, dev.mats);
    return;
  }
  if (s.bits == 32)
    stage_launch<float>(s, lp, dev);
  else
    stage_launch<double>(s, lp, dev);
}

}  // namespace qvdg
