// Plain-path gate kernels: one pass over the state per fused gate.
//
// These replace the reference's AVX2 sweeps (src/kernels.rs:252-473). The
// state is interleaved complex in physical index order; a gate on physical
// target bits t_0..t_{k-1} with controls acts on groups of 2^k amplitudes
// whose index differs only in the target bits and whose control bits hold.
// Group bases are enumerated by inserting zero bits at the (sorted) target
// and control positions of a running counter, so a controlled gate touches
// only the 2^-c of the state its controls select (the reference's
// `free_mask`/`control_value`, src/kernels.rs:78-135). Consecutive threads
// take consecutive bases: when bit 0 is free, a warp's loads of each group
// member are one contiguous 256-byte (complex64) or 512-byte (complex128)
// run, and complex64 threads take two neighbouring groups with one 16-byte
// load per member.

#include <cuda_runtime.h>

#include <algorithm>

#include "engine.hpp"

namespace qvdg {

namespace {

constexpr int kThreads = 256;

struct DenseGeom {
  uint64_t n_iter;         // number of groups
  uint64_t control_value;  // control bits that must be 1
  uint64_t offsets[64];    // index offset of each group member (matrix index order)
  uint8_t fixed[40];       // sorted target and control positions
  int32_t num_fixed;
};

template <typename T, int K, int G, bool VEC>
__global__ void __launch_bounds__(kThreads) k_dense(cplx_t<T>* __restrict__ psi, const DenseGeom g,
                                                    const cplx_t<T>* __restrict__ mat) {
  constexpr int D = 1 << K;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* sm = reinterpret_cast<cplx_t<T>*>(smem_raw);
  __shared__ uint8_t fixed[40];
  for (int i = threadIdx.x; i < D * D; i += blockDim.x) sm[i] = mat[i];
  if (threadIdx.x < 40) fixed[threadIdx.x] = g.fixed[threadIdx.x];
  __syncthreads();
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x * G;
  for (uint64_t it = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) * G; it < g.n_iter; it += stride) {
    uint64_t base[G];
#pragma unroll
    for (int q = 0; q < G; ++q) base[q] = insert_zeros(it + q, fixed, g.num_fixed) | g.control_value;
    cplx_t<T> x[G][D];
    if constexpr (VEC) {
      // complex64 with bit 0 free: groups it and it+1 are neighbours.
#pragma unroll
      for (int h = 0; h < D; ++h) {
        const float4 v = *reinterpret_cast<const float4*>(psi + base[0] + g.offsets[h]);
        x[0][h] = make_c<T>(v.x, v.y);
        x[G - 1][h] = make_c<T>(v.z, v.w);
      }
    } else {
#pragma unroll
      for (int h = 0; h < D; ++h)
#pragma unroll
        for (int q = 0; q < G; ++q) x[q][h] = psi[base[q] + g.offsets[h]];
    }
#pragma unroll 1
    for (int r = 0; r < D; ++r) {
      cplx_t<T> acc[G];
#pragma unroll
      for (int q = 0; q < G; ++q) acc[q] = make_c<T>(T(0), T(0));
#pragma unroll
      for (int c = 0; c < D; ++c) {
        const cplx_t<T> m = sm[r * D + c];
#pragma unroll
        for (int q = 0; q < G; ++q) cmac<T>(acc[q], m, x[q][c]);
      }
      if constexpr (VEC) {
        *reinterpret_cast<float4*>(psi + base[0] + g.offsets[r]) =
            make_float4(acc[0].x, acc[0].y, acc[G - 1].x, acc[G - 1].y);
      } else {
#pragma unroll
        for (int q = 0; q < G; ++q) psi[base[q] + g.offsets[r]] = acc[q];
      }
    }
  }
}

// Dense gates whose targets all lie in index bits 0-4 (the lane bits of a
// warp row of 32 consecutive amplitudes), with controls above them: the
// GPU form of the reference's in-register lane permutations for targets
// inside a SIMD vector (src/kernels.rs:185, 273, xor_perm). A warp takes
// whole rows, lane l holding amplitude l of the row (one coalesced 256- or
// 512-byte access); the other members of its group are in the lanes whose
// target bits differ, and come over by warp shuffles. Lane l computes its
// own output, row r(l) of the gate (r = its target bits in matrix order),
// held in registers, so neither shared memory nor a second pass over the
// row is needed. Each thread keeps R rows in flight.
struct LaneGeom {
  uint64_t rows;           // warp rows of 32 amplitudes the controls select
  uint64_t control_value;  // control bits that must be 1
  uint8_t fixed[40];       // bits 0-4 and the control positions, ascending
  int32_t num_fixed;
  uint8_t targets[4];      // target positions (matrix bit order), all below 5
};

template <typename T, int K, int R>
__global__ void __launch_bounds__(kThreads) k_dense_lanes(cplx_t<T>* __restrict__ psi, const LaneGeom g,
                                                          const cplx_t<T>* __restrict__ mat) {
  constexpr int D = 1 << K;
  __shared__ uint8_t fixed[40];
  if (threadIdx.x < 40) fixed[threadIdx.x] = g.fixed[threadIdx.x];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t tmask = 0, row = 0;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    tmask |= 1u << g.targets[j];
    row |= ((lane >> g.targets[j]) & 1u) << j;
  }
  cplx_t<T> m[D];
  int src[D];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    m[c] = mat[row * D + c];
    uint32_t p = lane & ~tmask;
#pragma unroll
    for (int j = 0; j < K; ++j) p |= uint32_t((c >> j) & 1) << g.targets[j];
    src[c] = int(p);
  }
  const uint64_t warps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  const uint64_t first = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  for (uint64_t w0 = first * R; w0 < g.rows; w0 += warps * R) {
    uint64_t base[R];
    cplx_t<T> x[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      base[q] = w0 + q < g.rows ? (insert_zeros(w0 + q, fixed, g.num_fixed) | g.control_value) + lane : ~uint64_t(0);
      if (base[q] != ~uint64_t(0)) x[q] = psi[base[q]];
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      cplx_t<T> acc = make_c<T>(T(0), T(0));
#pragma unroll
      for (int c = 0; c < D; ++c) {
        cplx_t<T> y;
        y.x = __shfl_sync(0xffffffffu, x[q].x, src[c]);
        y.y = __shfl_sync(0xffffffffu, x[q].y, src[c]);
        cmac<T>(acc, m[c], y);
      }
      if (base[q] != ~uint64_t(0)) psi[base[q]] = acc;
    }
  }
}

// Dense gates with targets among the low index bits: each thread's group is
// then a short contiguous run and a warp's loads stride by the run length.
// Instead, a block stages a tile of 2^13 amplitudes -- index bits 0..Lb-1
// (contiguous runs of 2^Lb) plus the targets above them -- in shared memory
// with coalesced 16-byte accesses, applies the gate to the tile's 2^(13-K)
// groups there (two per thread, so each matrix entry read serves both) and
// stores the tile back.
constexpr int kTileBits = 13;

struct DenseTileGeom {
  uint64_t tiles;
  int32_t lb;             // contiguous low bits of the tile
  int32_t nhigh;          // targets at or above lb
  uint8_t high[8];        // physical positions of those targets (ascending)
  uint8_t fixed_tile[8];  // tile-local positions of all targets (ascending)
  uint16_t offsets[64];   // tile-local offset of group member h (matrix index order)
};

// Shared-memory position of tile element e (bits 4-7 folded into 1-3; bit 0
// kept so 16-byte element pairs stay together).
__device__ __forceinline__ uint32_t dswz(uint32_t e) { return e ^ ((e >> 4) & 14u); }

template <int K>
__global__ void __launch_bounds__(kThreads) k_dense_tile(float2* __restrict__ psi, const DenseTileGeom g,
                                                         const float2* __restrict__ mat) {
  constexpr int D = 1 << K;
  constexpr uint32_t kTile = 1u << kTileBits;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tile = reinterpret_cast<float2*>(smem_raw);
  float2* sm = tile + kTile;
  __shared__ uint8_t fixed[8];
  __shared__ uint16_t off[64];
  for (int i = threadIdx.x; i < D * D; i += blockDim.x) sm[i] = mat[i];
  if (threadIdx.x < 8) fixed[threadIdx.x] = g.fixed_tile[threadIdx.x];
  if (threadIdx.x < 64) off[threadIdx.x] = g.offsets[threadIdx.x];
  __syncthreads();
  const uint32_t lowmask = (1u << g.lb) - 1u;
  for (uint64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    // Tile t: its bits above lb, with zeros at the high targets, give the
    // base index; element e adds its low bits and the high targets.
    uint64_t base = t << g.lb;
    for (int i = 0; i < g.nhigh; ++i) {
      const uint32_t p = g.high[i];
      base = ((base >> p) << (p + 1)) | (base & ((uint64_t(1) << p) - 1));
    }
    auto global_of = [&](uint32_t e) -> uint64_t {
      uint64_t x = base | (e & lowmask);
      uint32_t h = e >> g.lb;
      for (int i = 0; i < g.nhigh; ++i) x |= uint64_t((h >> i) & 1u) << g.high[i];
      return x;
    };
    // Every 16-byte copy of the tile in flight at once (cp.async).
    for (uint32_t u = threadIdx.x; u < kTile / 2; u += blockDim.x) {
      const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(tile + dswz(2 * u)));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(psi + global_of(2 * u)) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    constexpr uint32_t kGroups = kTile >> K;
    for (uint32_t q = threadIdx.x; q < kGroups / 2; q += blockDim.x) {
      uint32_t b[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        uint32_t x = q + s * (kGroups / 2);
#pragma unroll
        for (int i = 0; i < K; ++i) {
          const uint32_t p = fixed[i];
          x = ((x >> p) << (p + 1)) | (x & ((1u << p) - 1u));
        }
        b[s] = x;
      }
      float2 x[2][D];
#pragma unroll
      for (int h = 0; h < D; ++h) {
        x[0][h] = tile[dswz(b[0] | off[h])];
        x[1][h] = tile[dswz(b[1] | off[h])];
      }
#pragma unroll 1
      for (int r = 0; r < D; ++r) {
        float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < D; c += 2) {
          const float4 m = *reinterpret_cast<const float4*>(sm + r * D + c);
          const float2 m0 = make_float2(m.x, m.y), m1 = make_float2(m.z, m.w);
          cmac<float>(a0, m0, x[0][c]);
          cmac<float>(a1, m0, x[1][c]);
          cmac<float>(a0, m1, x[0][c + 1]);
          cmac<float>(a1, m1, x[1][c + 1]);
        }
        tile[dswz(b[0] | off[r])] = a0;
        tile[dswz(b[1] | off[r])] = a1;
      }
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < kTile / 2; u += blockDim.x)
      *reinterpret_cast<float4*>(psi + global_of(2 * u)) = *reinterpret_cast<const float4*>(tile + dswz(2 * u));
    __syncthreads();
  }
}

struct DiagGeom {
  uint64_t n_iter;         // amplitudes in the controlled subspace
  uint64_t control_value;
  uint8_t ctrl[40];        // sorted control positions
  int32_t num_ctrl;
  uint8_t targets[16];     // diagonal index bit j = targets[j]
  int32_t k;
};

template <typename T, int G>
__global__ void __launch_bounds__(kThreads) k_diag(cplx_t<T>* __restrict__ psi, const DiagGeom g,
                                                   const cplx_t<T>* __restrict__ diag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* sm = reinterpret_cast<cplx_t<T>*>(smem_raw);
  __shared__ uint8_t ctrl[40], tgt[16];
  for (int i = threadIdx.x; i < (1 << g.k); i += blockDim.x) sm[i] = diag[i];
  if (threadIdx.x < 40) ctrl[threadIdx.x] = g.ctrl[threadIdx.x];
  if (threadIdx.x < 16) tgt[threadIdx.x] = g.targets[threadIdx.x];
  __syncthreads();
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x * G;
  for (uint64_t it = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) * G; it < g.n_iter; it += stride) {
    // With G == 2, bit 0 is not a control: indices i and i+1 are neighbours.
    const uint64_t i = insert_zeros(it, ctrl, g.num_ctrl) | g.control_value;
    uint32_t d[G];
#pragma unroll
    for (int q = 0; q < G; ++q) {
      d[q] = 0;
      for (int j = 0; j < g.k; ++j) d[q] |= uint32_t(((i + q) >> tgt[j]) & 1) << j;
    }
    if constexpr (G == 2 && sizeof(T) == 4) {
      float4 v = *reinterpret_cast<float4*>(psi + i);
      const cplx_t<T> a = cmul<T>(sm[d[0]], make_c<T>(v.x, v.y));
      const cplx_t<T> b = cmul<T>(sm[d[1]], make_c<T>(v.z, v.w));
      *reinterpret_cast<float4*>(psi + i) = make_float4(a.x, a.y, b.x, b.y);
    } else {
#pragma unroll
      for (int q = 0; q < G; ++q) psi[i + q] = cmul<T>(sm[d[q]], psi[i + q]);
    }
  }
}

struct SwapGeom {
  uint64_t mask;  // every swapped bit
  int32_t np;
  uint8_t a[32], b[32];
};

template <typename T>
__global__ void k_swap_bits(cplx_t<T>* __restrict__ psi, uint64_t len, const SwapGeom g) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    uint64_t j = i & ~g.mask;
    for (int p = 0; p < g.np; ++p)
      j |= (((i >> g.a[p]) & 1) << g.b[p]) | (((i >> g.b[p]) & 1) << g.a[p]);
    if (i < j) {
      const cplx_t<T> t = psi[i];
      psi[i] = psi[j];
      psi[j] = t;
    }
  }
}

template <typename T>
__global__ void k_set_one(cplx_t<T>* psi) {
  psi[0] = make_c<T>(T(1), T(0));
}

// Logical index -> physical index through per-byte lookup tables.
__device__ __forceinline__ uint64_t to_physical(uint64_t i, const uint64_t* tables, int ntables) {
  if (ntables == 0) return i;
  uint64_t p = 0;
  for (int b = 0; b < ntables; ++b) p |= tables[b * 256 + ((i >> (8 * b)) & 255)];
  return p;
}

template <typename T>
__global__ void k_export(const cplx_t<T>* __restrict__ psi, double2* __restrict__ out, uint64_t first,
                         uint64_t count, const uint64_t* __restrict__ tables, int ntables) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += stride) {
    const cplx_t<T> a = psi[to_physical(first + t, tables, ntables)];
    out[t] = make_double2(double(a.x), double(a.y));
  }
}

template <typename T>
__global__ void k_import(cplx_t<T>* __restrict__ psi, const double2* __restrict__ in, uint64_t first,
                         uint64_t count, const uint64_t* __restrict__ tables, int ntables) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += stride) {
    const double2 a = in[t];
    psi[to_physical(first + t, tables, ntables)] = make_c<T>(T(a.x), T(a.y));
  }
}

template <typename T>
__global__ void k_scale(cplx_t<T>* __restrict__ psi, uint64_t len, double factor) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    cplx_t<T> a = psi[i];
    a.x = T(double(a.x) * factor);
    a.y = T(double(a.y) * factor);
    psi[i] = a;
  }
}

unsigned grid_for(const StateImpl& s, uint64_t work_items) {
  const uint64_t blocks = (work_items + kThreads - 1) / kThreads;
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(blocks, uint64_t(s.sms) * 16)));
}

template <typename T, int K, int G, bool VEC>
void dense_launch(StateImpl& s, const DenseGeom& g, const void* mat) {
  const size_t smem = size_t(1) << (2 * K);
  const size_t bytes = smem * sizeof(cplx_t<T>);
  static bool configured = false;  // per instantiation
  if (!configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_dense<T, K, G, VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    configured = true;
  }
  k_dense<T, K, G, VEC><<<grid_for(s, g.n_iter / G), kThreads, bytes, s.stream>>>(
      static_cast<cplx_t<T>*>(s.amp), g, static_cast<const cplx_t<T>*>(mat));
  QVDG_LAUNCH_CHECK();
}

template <typename T, int K>
void dense_pick(StateImpl& s, const DenseGeom& g, const void* mat, bool bit0_free) {
  if constexpr (K <= 4) {
    if (g.n_iter >= 2) {
      if (sizeof(T) == 4 && bit0_free)
        return dense_launch<T, K, 2, true>(s, g, mat);
      return dense_launch<T, K, 2, false>(s, g, mat);
    }
  }
  dense_launch<T, K, 1, false>(s, g, mat);
}

template <typename T, int K>
void lanes_launch(StateImpl& s, const LaneGeom& g, const void* mat) {
  constexpr int R = 4;
  const uint64_t warps_needed = (g.rows + R - 1) / R;
  const unsigned grid = grid_for(s, warps_needed * 32);
  k_dense_lanes<T, K, R><<<grid, kThreads, 0, s.stream>>>(static_cast<cplx_t<T>*>(s.amp), g,
                                                          static_cast<const cplx_t<T>*>(mat));
  QVDG_LAUNCH_CHECK();
}

template <typename T>
void lanes_pick(StateImpl& s, const PlainGate& pg, uint64_t control_value, const std::vector<uint8_t>& ctrl,
                const void* mat) {
  LaneGeom g{};
  g.rows = uint64_t(1) << (s.n - 5 - ctrl.size());
  g.control_value = control_value;
  std::vector<uint8_t> fixed = {0, 1, 2, 3, 4};
  fixed.insert(fixed.end(), ctrl.begin(), ctrl.end());
  std::sort(fixed.begin(), fixed.end());
  g.num_fixed = int(fixed.size());
  for (size_t i = 0; i < fixed.size(); ++i) g.fixed[i] = fixed[i];
  for (size_t j = 0; j < pg.targets.size(); ++j) g.targets[j] = uint8_t(pg.targets[j]);
  switch (pg.targets.size()) {
    case 1: return lanes_launch<T, 1>(s, g, mat);
    case 2: return lanes_launch<T, 2>(s, g, mat);
    default: return lanes_launch<T, 3>(s, g, mat);
  }
}

template <typename T>
void plain_gate(StateImpl& s, const PlainGate& pg, const void* matrices) {
  const int k = int(pg.targets.size());
  const int c = int(pg.controls.size());
  uint64_t control_value = 0;
  std::vector<uint8_t> ctrl;
  for (auto& cv : pg.controls) {
    ctrl.push_back(uint8_t(cv.first));
    if (cv.second) control_value |= uint64_t(1) << cv.first;
  }
  std::sort(ctrl.begin(), ctrl.end());
  const cplx_t<T>* mat = static_cast<const cplx_t<T>*>(matrices) + pg.matrix_offset;
  if (pg.diagonal) {
    DiagGeom g{};
    g.n_iter = uint64_t(1) << (s.n - c);
    g.control_value = control_value;
    g.num_ctrl = c;
    for (int i = 0; i < c; ++i) g.ctrl[i] = ctrl[i];
    g.k = k;
    for (int j = 0; j < k; ++j) g.targets[j] = uint8_t(pg.targets[j]);
    const bool bit0_ctrl = c > 0 && ctrl[0] == 0;
    const size_t bytes = (size_t(1) << k) * sizeof(cplx_t<T>);
    if (g.n_iter >= 2 && !bit0_ctrl)
      k_diag<T, 2><<<grid_for(s, g.n_iter / 2), kThreads, bytes, s.stream>>>(static_cast<cplx_t<T>*>(s.amp), g, mat);
    else
      k_diag<T, 1><<<grid_for(s, g.n_iter), kThreads, bytes, s.stream>>>(static_cast<cplx_t<T>*>(s.amp), g, mat);
    QVDG_LAUNCH_CHECK();
    return;
  }
  DenseGeom g{};
  g.n_iter = uint64_t(1) << (s.n - k - c);
  g.control_value = control_value;
  std::vector<uint8_t> fixed(ctrl);
  for (uint32_t t : pg.targets) fixed.push_back(uint8_t(t));
  std::sort(fixed.begin(), fixed.end());
  g.num_fixed = int(fixed.size());
  for (size_t i = 0; i < fixed.size(); ++i) g.fixed[i] = fixed[i];
  for (int h = 0; h < (1 << k); ++h) {
    uint64_t o = 0;
    for (int j = 0; j < k; ++j) o |= uint64_t((h >> j) & 1) << pg.targets[j];
    g.offsets[h] = o;
  }
  const bool bit0_free = fixed.empty() || fixed[0] != 0;
  // Targets all in the lane bits 0-4 (controls above them): warp shuffles.
  {
    bool lanes = k <= 3 && s.n >= 5;
    for (uint32_t t : pg.targets) lanes = lanes && t < 5;
    for (uint8_t cq : ctrl) lanes = lanes && cq >= 5;
    if (lanes) return lanes_pick<T>(s, pg, control_value, ctrl, mat);
  }
  // complex64, no controls, targets (nearly) all among bits 0-3 -- each
  // group one short contiguous run -- and a state of at least one tile:
  // stage tiles through shared memory (coalesced) instead. With fewer low
  // targets the direct kernel's accesses are coalesced enough and it is faster.
  int low_targets = 0;
  for (uint32_t t : pg.targets) low_targets += t < 4 ? 1 : 0;
  if (sizeof(T) == 4 && c == 0 && k >= 2 && k <= 4 && low_targets >= std::min(k, 3) &&
      s.n >= uint32_t(kTileBits) + 1) {
    DenseTileGeom tg{};
    int lb = kTileBits, nhigh = 0;
    for (int iter = 0; iter < 8; ++iter) {
      nhigh = 0;
      for (uint32_t t : pg.targets) nhigh += t >= uint32_t(lb) ? 1 : 0;
      const int next = kTileBits - nhigh;
      if (next == lb) break;
      lb = next;
    }
    std::vector<uint32_t> high;
    for (uint32_t t : pg.targets)
      if (t >= uint32_t(lb)) high.push_back(t);
    std::sort(high.begin(), high.end());
    if (int(high.size()) == nhigh && lb + nhigh == kTileBits) {
      tg.lb = lb;
      tg.nhigh = nhigh;
      tg.tiles = uint64_t(1) << (s.n - kTileBits);
      for (int i = 0; i < nhigh; ++i) tg.high[i] = uint8_t(high[i]);
      auto local = [&](uint32_t t) -> uint32_t {
        if (t < uint32_t(lb)) return t;
        return uint32_t(lb) + uint32_t(std::find(high.begin(), high.end(), t) - high.begin());
      };
      std::vector<uint8_t> ft;
      for (uint32_t t : pg.targets) ft.push_back(uint8_t(local(t)));
      std::sort(ft.begin(), ft.end());
      for (size_t i = 0; i < ft.size(); ++i) tg.fixed_tile[i] = ft[i];
      for (int h = 0; h < (1 << k); ++h) {
        uint32_t o = 0;
        for (int j = 0; j < k; ++j) o |= uint32_t((h >> j) & 1) << local(pg.targets[j]);
        tg.offsets[h] = uint16_t(o);
      }
      const size_t bytes = (size_t(1) << kTileBits) * sizeof(float2) + (size_t(1) << (2 * k)) * sizeof(float2);
      const unsigned grid = unsigned(std::min<uint64_t>(tg.tiles, uint64_t(s.sms) * 3));
      auto* psi = static_cast<float2*>(s.amp);
      auto* m = reinterpret_cast<const float2*>(mat);
      static bool configured[5] = {false, false, false, false, false};
      if (!configured[k]) {
        const void* fn = k == 2 ? reinterpret_cast<const void*>(k_dense_tile<2>)
                                : (k == 3 ? reinterpret_cast<const void*>(k_dense_tile<3>)
                                          : reinterpret_cast<const void*>(k_dense_tile<4>));
        QVDG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
        configured[k] = true;
      }
      switch (k) {
        case 2:
          k_dense_tile<2><<<grid, kThreads, bytes, s.stream>>>(psi, tg, m);
          break;
        case 3: k_dense_tile<3><<<grid, kThreads, bytes, s.stream>>>(psi, tg, m); break;
        default: k_dense_tile<4><<<grid, kThreads, bytes, s.stream>>>(psi, tg, m); break;
      }
      QVDG_LAUNCH_CHECK();
      return;
    }
  }
  switch (k) {
    case 1: return dense_pick<T, 1>(s, g, mat, bit0_free);
    case 2: return dense_pick<T, 2>(s, g, mat, bit0_free);
    case 3: return dense_pick<T, 3>(s, g, mat, bit0_free);
    case 4: return dense_pick<T, 4>(s, g, mat, bit0_free);
    case 5: return dense_pick<T, 5>(s, g, mat, bit0_free);
    case 6: return dense_pick<T, 6>(s, g, mat, bit0_free);
    default: throw Error(4, "dense gates on more than 6 qubits are not supported");
  }
}

// Byte-wise logical->physical tables for a non-identity layout (uploaded to
// the workspace); returns the number of tables (0 for the identity).
int layout_tables(StateImpl& s, uint64_t** dev_tables) {
  if (s.identity_layout()) {
    *dev_tables = nullptr;
    return 0;
  }
  const int ntables = int((s.n + 7) / 8);
  std::vector<uint64_t> t(size_t(ntables) * 256, 0);
  for (int b = 0; b < ntables; ++b)
    for (int v = 0; v < 256; ++v) {
      uint64_t p = 0;
      for (int bit = 0; bit < 8; ++bit) {
        const uint32_t q = uint32_t(8 * b + bit);
        if (q < s.n && ((v >> bit) & 1)) p |= uint64_t(1) << s.layout[q];
      }
      t[size_t(b) * 256 + v] = p;
    }
  uint64_t* d = static_cast<uint64_t*>(s.work2.get(t.size() * sizeof(uint64_t)));
  QVDG_CUDA(cudaMemcpyAsync(d, t.data(), t.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));  // `t` is pageable and goes out of scope
  *dev_tables = d;
  return ntables;
}

}  // namespace

void launch_plain_gate(StateImpl& s, const PlainGate& g, const void* matrices) {
  if (s.bits == 32)
    plain_gate<float>(s, g, matrices);
  else
    plain_gate<double>(s, g, matrices);
}

void launch_swap_bits(StateImpl& s, const std::vector<std::pair<uint32_t, uint32_t>>& pairs) {
  if (pairs.empty()) return;
  SwapGeom g{};
  g.np = int(pairs.size());
  for (size_t p = 0; p < pairs.size(); ++p) {
    g.a[p] = uint8_t(pairs[p].first);
    g.b[p] = uint8_t(pairs[p].second);
    g.mask |= (uint64_t(1) << pairs[p].first) | (uint64_t(1) << pairs[p].second);
  }
  if (s.bits == 32)
    k_swap_bits<float><<<grid_for(s, s.size()), kThreads, 0, s.stream>>>(static_cast<float2*>(s.amp), s.size(), g);
  else
    k_swap_bits<double><<<grid_for(s, s.size()), kThreads, 0, s.stream>>>(static_cast<double2*>(s.amp), s.size(), g);
  QVDG_LAUNCH_CHECK();
}

void launch_zero(StateImpl& s) {
  QVDG_CUDA(cudaMemsetAsync(s.amp, 0, s.amp_bytes, s.stream));
  if (s.bits == 32)
    k_set_one<float><<<1, 1, 0, s.stream>>>(static_cast<float2*>(s.amp));
  else
    k_set_one<double><<<1, 1, 0, s.stream>>>(static_cast<double2*>(s.amp));
  QVDG_LAUNCH_CHECK();
}

void launch_export(StateImpl& s, uint64_t first, uint64_t count, double* out_dev) {
  uint64_t* tables;
  const int nt = layout_tables(s, &tables);
  if (s.bits == 32)
    k_export<float><<<grid_for(s, count), kThreads, 0, s.stream>>>(static_cast<const float2*>(s.amp),
                                                                    reinterpret_cast<double2*>(out_dev), first,
                                                                    count, tables, nt);
  else
    k_export<double><<<grid_for(s, count), kThreads, 0, s.stream>>>(static_cast<const double2*>(s.amp),
                                                                     reinterpret_cast<double2*>(out_dev), first,
                                                                     count, tables, nt);
  QVDG_LAUNCH_CHECK();
}

void launch_import(StateImpl& s, uint64_t first, uint64_t count, const double* in_dev) {
  uint64_t* tables;
  const int nt = layout_tables(s, &tables);
  if (s.bits == 32)
    k_import<float><<<grid_for(s, count), kThreads, 0, s.stream>>>(static_cast<float2*>(s.amp),
                                                                    reinterpret_cast<const double2*>(in_dev), first,
                                                                    count, tables, nt);
  else
    k_import<double><<<grid_for(s, count), kThreads, 0, s.stream>>>(static_cast<double2*>(s.amp),
                                                                     reinterpret_cast<const double2*>(in_dev),
                                                                     first, count, tables, nt);
  QVDG_LAUNCH_CHECK();
}

void launch_scale(StateImpl& s, double factor) {
  if (s.bits == 32)
    k_scale<float><<<grid_for(s, s.size()), kThreads, 0, s.stream>>>(static_cast<float2*>(s.amp), s.size(), factor);
  else
    k_scale<double><<<grid_for(s, s.size()), kThreads, 0, s.stream>>>(static_cast<double2*>(s.amp), s.size(),
                                                                       factor);
  QVDG_LAUNCH_CHECK();
}

}  // namespace qvdg
