// Plain passes of a fused dense gate on the 5th-generation tensor cores
// (tcgen05), complex64 state: the streaming form of the reference's dense
// fused-gate sweep (src/kernels.rs:252-473, one pass over the state per
// fused op) for 4-6 target qubits, where the 4^K complex multiply-adds per
// group would otherwise load the FP32 pipe as much as HBM.
//
// The gate is one real matrix product per block of 128 groups, as in the
// tensor-core stage kernel: row g of A holds group g's 2^K real parts and
// then its 2^K imaginary parts, B is [[Re M, Im M], [-Im M, Re M]]^T, both
// split into bf16 high and low parts, and D (fp32, tensor memory)
// accumulates A_hi B_hi + A_hi B_lo + A_lo B_hi (M = 128, N = K = 2^(K+1),
// canonical no-swizzle K-major layout, K-adjacent core matrices 128 bytes
// apart, row-group-adjacent ones 16 * 2^(K+1) bytes apart).
//
// Persistent CTAs of 512 threads; one CTA iteration covers 8192 amplitudes
// (4, 2 or 1 blocks for K = 4, 5, 6). Thread (w = tid / 128, r = tid % 128)
// owns 16 members of group r of block w / P, P = 2^K / 16: it loads them
// (consecutive threads take consecutive groups, so a warp's loads of one
// member are contiguous when bit 0 is free; with a target on bit 0 the
// members pair into 16-byte accesses, with targets on bits 0 and 1 into
// 32-byte ones), writes their bf16 parts into its lane r of one of two A
// buffers in tensor memory (tcgen05.st; the products read A from there and
// only the gate B sits in shared memory, which keeps the L1 / shared-memory
// path free for the global loads and stores), and, once TMEM lane r holds
// the block's products, reads its 16 members back and stores them where
// they came from. The loads of
// iteration i + 1 are issued before iteration i's products, and iteration
// i's read-back runs during iteration i + 1, so HBM traffic, the bf16 split,
// the tensor cores and the stores overlap. Every wait on an MMA completion
// barrier is bounded: on timeout the kernel records an error, every thread
// leaves the loop at the next CTA barrier and the tensor memory is freed.
// Group bases advance by a running deposit (the carry of an add skips the
// fixed bits), so no per-iteration bit insertion sits before the loads.
//
// Gates whose targets cover index bits 1-3 take a staged variant
// (k_dense_tc_tile, below): there each group is a short contiguous run and
// the direct kernel's warps would stride across runs.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "dense_tc.hpp"
#include "dense_tc_common.cuh"
#include "stage_kernel.hpp"
#include "tc_ptx.cuh"

namespace qvdg {

namespace {

template <int K, int VW>
__global__ void __launch_bounds__(kThreads, 1) k_dense_tc(float2* __restrict__ psi, const DenseTcGeom g,
                                                          const uint8_t* __restrict__ bmats,
                                                          int* __restrict__ status) {
  constexpr uint32_t D = 1u << K, kd = 2u * D;
  constexpr uint32_t P = D / 16;     // threads per group
  constexpr uint32_t T = 4 / P;      // blocks of 128 groups per iteration
  constexpr uint32_t GPI = T * 128;  // groups per iteration
  constexpr uint32_t BPART = kd * kd * 2;   // bytes of one part of B
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ uint8_t fixed[40];
  unsigned char* bmat = smem;  // B hi, then B lo
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t wg = uint32_t(tid) >> 7, r = uint32_t(tid) & 127u;
  const uint32_t blk = wg / P, chunk = wg % P;

  if (tid < 40) fixed[tid] = g.fixed[tid];
  {
    const uint4* src = reinterpret_cast<const uint4*>(bmats + g.b_offset);
    uint4* dst = reinterpret_cast<uint4*>(bmat);
    for (uint32_t i = tid; i < 2 * BPART / 16; i += kThreads) dst[i] = src[i];
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  // Member 16 * chunk + i sits at off_lo[i] (targets 0-3, below bit 32)
  // from this thread's base, which carries the chunk's higher targets.
  uint32_t off_lo[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) off_lo[i] = uint32_t(g.offsets[i]);
  // Group index = iteration * GPI + (blk * 128 + r): the two parts occupy
  // disjoint bits, so their deposits into the free positions OR together.
  const uint64_t tdep = insert_zeros(blk * 128 + r, fixed, g.num_fixed) | g.control_value | g.offsets[16 * chunk];
  const uint64_t my_iters = blockIdx.x < g.iters ? (g.iters - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // Iteration bases in load order and in store order, advanced by the
  // deposit of gridDim.x * GPI.
  uint64_t fmask = 0;
  for (int i = 0; i < g.num_fixed; ++i) fmask |= uint64_t(1) << fixed[i];
  const uint64_t dstep = insert_zeros(uint64_t(gridDim.x) * GPI, fixed, g.num_fixed);
  uint64_t dload = insert_zeros(uint64_t(blockIdx.x) * GPI, fixed, g.num_fixed), dstore = dload;
  auto next_load = [&]() -> uint64_t {
    const uint64_t b = dload | tdep;
    dload = dep_add(dload, dstep, fmask);
    return b;
  };
  auto next_store = [&]() -> uint64_t {
    const uint64_t b = dstore | tdep;
    dstore = dep_add(dstore, dstep, fmask);
    return b;
  };
  auto load = [&](float2 (&x)[16], uint64_t base) {
    if constexpr (VW == 4) {
#pragma unroll
      for (int m = 0; m < 4; ++m) ld_early32(psi + base + off_lo[4 * m], &x[4 * m]);
    } else if constexpr (VW == 2) {
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const float4 v = ld_early(psi + base + off_lo[2 * m]);
        x[2 * m] = make_float2(v.x, v.y);
        x[2 * m + 1] = make_float2(v.z, v.w);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) x[i] = ld_early8(psi + base + off_lo[i]);
    }
  };
  // Thread (w, r) owns tensor-memory lane r: its warp's quarter of the
  // lanes is r / 32 = w % 4.
  const uint32_t lanes = (uint32_t(warp & 3) * 32u) << 16;
  int failed = 0;
  // One step: iteration li's members into A (tensor memory) and its
  // products issued (the registers then take the loads of iteration
  // li + 2), and the previous iteration read back and stored. Returns
  // whether another step follows.
  auto step = [&](uint64_t li, float2 (&x)[16]) -> bool {
    const uint32_t b = uint32_t(li & 1);
    const uint32_t acol = kTmemA + b * 128;
    if (li < my_iters) {
      write_a8_tmem<K>(x, tmem + lanes + acol + blk * kd, chunk, 0);
      write_a8_tmem<K>(x + 8, tmem + lanes + acol + blk * kd, chunk, 1);
      if (li + 2 < my_iters) load(x, next_load());
      tmem_wait_st();
    }
    tc_fence_before();
    if (__syncthreads_or(failed)) return false;
    if (li < my_iters && tid == 0) issue_products_tmem_a<K>(tmem + acol, bmat, tmem + b * 128, smem_addr(&bar[b]));
    if (li > 0) {
      const uint32_t pb = b ^ 1u;
      const uint32_t parity = uint32_t(((li - 1) >> 1) & 1);
      const uint32_t barp = smem_addr(&bar[pb]);
      const uint64_t base = next_store();
      if (!wait_products(barp, parity)) {
        failed = 1;
        atomicExch(status, 1);
      } else {
        tc_fence_after();
        const uint32_t taddr = tmem + lanes + pb * 128 + blk * kd + 16 * chunk;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          float re[8], im[8];
          tmem_ld8(taddr + 8 * hh, re);
          tmem_ld8(taddr + D + 8 * hh, im);
          tmem_wait_ld();
          if constexpr (VW == 4) {
#pragma unroll
            for (int m = 0; m < 2; ++m) st32(psi + base + off_lo[8 * hh + 4 * m], re + 4 * m, im + 4 * m);
          } else if constexpr (VW == 2) {
#pragma unroll
            for (int m = 0; m < 4; ++m)
              *reinterpret_cast<float4*>(psi + base + off_lo[8 * hh + 2 * m]) =
                  make_float4(re[2 * m], im[2 * m], re[2 * m + 1], im[2 * m + 1]);
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) psi[base + off_lo[8 * hh + i]] = make_float2(re[i], im[i]);
          }
        }
      }
    }
    return li < my_iters;
  };
  // Two register sets in flight, so each iteration's loads are issued two
  // iterations ahead of their use.
  float2 xa[16], xb[16];
  if (my_iters > 0) load(xa, next_load());
  if (my_iters > 1) load(xb, next_load());
  for (uint64_t li = 0;; li += 2) {
    if (!step(li, xa)) break;
    if (!step(li + 1, xb)) break;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// Gates with targets on index bits 1-3: a warp's 32 consecutive groups are
// then scattered in memory, so the state moves through a shared-memory
// stage instead. A CTA of 128 * 2^K / 16 threads takes tiles of 128 groups:
// the 2^(7+K) amplitudes spanned by the bits `g.tile` (the targets and the
// seven lowest free bits, bit 0 always among them, so a tile is contiguous
// runs of at least 128 amplitudes). A tile is loaded with coalesced 16-byte
// accesses (two tiles ahead, in registers) into the stage S, gathered per
// group from S into A (tensor memory, as in the direct kernel), multiplied,
// written back into S by the owning threads and stored with coalesced
// 16-byte accesses. With two A and product buffers (NB = 2) a tile's
// products run while the previous tile is read back and stored. Small CTAs
// let several run per SM (four for K = 4, two for K = 5, as many as tensor
// memory holds), so one CTA's barriers overlap another's memory traffic. S position of tile element e: e ^ s(e), s(e) = (e >> 4 ^ e >> 8
// ^ e >> 12) & 15, which keeps element pairs (2v, 2v + 1) in one 16-byte
// slot (swapped when s(e) is odd) and spreads the group-parallel accesses
// over the banks.
__device__ __forceinline__ uint32_t stage_pos(uint32_t e) { return e ^ (((e >> 4) ^ (e >> 8) ^ (e >> 12)) & 15u); }

template <int K>
constexpr int tile_threads() {
  return 128 * (1 << K) / 16;
}

// Tensor-memory columns of one staged CTA: NB product buffers and NB A
// operand buffers of 2^(K+1) columns each (a power of two, at least 32).
template <int K, int NB>
constexpr uint32_t tile_tmem_cols() {
  return 2u * NB * (2u << K) < 32 ? 32 : 2u * NB * (2u << K);
}

template <int K, int NB>
__global__ void __launch_bounds__(tile_threads<K>(), 512 / tile_threads<K>()) k_dense_tc_tile(float2* __restrict__ psi,
                                                                     const DenseTcTileGeom g,
                                                                     const uint8_t* __restrict__ bmats,
                                                                     int* __restrict__ status) {
  constexpr uint32_t D = 1u << K, kd = 2u * D;
  constexpr int NT = tile_threads<K>();      // threads: 16 members of one group each
  constexpr uint32_t TILE = 128 * D;         // amplitudes per tile
  constexpr uint32_t BPART = kd * kd * 2;
  constexpr int TB = 7 + K;                  // tile bits
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ uint8_t tile[16];
  __shared__ uint64_t dep_hi[8];
  float2* stage = reinterpret_cast<float2*>(smem);                          // TILE complex64
  unsigned char* bmat = smem + size_t(TILE) * sizeof(float2);               // B hi, then B lo
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t r = uint32_t(tid) & 127u, chunk = uint32_t(tid) >> 7;

  if (tid == 0) {  // static indices: a parameter array indexed by tid would be copied to local memory
#pragma unroll
    for (int i = 0; i < 16; ++i) tile[i] = g.tile[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) dep_hi[i] = g.dep_hi[i];
  }
  {
    const uint4* src = reinterpret_cast<const uint4*>(bmats + g.b_offset);
    uint4* dst = reinterpret_cast<uint4*>(bmat);
    for (uint32_t i = tid; i < 2 * BPART / 16; i += NT) dst[i] = src[i];
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // NB product buffers (D) of kd columns, then NB operand buffers (A).
  constexpr uint32_t kCols = tile_tmem_cols<K, NB>();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  // Coalesced part: thread tid moves element pairs v = tid + NT j
  // (j = 0..7): tile bits 1..K+3 from tid, K+4..K+6 from j.
  uint64_t dep_t = 0, tmask = 0;
#pragma unroll
  for (int b = 1; b < K + 4; ++b)
    if ((uint32_t(tid) >> (b - 1)) & 1u) dep_t |= uint64_t(1) << tile[b];
#pragma unroll
  for (int b = 0; b < TB; ++b) tmask |= uint64_t(1) << tile[b];
  // Group part: this thread's members 16 * chunk + i of group r are tile
  // elements eg | tm(i), tm(i) depositing i into the four lowest target
  // positions.
  uint32_t eg = 0;
#pragma unroll
  for (int i = 0; i < 7; ++i)
    if ((r >> i) & 1u) eg |= 1u << g.fpos[i];
#pragma unroll
  for (int j = 4; j < K; ++j)
    if ((chunk >> (j - 4)) & 1u) eg |= 1u << g.tpos[j];
  const uint32_t t0 = 1u << g.tpos[0], t1 = 1u << g.tpos[1], t2 = 1u << g.tpos[2], t3 = 1u << g.tpos[3];
  auto member = [&](int i) -> uint32_t {
    return eg | ((i & 1) ? t0 : 0u) | ((i & 2) ? t1 : 0u) | ((i & 4) ? t2 : 0u) | ((i & 8) ? t3 : 0u);
  };
  const uint64_t my_iters = blockIdx.x < g.iters ? (g.iters - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // Tile bases in load order and in store order (running deposits of the
  // tile index into the bits outside the tile).
  const uint64_t dstep = insert_zeros(gridDim.x, tile, TB);
  uint64_t dload = insert_zeros(blockIdx.x, tile, TB), dstore = dload;
  auto load = [&](float4 (&x)[8]) {
    const uint64_t base = dload | dep_t;
    dload = dep_add(dload, dstep, tmask);
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = ld_early(psi + (base | dep_hi[j]));
  };
  const uint32_t lanes = (uint32_t(warp & 3) * 32u) << 16;
  int failed = 0;
  // One step: tile li into the stage and gathered into A, its products
  // issued; then the products of tile li - 1 (NB = 2; the MMA ran during
  // this step's first half) or of tile li itself (NB = 1) read back into
  // the stage and stored.
  auto step = [&](uint64_t li, float4 (&x)[8]) -> bool {
    const bool have = li < my_iters;
    const uint32_t b = NB == 2 ? uint32_t(li & 1) : 0u;
    const uint32_t acol = NB * kd + b * kd;  // this tile's A columns
    if (have) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t e = 2u * (uint32_t(tid) + uint32_t(NT) * uint32_t(j));
        const uint32_t pos = stage_pos(e);
        const float4 v = x[j];
        reinterpret_cast<float4*>(stage)[pos >> 1] = (pos & 1) ? make_float4(v.z, v.w, v.x, v.y) : v;
      }
      if (li + 2 < my_iters) load(x);
    }
    __syncthreads();
    if (have) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        float2 m[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) m[i] = stage[stage_pos(member(8 * q + i))];
        write_a8_tmem<K>(m, tmem + lanes + acol, chunk, q);
      }
      tmem_wait_st();
    }
    tc_fence_before();
    if (__syncthreads_or(failed)) return false;
    if (have && tid == 0) issue_products_tmem_a<K, 1>(tmem + acol, bmat, tmem + b * kd, smem_addr(&bar[b]));
    const bool back = NB == 2 ? li > 0 : have;
    if (back) {
      const uint64_t rl = NB == 2 ? li - 1 : li;
      const uint32_t rb = NB == 2 ? uint32_t(rl & 1) : 0u;
      const uint32_t parity = uint32_t((NB == 2 ? rl >> 1 : rl) & 1);
      if (!wait_products(smem_addr(&bar[rb]), parity)) {
        failed = 1;
        atomicExch(status, 1);
      } else {
        tc_fence_after();
        const uint32_t taddr = tmem + lanes + rb * kd + 16 * chunk;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          float re[8], im[8];
          tmem_ld8(taddr + 8 * hh, re);
          tmem_ld8(taddr + D + 8 * hh, im);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 8; ++i) stage[stage_pos(member(8 * hh + i))] = make_float2(re[i], im[i]);
        }
      }
    }
    tc_fence_before();
    if (__syncthreads_or(failed)) return false;
    if (back) {
      const uint64_t base = dstore | dep_t;
      dstore = dep_add(dstore, dstep, tmask);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t e = 2u * (uint32_t(tid) + uint32_t(NT) * uint32_t(j));
        const uint32_t pos = stage_pos(e);
        float4 v = reinterpret_cast<const float4*>(stage)[pos >> 1];
        if (pos & 1) v = make_float4(v.z, v.w, v.x, v.y);
        *reinterpret_cast<float4*>(psi + (base | dep_hi[j])) = v;
      }
    }
    __syncthreads();  // the stage is free for the next step
    return NB == 2 ? have : li + 1 < my_iters;
  };
  float4 xa[8], xb[8];
  if (my_iters > 0) load(xa);
  if (my_iters > 1) load(xb);
  if (my_iters > 0) {
    for (uint64_t li = 0;; li += 2) {
      if (!step(li, xa)) break;
      if (!step(li + 1, xb)) break;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
  }
}

template <int K, int VW>
void launch_k(StateImpl& s, const DenseTcGeom& g, const uint8_t* bmats) {
  const size_t smem = tc_gate_bytes(K);
  static bool configured = false;  // per instantiation
  if (!configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_dense_tc<K, VW>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    // The rest of the unified L1 / shared storage as L1, which holds the
    // global loads in flight.
    int dev = 0, smem_sm = 0;
    QVDG_CUDA(cudaGetDevice(&dev));
    QVDG_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    const int percent = int(std::min<size_t>(100, (100 * (smem + 4096) + size_t(smem_sm) - 1) / size_t(smem_sm)));
    QVDG_CUDA(cudaFuncSetAttribute(k_dense_tc<K, VW>, cudaFuncAttributePreferredSharedMemoryCarveout, percent));
    configured = true;
  }
  const unsigned grid = unsigned(std::min<uint64_t>(g.iters, uint64_t(s.sms)));
  k_dense_tc<K, VW><<<grid, kThreads, smem, s.stream>>>(static_cast<float2*>(s.amp), g, bmats, s.status);
  QVDG_LAUNCH_CHECK();
}

// Two A and product buffers in tensor memory: a tile's products run while
// the previous tile is read back and stored.
template <int K>
void launch_tile(StateImpl& s, const DenseTcTileGeom& g, const uint8_t* bmats) {
  constexpr int NB = 2;
  constexpr int NT = tile_threads<K>();
  const size_t smem = (size_t(128) << K) * sizeof(float2) + tc_gate_bytes(K);
  static int per_sm = 0;  // per instantiation
  if (!per_sm) {
    QVDG_CUDA(cudaFuncSetAttribute(k_dense_tc_tile<K, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    // All of the unified L1/shared storage as shared memory, so that several
    // CTAs fit (the default carveout leaves room for one).
    QVDG_CUDA(cudaFuncSetAttribute(k_dense_tc_tile<K, NB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   int(cudaSharedmemCarveoutMaxShared)));
    // CTAs per SM from the kernel's registers and shared memory (the
    // occupancy query reported one CTA here where four fit).
    cudaFuncAttributes fa{};
    QVDG_CUDA(cudaFuncGetAttributes(&fa, k_dense_tc_tile<K, NB>));
    int dev = 0, smem_sm = 0, regs_sm = 0;
    QVDG_CUDA(cudaGetDevice(&dev));
    QVDG_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    QVDG_CUDA(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    const int regs = (fa.numRegs + 7) / 8 * 8;
    const int by_smem = smem_sm / int(smem + fa.sharedSizeBytes + 1024);
    const int by_regs = regs_sm / (regs * NT);
    const int by_tmem = int(512 / tile_tmem_cols<K, NB>());
    per_sm = std::max(1, std::min({by_smem, by_regs, by_tmem, 2048 / NT}));
  }
  const unsigned grid = unsigned(std::min<uint64_t>(g.iters, uint64_t(s.sms) * uint64_t(per_sm)));
  k_dense_tc_tile<K, NB><<<grid, NT, smem, s.stream>>>(static_cast<float2*>(s.amp), g, bmats, s.status);
  QVDG_LAUNCH_CHECK();
}

}  // namespace

bool dense_tc_ok(uint32_t n, int bits, const std::vector<uint32_t>& targets, size_t controls) {
  if (bits != 32 || targets.size() < 4 || targets.size() > 6 || n < 13 + controls) return false;
  std::vector<uint32_t> t(targets);
  std::sort(t.begin(), t.end());
  return t[3] < 32;  // member offsets of the four lowest targets in 32 bits
}

bool dense_tc_staged(uint32_t n, const std::vector<uint32_t>& targets, size_t controls) {
  auto has = [&](uint32_t b) { return std::find(targets.begin(), targets.end(), b) != targets.end(); };
  // With bit 0 a target too, 6-qubit gates go faster on the direct kernel's
  // 32-byte accesses; narrower ones (several CTAs per SM here) on this one.
  return controls == 0 && n >= uint32_t(7 + targets.size()) && has(1) && has(2) && has(3) &&
         (targets.size() <= 5 || !has(0));
}

void launch_dense_tc(StateImpl& s, const PlainGate& pg, const uint8_t* tc_blob) {
  const int k = int(pg.targets.size()), c = int(pg.controls.size());
  if (!dense_tc_ok(s.n, s.bits, pg.targets, size_t(c)) || !std::is_sorted(pg.targets.begin(), pg.targets.end()))
    throw Error(QVDG_ERR_INVALID, "internal: gate does not fit the tensor-core plain pass");
  if (dense_tc_staged(s.n, pg.targets, size_t(c))) {
    // Bits 1-3 all targets: each group is a contiguous run of at least 8
    // amplitudes and the direct kernel's warps stride by that run, so the
    // state goes through the shared-memory stage. With fewer low targets,
    // and for 6-qubit gates that also target bit 0, the direct kernel is
    // faster (measured on the 30-qubit grid circuit).
    DenseTcTileGeom tg{};
    std::vector<uint32_t> bits(pg.targets.begin(), pg.targets.end());
    const int tb = 7 + k;
    for (uint32_t b = 0; int(bits.size()) < tb; ++b)
      if (std::find(pg.targets.begin(), pg.targets.end(), b) == pg.targets.end()) bits.push_back(b);
    std::sort(bits.begin(), bits.end());
    for (int i = 0; i < tb; ++i) tg.tile[i] = uint8_t(bits[i]);
    int nf = 0;
    for (int i = 0; i < tb; ++i) {
      const auto it = std::find(pg.targets.begin(), pg.targets.end(), bits[i]);
      if (it == pg.targets.end())
        tg.fpos[nf++] = uint8_t(i);
      else
        tg.tpos[it - pg.targets.begin()] = uint8_t(i);
    }
    for (int j = 0; j < 8; ++j)
      for (int b = 0; b < 3; ++b)
        if ((j >> b) & 1) tg.dep_hi[j] |= uint64_t(1) << bits[k + 4 + b];
    tg.iters = uint64_t(1) << (s.n - uint32_t(tb));
    tg.b_offset = uint32_t(pg.tc_offset);
    switch (k) {
      case 4: return launch_tile<4>(s, tg, tc_blob);
      case 5: return launch_tile<5>(s, tg, tc_blob);
      default: return launch_tile<6>(s, tg, tc_blob);
    }
  }
  DenseTcGeom g{};
  std::vector<uint8_t> fixed;
  for (auto& cv : pg.controls) {
    fixed.push_back(uint8_t(cv.first));
    if (cv.second) g.control_value |= uint64_t(1) << cv.first;
  }
  for (uint32_t t : pg.targets) fixed.push_back(uint8_t(t));
  std::sort(fixed.begin(), fixed.end());
  g.num_fixed = int(fixed.size());
  for (size_t i = 0; i < fixed.size(); ++i) g.fixed[i] = fixed[i];
  for (int h = 0; h < (1 << k); ++h) {
    uint64_t o = 0;
    for (int j = 0; j < k; ++j) o |= uint64_t((h >> j) & 1) << pg.targets[j];
    g.offsets[h] = o;
  }
  g.iters = (uint64_t(1) << (s.n - uint32_t(k) - uint32_t(c))) / (kIterAmps >> k);
  g.b_offset = uint32_t(pg.tc_offset);
  // Members 2m and 2m + 1 are neighbours when targets[0] is bit 0 (the
  // lowering sorts targets ascending).
  // Access width: members 4m..4m+3 are neighbours when bits 0 and 1 are
  // both targets (32-byte accesses), 2m and 2m+1 when bit 0 is (16-byte).
  const int vw = pg.targets[0] == 0 ? (pg.targets[1] == 1 ? 4 : 2) : 1;
  auto go = [&](auto kk) {
    constexpr int KK = decltype(kk)::value;
    if (vw == 4) return launch_k<KK, 4>(s, g, tc_blob);
    if (vw == 2) return launch_k<KK, 2>(s, g, tc_blob);
    return launch_k<KK, 1>(s, g, tc_blob);
  };
  switch (k) {
    case 4: return go(std::integral_constant<int, 4>());
    case 5: return go(std::integral_constant<int, 5>());
    default: return go(std::integral_constant<int, 6>());
  }
}

}  // namespace qvdg
