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
// members pair into 16-byte accesses), writes their bf16 parts into one of
// two A buffers, and, once TMEM lane r holds the block's products, reads
// its 16 members back and stores them where they came from. The loads of
// iteration i + 1 are issued before iteration i's products, and iteration
// i's read-back runs during iteration i + 1, so HBM traffic, the bf16 split,
// the tensor cores and the stores overlap. Every wait on an MMA completion
// barrier is bounded: on timeout the kernel records an error, every thread
// leaves the loop at the next CTA barrier and the tensor memory is freed.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "dense_tc.hpp"
#include "stage_kernel.hpp"
#include "tc_ptx.cuh"

namespace qvdg {

namespace {

constexpr int kThreads = 512;
constexpr uint32_t kIterAmps = 8192;
constexpr uint32_t kPartBytes = kIterAmps * 2 * 2;  // one bf16 part (hi or lo) of an iteration's A
constexpr uint32_t kTmemCols = 256;                 // two buffers of 128 fp32 columns

template <int K, bool PAIR>
__global__ void __launch_bounds__(kThreads, 1) k_dense_tc(float2* __restrict__ psi, const DenseTcGeom g,
                                                          const uint8_t* __restrict__ bmats,
                                                          int* __restrict__ status) {
  constexpr uint32_t D = 1u << K, kd = 2u * D;
  constexpr uint32_t P = D / 16;     // threads per group
  constexpr uint32_t T = 4 / P;      // blocks of 128 groups per iteration
  constexpr uint32_t GPI = T * 128;  // groups per iteration
  constexpr uint32_t SBO = kd * 16;
  constexpr uint32_t BLOCK = 128 * kd * 2;  // bytes of one block's A part
  constexpr uint32_t BPART = kd * kd * 2;   // bytes of one part of B
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ uint8_t fixed[40];
  unsigned char* abuf = smem;                  // buffer b: hi at 2b * kPartBytes, lo right after
  unsigned char* bmat = smem + 4 * kPartBytes;  // B hi, then B lo
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
  auto base_of = [&](uint64_t li) -> uint64_t {
    const uint64_t it = blockIdx.x + li * gridDim.x;
    return insert_zeros(it * GPI, fixed, g.num_fixed) | tdep;
  };
  auto load = [&](float2 (&x)[16], uint64_t base) {
    if constexpr (PAIR) {
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
  const uint32_t row = blk * BLOCK + (r >> 3) * SBO + (r & 7) * 16;
  const uint32_t lanes = (uint32_t(warp & 3) * 32u) << 16;
  int failed = 0;
  // One step: iteration li's members into A and its products issued (the
  // registers then take the loads of iteration li + 2), and the previous
  // iteration read back and stored. Returns whether another step follows.
  auto step = [&](uint64_t li, float2 (&x)[16]) -> bool {
    const uint32_t b = uint32_t(li & 1);
    unsigned char* ah = abuf + b * 2 * kPartBytes;
    unsigned char* al = ah + kPartBytes;
    if (li < my_iters) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        float re[8], im[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          re[i] = x[8 * q + i].x;
          im[i] = x[8 * q + i].y;
        }
        uint4 h, l;
        const uint32_t cre = (2 * chunk + q) * 128, cim = (D / 8 + 2 * chunk + q) * 128;
        split8(re, h, l);
        *reinterpret_cast<uint4*>(ah + row + cre) = h;
        *reinterpret_cast<uint4*>(al + row + cre) = l;
        split8(im, h, l);
        *reinterpret_cast<uint4*>(ah + row + cim) = h;
        *reinterpret_cast<uint4*>(al + row + cim) = l;
      }
      if (li + 2 < my_iters) load(x, base_of(li + 2));
      fence_async_shared();
    }
    tc_fence_before();
    if (__syncthreads_or(failed)) return false;
    if (li < my_iters && tid == 0) {
      tc_fence_after();
      const uint32_t idesc = umma_idesc(kd);
      const uint64_t dah = umma_desc(smem_addr(ah), 128, SBO), dal = umma_desc(smem_addr(al), 128, SBO);
      const uint64_t dbh = umma_desc(smem_addr(bmat), 128, SBO), dbl = umma_desc(smem_addr(bmat + BPART), 128, SBO);
#pragma unroll
      for (uint32_t t = 0; t < T; ++t) {
        const uint32_t d = tmem + b * 128 + t * kd;
        const uint64_t boff = (t * BLOCK) >> 4;
        uint32_t acc = 0;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint64_t a0 = (p == 2 ? dal : dah) + boff, b0 = p == 1 ? dbl : dbh;
#pragma unroll
          for (uint32_t s = 0; s < kd / 16; ++s) {
            umma_bf16(d, a0 + 16 * s, b0 + 16 * s, idesc, acc);
            acc = 1;
          }
        }
      }
      umma_commit(smem_addr(&bar[b]));
    }
    if (li > 0) {
      const uint32_t pb = b ^ 1u;
      const uint32_t parity = uint32_t(((li - 1) >> 1) & 1);
      const uint32_t barp = smem_addr(&bar[pb]);
      const uint64_t base = base_of(li - 1);
      const long long t0 = clock64();
      bool done = mbar_try_wait(barp, parity);
      while (!done && clock64() - t0 <= kWaitCycles) done = mbar_try_wait(barp, parity);
      if (!done) {
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
          if constexpr (PAIR) {
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
  if (my_iters > 0) load(xa, base_of(0));
  if (my_iters > 1) load(xb, base_of(1));
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

template <int K, bool PAIR>
void launch_k(StateImpl& s, const DenseTcGeom& g, const uint8_t* bmats) {
  const size_t smem = 4 * size_t(kPartBytes) + tc_gate_bytes(K);
  static bool configured = false;  // per instantiation
  if (!configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_dense_tc<K, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    configured = true;
  }
  const unsigned grid = unsigned(std::min<uint64_t>(g.iters, uint64_t(s.sms)));
  k_dense_tc<K, PAIR><<<grid, kThreads, smem, s.stream>>>(static_cast<float2*>(s.amp), g, bmats, s.status);
  QVDG_LAUNCH_CHECK();
}

}  // namespace

bool dense_tc_ok(uint32_t n, int bits, const std::vector<uint32_t>& targets, size_t controls) {
  if (bits != 32 || targets.size() < 4 || targets.size() > 6 || n < 13 + controls) return false;
  std::vector<uint32_t> t(targets);
  std::sort(t.begin(), t.end());
  return t[3] < 32;  // member offsets of the four lowest targets in 32 bits
}

void launch_dense_tc(StateImpl& s, const PlainGate& pg, const uint8_t* tc_blob) {
  const int k = int(pg.targets.size()), c = int(pg.controls.size());
  if (!dense_tc_ok(s.n, s.bits, pg.targets, size_t(c)) || !std::is_sorted(pg.targets.begin(), pg.targets.end()))
    throw Error(QVDG_ERR_INVALID, "internal: gate does not fit the tensor-core plain pass");
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
  const bool pair = pg.targets[0] == 0;
  switch (k) {
    case 4: return pair ? launch_k<4, true>(s, g, tc_blob) : launch_k<4, false>(s, g, tc_blob);
    case 5: return pair ? launch_k<5, true>(s, g, tc_blob) : launch_k<5, false>(s, g, tc_blob);
    default: return pair ? launch_k<6, true>(s, g, tc_blob) : launch_k<6, false>(s, g, tc_blob);
  }
}

}  // namespace qvdg
