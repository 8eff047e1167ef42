// Two fused 6-qubit gates in one plain pass over a complex64 state, on the
// tensor cores: the reference applies each fused op as its own sweep over
// the state (src/simulator.rs:136-143, src/kernels.rs:252-473); here two
// consecutive fused gates share one HBM pass, so a plan of plain fused
// passes moves the state about half as often.
//
// An iteration covers the 8192 amplitudes spanned by 13 bits I: the
// targets of both gates and the lowest other bits. Gate 1 sees them as 128
// groups of 64 members (groups over I minus its targets), gate 2 as another
// 128 groups. Persistent CTAs of 16 compute warps and one issuing
// warpgroup; compute thread (w, r) owns 16 members of group r for either
// gate (w / 4 picks which 16), as in the single-gate kernel (dense_tc.cu),
// and tensor-memory lane r holds group r:
//
//   1. gate 1's members come from HBM (loaded two iterations ahead into
//      registers), are split into bf16 high and low parts and written to
//      the A operand in tensor memory; the issuing thread then runs the
//      products A_hi B1_hi + A_hi B1_lo + A_lo B1_hi (fp32 accumulation);
//   2. the products are read back (tcgen05.ld) and written into a 64 KB
//      shared-memory buffer at the amplitudes' positions in I; after a
//      barrier of the compute warps every thread reads its 16 members of
//      gate 2's group r from it, splits them into the same A operand, and
//      the products with B2 run;
//   3. gate 2's products are read back and stored to HBM where gate 2's
//      members lie.
//
// Two iterations are in flight, each with its own tensor-memory slot (A and
// D, 128 columns each), so that the compute warps' work on one slot
// overlaps the products of the other. The products are issued by a thread
// of their own because issuing holds that thread until the tensor cores
// have nearly finished them (measured on B200: 24 products of M = N = 128,
// K = 16 keep the issuing thread about as long as they run, about 67 cycles
// each). Compute warps and the issuing thread hand slots to each other
// through mbarriers: the compute warps arrive on "ready" barriers, the
// products complete "done" barriers (tcgen05.commit). Positions in the
// transpose buffer are XOR-swizzled (low four index bits with a host-chosen
// linear map of the high ones) so that both gates' group-parallel accesses
// hit distinct banks. Every wait is bounded: on timeout the kernel records
// an error, every thread leaves its loop, and the tensor memory is freed
// after a bounded wait for the products still in flight.

#include <cuda_runtime.h>

#include <algorithm>
#include <random>

#include "dense_tc.hpp"
#include "dense_tc_common.cuh"
#include "stage_kernel.hpp"

namespace qvdg {

namespace {

constexpr uint32_t kPairBytes = 64 * 1024;  // one 6-qubit gate's bf16 matrices (hi and lo)
constexpr uint32_t kXBytes = kIterAmps * 8;  // the transpose buffer: one iteration in complex64

template <int VW>
__device__ __forceinline__ void load16(const float2* psi, uint64_t base, const uint32_t* lo, float2 (&x)[16]) {
  if constexpr (VW == 4) {
#pragma unroll
    for (int m = 0; m < 4; ++m) ld_early32(psi + base + lo[4 * m], &x[4 * m]);
  } else if constexpr (VW == 2) {
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const float4 v = ld_early(psi + base + lo[2 * m]);
      x[2 * m] = make_float2(v.x, v.y);
      x[2 * m + 1] = make_float2(v.z, v.w);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = ld_early8(psi + base + lo[i]);
  }
}

// Eight members 8 hh .. 8 hh + 7 of one group from registers to HBM.
template <int VW>
__device__ __forceinline__ void store8(float2* psi, uint64_t base, const uint32_t* lo, int hh, const float* re,
                                       const float* im) {
  if constexpr (VW == 4) {
#pragma unroll
    for (int m = 0; m < 2; ++m) st32(psi + base + lo[8 * hh + 4 * m], re + 4 * m, im + 4 * m);
  } else if constexpr (VW == 2) {
#pragma unroll
    for (int m = 0; m < 4; ++m)
      *reinterpret_cast<float4*>(psi + base + lo[8 * hh + 2 * m]) =
          make_float4(re[2 * m], im[2 * m], re[2 * m + 1], im[2 * m + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) psi[base + lo[8 * hh + i]] = make_float2(re[i], im[i]);
  }
}

// Threads: 16 compute warps (512 threads: group r = tid % 128, member
// chunk tid / 128) and a fifth warpgroup whose first thread issues the
// products (an issuing thread is held until its products are nearly done,
// so it does nothing else). Launched at 96 registers a thread (640 x 96 =
// 61440); the issuing warpgroup keeps 32 and the compute warps take 112
// (128 x 32 + 512 x 112 = 61440).
constexpr int kPairThreads = kThreads + 128;
constexpr uint32_t kIssueRegs = 32, kComputeRegs = 112;
constexpr uint32_t kComputeWarps = kThreads / 32;

// Barrier among the 512 compute threads (named barrier 1), returning
// whether any of them passed a nonzero `flag`.
__device__ __forceinline__ bool compute_sync_or(int flag) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"(flag), "n"(kThreads)
      : "memory");
  return out != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for a barrier phase that also gives up when another thread
// of the CTA has raised `abort` (then or on its own timeout it returns
// false; a timeout raises `abort` and the status word).
__device__ __forceinline__ bool wait_or_abort(uint32_t bar, uint32_t parity, volatile int* abort, int* status) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort) return false;
    if (clock64() - t0 > kWaitCycles) {
      *abort = 1;
      atomicExch(status, 1);
      return false;
    }
  }
  return true;
}

// Gate products of one slot, D = A_hi B_hi + A_hi B_lo + A_lo B_hi with A
// in tensor memory (`acol`: A_hi, A_lo 64 columns later), B in shared
// memory (hi, then lo), fp32 into `dcol`; then one commit to `bar`. The 24
// instructions are unrolled: measured on B200 with other warps streaming
// tensor-memory stores, a rolled issue loop let each product take up to 95
// cycles, the unrolled sequence 64-68 (and a commit per product instead of
// per gate serialises them at about 300 cycles each).
__device__ __forceinline__ void issue_pair_products(uint32_t acol, const unsigned char* bmat, uint32_t dcol,
                                                    uint32_t bar) {
  constexpr uint32_t kd = 128, SBO = kd * 16, BPART = kd * kd * 2;
  tc_fence_after();
  const uint32_t idesc = umma_idesc(kd);
  uint64_t dbh = umma_desc(smem_addr(bmat), 128, SBO), dbl = umma_desc(smem_addr(bmat + BPART), 128, SBO);
  // Opaque here, so that the 24 operands are formed at each call, one by
  // one, rather than all hoisted out of the caller's loop.
  asm volatile("" : "+l"(dbh), "+l"(dbl), "+r"(acol));
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const uint32_t a0 = acol + (p == 2 ? 64u : 0u);
    const uint64_t b0 = p == 1 ? dbl : dbh;
#pragma unroll
    for (uint32_t s = 0; s < kd / 16; ++s) umma_bf16_tmem_a(dcol, a0 + 8 * s, b0 + 16 * s, idesc, (p | s) != 0);
  }
  umma_commit(bar);
}

template <int VW1, int VW2>
__global__ void __launch_bounds__(kPairThreads, 1) k_dense_tc_pair(float2* __restrict__ psi, const DenseTcPairGeom g,
                                                                   const uint8_t* __restrict__ bmats,
                                                                   int* __restrict__ status) {
  constexpr uint32_t D = 64;
  extern __shared__ __align__(1024) unsigned char smem[];
  // ready*: the compute warps' operands (and freed products) of a slot are
  // in place for gate 1's / gate 2's products; done*: those products
  // completed (tcgen05.commit).
  __shared__ __align__(8) uint64_t ready1[2], ready2[2], done1[2], done2[2];
  __shared__ uint32_t tmem_slot;
  __shared__ uint8_t ibits[16];
  __shared__ volatile int abort;
  unsigned char* bmat1 = smem;                                        // gate 1: B hi, then B lo
  unsigned char* bmat2 = smem + kPairBytes;                           // gate 2
  unsigned char* xbytes = smem + 2 * kPairBytes;                    // 8192 complex64, byte offsets
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t r = uint32_t(tid) & 127u, chunk = uint32_t(tid) >> 7;

  if (tid < 16) ibits[tid] = g.ibits[tid];
  if (tid == 0) abort = 0;
  {
    const uint4* s1 = reinterpret_cast<const uint4*>(bmats + g.b1_offset);
    const uint4* s2 = reinterpret_cast<const uint4*>(bmats + g.b2_offset);
    uint4* d1 = reinterpret_cast<uint4*>(bmat1);
    uint4* d2 = reinterpret_cast<uint4*>(bmat2);
    for (uint32_t i = tid; i < kPairBytes / 16; i += kPairThreads) {
      d1[i] = s1[i];
      d2[i] = s2[i];
    }
  }
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&ready1[b])), "n"(kComputeWarps));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&ready2[b])), "n"(kComputeWarps));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&done1[b])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&done2[b])));
    }
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
  const uint64_t my_iters = blockIdx.x < g.iters ? (g.iters - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint64_t periods = (my_iters + 1) / 2;

  // Period j runs iterations a = 2j (slot 0) and b = 2j + 1 (slot 1). The
  // issuing thread takes, in order, M1(a), M1(b), M2(a), M2(b), each once
  // its slot's compute warps have arrived on the ready barrier; the
  // compute warps meanwhile
  //   1. store a - 2 (slot 0) and put gate 1 of a into A  -> ready1[0]
  //   2. store b - 2 (slot 1) and put gate 1 of b into A  -> ready1[1]
  //   3. transpose a into gate 2's groups in A             -> ready2[0]
  //   4. transpose b                                      -> ready2[1]
  // so every step's SM work overlaps a product issued earlier, and no
  // compute warp waits for the issue of a product.
  if (warp >= int(kComputeWarps)) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kIssueRegs));
    if (tid == kThreads) {
      uint32_t n10 = 0, n11 = 0, n20 = 0, n21 = 0;  // products issued per slot and gate
      const uint32_t iters32 = uint32_t(my_iters), periods32 = uint32_t(periods);  // at most 2^27 (n <= 40)
#pragma unroll 1
      for (uint32_t j = 0; j < periods32; ++j) {
        const bool hb = 2 * j + 1 < iters32;
        const uint32_t par = j & 1;
        if (!wait_or_abort(smem_addr(&ready1[0]), par, &abort, status)) break;
        issue_pair_products(tmem + kTmemA, bmat1, tmem, smem_addr(&done1[0]));
        ++n10;
        if (hb) {
          if (!wait_or_abort(smem_addr(&ready1[1]), par, &abort, status)) break;
          issue_pair_products(tmem + kTmemA + 128, bmat1, tmem + 128, smem_addr(&done1[1]));
          ++n11;
        }
        if (!wait_or_abort(smem_addr(&ready2[0]), par, &abort, status)) break;
        issue_pair_products(tmem + kTmemA, bmat2, tmem, smem_addr(&done2[0]));
        ++n20;
        if (hb) {
          if (!wait_or_abort(smem_addr(&ready2[1]), par, &abort, status)) break;
          issue_pair_products(tmem + kTmemA + 128, bmat2, tmem + 128, smem_addr(&done2[1]));
          ++n21;
        }
      }
      // Every issued product completes before the tensor memory is freed
      // (bounded: after a timeout a barrier may never complete).
      if (n10 > 0) wait_products(smem_addr(&done1[0]), (n10 - 1) & 1);
      if (n11 > 0) wait_products(smem_addr(&done1[1]), (n11 - 1) & 1);
      if (n20 > 0) wait_products(smem_addr(&done2[0]), (n20 - 1) & 1);
      if (n21 > 0) wait_products(smem_addr(&done2[1]), (n21 - 1) & 1);
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kComputeRegs));
    const uint32_t lanes = (uint32_t(warp & 3) * 32u) << 16;
    // This thread's group r and member chunk (members 16 chunk .. + 15), for
    // either gate: HBM offset of its group and chunk, and its position
    // (swizzled) in the transpose buffer; member i adds lo*[i] / XORs llo*[i].
    uint64_t gb1 = chunk == 0 ? g.hi1[0] : chunk == 1 ? g.hi1[1] : chunk == 2 ? g.hi1[2] : g.hi1[3];
    uint64_t gb2 = chunk == 0 ? g.hi2[0] : chunk == 1 ? g.hi2[1] : chunk == 2 ? g.hi2[2] : g.hi2[3];
    uint32_t lb1 = chunk == 0 ? g.lhi1[0] : chunk == 1 ? g.lhi1[1] : chunk == 2 ? g.lhi1[2] : g.lhi1[3];
    uint32_t lb2 = chunk == 0 ? g.lhi2[0] : chunk == 1 ? g.lhi2[1] : chunk == 2 ? g.lhi2[2] : g.lhi2[3];
#pragma unroll
    for (int j = 0; j < 7; ++j)
      if ((r >> j) & 1u) {
        gb1 += g.grp1[j];
        gb2 += g.grp2[j];
        lb1 ^= g.lgrp1[j];
        lb2 ^= g.lgrp2[j];
      }
    // Iteration bases (the bits outside I), advanced by a running deposit
    // in iteration order, one for the loads and one for the stores.
    const uint64_t dstep = insert_zeros(gridDim.x, ibits, 13);
    uint64_t dload = insert_zeros(blockIdx.x, ibits, 13), dstore = dload, dpre = dload;
    int failed = 0;

    auto load = [&](float2 (&x)[16]) {
      load16<VW1>(psi, dload + gb1, g.lo1, x);
      dload = dep_add(dload, dstep, g.imask);
    };
    // Warp-uniform wait (tcgen05.ld and .st after it are warp-wide).
    auto wait = [&](uint64_t* bar, uint32_t parity) {
      const bool ok = __all_sync(0xffffffffu, wait_or_abort(smem_addr(bar), parity, &abort, status));
      if (!ok) failed = 1;
      return ok;
    };
    // The warp's tensor-memory writes and reads are done: one arrival.
    auto arrive = [&](uint64_t* bar) {
      tc_fence_before();
      __syncwarp();
      if ((tid & 31) == 0) mbar_arrive(smem_addr(bar));
    };
    // Gate 2's products in slot s (the next iteration in store order) to HBM.
    auto store_slot = [&](uint32_t s, uint32_t parity) {
      const uint64_t base = dstore + gb2;
      dstore = dep_add(dstore, dstep, g.imask);
      if (failed || !wait(&done2[s], parity)) return;
      tc_fence_after();
      const uint32_t taddr = tmem + lanes + s * 128 + 16 * chunk;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        float re[8], im[8];
        tmem_ld8(taddr + 8 * hh, re);
        tmem_ld8(taddr + D + 8 * hh, im);
        tmem_wait_ld();
        store8<VW2>(psi, base, g.lo2, hh, re, im);
      }
    };
    auto write_gate1 = [&](uint32_t s, float2 (&x)[16], bool more) {
      if (failed) return;
      const uint32_t acol = tmem + lanes + kTmemA + s * 128;
      write_a8_tmem<6>(x, acol, chunk, 0);
      write_a8_tmem<6>(x + 8, acol, chunk, 1);
      if (more) load(x);
      tmem_wait_st();
    };
    // Gate 1's products in slot s through the transpose buffer into gate
    // 2's groups in slot s's A; false when the CTA stops.
    auto transpose = [&](uint32_t s, uint32_t parity) -> bool {
      if (!failed && wait(&done1[s], parity)) {
        tc_fence_after();
        const uint32_t taddr = tmem + lanes + s * 128 + 16 * chunk;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          float re[8], im[8];
          tmem_ld8(taddr + 8 * hh, re);
          tmem_ld8(taddr + D + 8 * hh, im);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 8; ++i)
            *reinterpret_cast<float2*>(xbytes + (lb1 ^ g.llo1[8 * hh + i])) = make_float2(re[i], im[i]);
        }
      }
      if (compute_sync_or(failed)) return false;
      const uint32_t acol = tmem + lanes + kTmemA + s * 128;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        float2 m[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) m[i] = *reinterpret_cast<const float2*>(xbytes + (lb2 ^ g.llo2[8 * q + i]));
        write_a8_tmem<6>(m, acol, chunk, q);
      }
      tmem_wait_st();
      arrive(&ready2[s]);
      // The buffer is free for the next transpose once every warp read it.
      return !compute_sync_or(0);
    };

    float2 xa[16], xb[16];
    if (my_iters > 0) load(xa);
    if (my_iters > 1) load(xb);
    for (uint64_t j = 0; j < periods; ++j) {
      const bool hb = 2 * j + 1 < my_iters;
      const uint32_t par = uint32_t(j & 1), ppar = uint32_t((j + 1) & 1);
      if (j > 0) store_slot(0, ppar);
      write_gate1(0, xa, 2 * j + 2 < my_iters);
      arrive(&ready1[0]);
      if (j > 0) store_slot(1, ppar);
      if (hb) {
        write_gate1(1, xb, 2 * j + 3 < my_iters);
        arrive(&ready1[1]);
      }
      if (!transpose(0, par)) {
        failed = 1;
        break;
      }
      if (hb && !transpose(1, par)) {
        failed = 1;
        break;
      }
    }
    if (!failed && periods > 0) {
      const uint32_t last = uint32_t((periods - 1) & 1);
      store_slot(0, last);
      if (my_iters % 2 == 0) store_slot(1, last);
    }
    if (failed) abort = 1;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

template <int VW1, int VW2>
void launch_pair(StateImpl& s, const DenseTcPairGeom& g, const uint8_t* bmats) {
  const size_t smem = 2 * size_t(kPairBytes) + kXBytes;
  static bool configured = false;  // per instantiation
  if (!configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_dense_tc_pair<VW1, VW2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(smem)));
    // The register split (setmaxnreg) must fit in what the CTA is launched
    // with, or the compute warps would wait for registers forever.
    cudaFuncAttributes fa{};
    QVDG_CUDA(cudaFuncGetAttributes(&fa, k_dense_tc_pair<VW1, VW2>));
    if (uint64_t(fa.numRegs) * kPairThreads < uint64_t(kThreads) * kComputeRegs + 128ull * kIssueRegs)
      throw Error(QVDG_ERR_INVALID, "internal: pair kernel compiled with too few registers for its register split");
    configured = true;
  }
  const unsigned grid = unsigned(std::min<uint64_t>(g.iters, uint64_t(s.sms)));
  k_dense_tc_pair<VW1, VW2><<<grid, kPairThreads, smem, s.stream>>>(static_cast<float2*>(s.amp), g, bmats, s.status);
  QVDG_LAUNCH_CHECK();
}

template <int VW1>
void launch_pair_vw2(StateImpl& s, const DenseTcPairGeom& g, const uint8_t* bmats) {
  if (g.vw2 == 4) return launch_pair<VW1, 4>(s, g, bmats);
  if (g.vw2 == 2) return launch_pair<VW1, 2>(s, g, bmats);
  return launch_pair<VW1, 1>(s, g, bmats);
}

}  // namespace

namespace {

// The 13 bits of a pair's iteration: both gates' targets and the lowest
// other bits.
std::vector<uint32_t> pair_bits(const std::vector<uint32_t>& t1, const std::vector<uint32_t>& t2) {
  uint64_t imask = 0;
  for (uint32_t q : t1) imask |= uint64_t(1) << q;
  for (uint32_t q : t2) imask |= uint64_t(1) << q;
  for (uint32_t q = 0; __builtin_popcountll(imask) < 13; ++q) imask |= uint64_t(1) << q;
  std::vector<uint32_t> bits;
  for (uint32_t q = 0; q < 64; ++q)
    if ((imask >> q) & 1) bits.push_back(q);
  return bits;
}

// Whether a warp's HBM accesses for one gate of a pair stay coalesced: its
// 32 lanes take the gate's 32 lowest groups (the five lowest bits of the
// iteration outside its targets), each lane one member vector (1, 2 or 4
// neighbouring amplitudes). Coalesced: the lanes' vectors form contiguous
// runs of at least 8 amplitudes (64 bytes), or of at least 4 within 2048
// amplitudes. Elsewhere a warp touches many scattered sectors and the pass
// runs several times slower than two single passes (measured at 30 qubits;
// pairs within the rule took 3.5-4.9 ms against 2.6-3.0 ms per single pass).
// `t`: the gate's physical targets, `imask`: the iteration's bits.
bool pair_gate_coalesced(uint64_t t, uint64_t imask) {
  const uint32_t vw = (t & 1) ? ((t & 2) ? 4u : 2u) : 1u;
  uint64_t rest = imask & ~t, lanes = 0;
  for (int k = 0; k < 5 && rest; ++k) {
    const uint64_t low = rest & (~rest + 1);
    lanes |= low;
    rest ^= low;
  }
  const uint32_t next = vw == 4 ? 2u : (vw == 2 ? 1u : 0u);
  // Lane bits next, next + 1, ... each double the contiguous run.
  const uint32_t k = uint32_t(__builtin_ctzll(~(lanes >> next)));
  const uint32_t run = vw << std::min(k, 5u);
  const uint32_t last = lanes ? uint32_t(63 - __builtin_clzll(lanes)) : 0u;
  return run >= 8 || (run >= 4 && last <= 11);
}

}  // namespace

bool dense_tc_pair_masks_ok(uint64_t m1, uint64_t m2) {
  if (__builtin_popcountll(m1) != 6 || __builtin_popcountll(m2) != 6) return false;
  uint64_t imask = m1 | m2;  // both gates' targets and the lowest other bits, 13 in all
  while (__builtin_popcountll(imask) < 13) imask |= ~imask & (imask + 1);
  return pair_gate_coalesced(m1, imask) && pair_gate_coalesced(m2, imask);
}

bool dense_tc_pair_ok(uint32_t n, int bits, const std::vector<uint32_t>& t1, const std::vector<uint32_t>& t2) {
  if (bits != 32 || n < 14 || t1.size() != 6 || t2.size() != 6) return false;
  if (!dense_tc_ok(n, bits, t1, 0) || !dense_tc_ok(n, bits, t2, 0)) return false;
  uint64_t m1 = 0, m2 = 0;
  for (uint32_t q : t1) m1 |= uint64_t(1) << q;
  for (uint32_t q : t2) m2 |= uint64_t(1) << q;
  return dense_tc_pair_masks_ok(m1, m2);
}

DenseTcPairGeom dense_tc_pair_geom(uint32_t n, const std::vector<uint32_t>& t1, const std::vector<uint32_t>& t2,
                                   size_t b1_offset, size_t b2_offset) {
  if (!std::is_sorted(t1.begin(), t1.end()) || !std::is_sorted(t2.begin(), t2.end()) ||
      !dense_tc_pair_ok(n, 32, t1, t2))
    throw Error(QVDG_ERR_INVALID, "internal: gates do not fit the tensor-core pair pass");
  DenseTcPairGeom g{};
  // I: both gates' targets and the lowest other bits, 13 in all.
  const std::vector<uint32_t> ibits = pair_bits(t1, t2);
  uint64_t imask = 0;
  for (uint32_t q : ibits) imask |= uint64_t(1) << q;
  g.imask = imask;
  for (int i = 0; i < 13; ++i) g.ibits[i] = uint8_t(ibits[i]);
  g.iters = uint64_t(1) << (n - 13);
  auto local = [&](uint32_t q) { return uint32_t(std::find(ibits.begin(), ibits.end(), q) - ibits.begin()); };
  // Group bits of each gate: I minus its targets, ascending.
  std::vector<uint32_t> grp[2];
  const std::vector<uint32_t>* tg[2] = {&t1, &t2};
  for (int k = 0; k < 2; ++k)
    for (uint32_t q : ibits)
      if (std::find(tg[k]->begin(), tg[k]->end(), q) == tg[k]->end()) grp[k].push_back(q);
  // The swizzle: local index e at position e ^ L(e >> 4), L linear with
  // columns v[p] for local bits p = 4..12. A half-warp's 16 lanes step over
  // a gate's four lowest group bits; they hit distinct bank pairs when
  // those bits' low nibbles after swizzling are linearly independent.
  uint32_t v[13] = {};
  auto nib = [&](uint32_t p) { return p < 4 ? (1u << p) : v[p]; };
  auto independent = [&](const std::vector<uint32_t>& gr) {
    uint32_t span = 1;  // bit x set: nibble x reachable
    for (int j = 0; j < 4; ++j) {
      const uint32_t w = nib(local(gr[j]));
      if ((span >> w) & 1) return false;
      uint32_t next = span;
      for (uint32_t x = 0; x < 16; ++x)
        if ((span >> x) & 1) next |= 1u << (x ^ w);
      span = next;
    }
    return true;
  };
  std::mt19937 rng(12345);
  bool ok = false;
  for (int attempt = 0; attempt < 4096 && !ok; ++attempt) {
    for (uint32_t p = 4; p < 13; ++p) v[p] = attempt == 0 ? 0u : uint32_t(rng() & 15u);
    ok = independent(grp[0]) && independent(grp[1]);
  }
  if (!ok)
    for (uint32_t p = 4; p < 13; ++p) v[p] = 0;  // still correct, with bank conflicts
  auto swz = [&](uint32_t e) {
    uint32_t out = e;
    for (uint32_t p = 4; p < 13; ++p)
      if ((e >> p) & 1) out ^= v[p];
    return out;
  };
  for (int k = 0; k < 2; ++k) {
    const std::vector<uint32_t>& t = *tg[k];
    uint64_t* grp_off = k == 0 ? g.grp1 : g.grp2;
    uint32_t* lgrp = k == 0 ? g.lgrp1 : g.lgrp2;
    for (int j = 0; j < 7; ++j) {
      grp_off[j] = uint64_t(1) << grp[k][j];
      lgrp[j] = 8 * swz(1u << local(grp[k][j]));
    }
    uint64_t* hi = k == 0 ? g.hi1 : g.hi2;
    uint32_t* lhi = k == 0 ? g.lhi1 : g.lhi2;
    for (uint32_t c = 0; c < 4; ++c) {
      uint64_t o = 0;
      uint32_t l = 0;
      for (int j = 0; j < 2; ++j)
        if ((c >> j) & 1) {
          o |= uint64_t(1) << t[4 + j];
          l |= 1u << local(t[4 + j]);
        }
      hi[c] = o;
      lhi[c] = 8 * swz(l);
    }
    uint32_t* lo = k == 0 ? g.lo1 : g.lo2;
    uint32_t* llo = k == 0 ? g.llo1 : g.llo2;
    for (uint32_t i = 0; i < 16; ++i) {
      uint64_t o = 0;
      uint32_t l = 0;
      for (int j = 0; j < 4; ++j)
        if ((i >> j) & 1) {
          o |= uint64_t(1) << t[j];
          l |= 1u << local(t[j]);
        }
      lo[i] = uint32_t(o);
      llo[i] = 8 * swz(l);
    }
  }
  // Members 4m..4m+3 are neighbours in HBM when bits 0 and 1 are targets,
  // 2m and 2m + 1 when bit 0 is.
  g.vw1 = t1[0] == 0 ? (t1[1] == 1 ? 4 : 2) : 1;
  g.vw2 = t2[0] == 0 ? (t2[1] == 1 ? 4 : 2) : 1;
  g.b1_offset = uint32_t(b1_offset);
  g.b2_offset = uint32_t(b2_offset);
  return g;
}

void launch_dense_tc_pair(StateImpl& s, const DenseTcPairGeom& g, const uint8_t* tc_blob) {
  if (s.bits != 32) throw Error(QVDG_ERR_INVALID, "internal: pair pass on a complex128 state");
  if (g.vw1 == 4) return launch_pair_vw2<4>(s, g, tc_blob);
  if (g.vw1 == 2) return launch_pair_vw2<2>(s, g, tc_blob);
  return launch_pair_vw2<1>(s, g, tc_blob);
}

}  // namespace qvdg
