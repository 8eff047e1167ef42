// Two fused 6-qubit gates in one plain pass over a complex64 state, on the
// tensor cores: the reference applies each fused op as its own sweep over
// the state (src/simulator.rs:136-143, src/kernels.rs:252-473); here two
// consecutive fused gates share one HBM pass, so a plan of plain fused
// passes moves the state about half as often.
//
// An iteration covers the 8192 amplitudes spanned by 13 bits I: the
// targets of both gates and the lowest other bits. Gate 1 sees them as 128
// groups of 64 members (groups over I minus its targets), gate 2 as another
// 128 groups. Persistent CTAs of 512 threads; thread (w, r) owns 16 members
// of group r for either gate (w / 4 picks which 16), as in the single-gate
// kernel (dense_tc.cu), and tensor-memory lane r holds group r:
//
//   1. gate 1's members come from HBM (loaded two iterations ahead into
//      registers), are split into bf16 high and low parts and written to
//      the A buffer in tensor memory; one thread issues the products
//      A_hi B1_hi + A_hi B1_lo + A_lo B1_hi (fp32 accumulation);
//   2. the products are read back (tcgen05.ld) and written into a 64 KB
//      shared-memory buffer at the amplitudes' positions in I; after a CTA
//      barrier every thread reads its 16 members of gate 2's group r from
//      it, splits them into the same A buffer, and the products with B2
//      are issued;
//   3. one iteration later gate 2's products are read back and stored to
//      HBM where gate 2's members lie.
//
// Two sets of tensor-memory buffers (A and D, 256 columns each) alternate
// between iterations, so iteration i's first products run while iteration
// i - 1 is stored. Positions in the transpose buffer are XOR-swizzled (low
// four index bits with a host-chosen linear map of the high ones) so that
// both gates' group-parallel accesses hit distinct banks. Every wait on a
// product barrier is bounded: on timeout the kernel records an error, all
// threads leave at the next CTA barrier and the tensor memory is freed.

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

template <int VW1, int VW2>
__global__ void __launch_bounds__(kThreads, 1) k_dense_tc_pair(float2* __restrict__ psi, const DenseTcPairGeom g,
                                                               const uint8_t* __restrict__ bmats,
                                                               int* __restrict__ status) {
  constexpr uint32_t D = 64;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar1[2], bar2[2];
  __shared__ uint32_t tmem_slot;
  __shared__ uint8_t ibits[16];
  unsigned char* bmat1 = smem;                            // gate 1: B hi, then B lo
  unsigned char* bmat2 = smem + kPairBytes;               // gate 2
  float2* xbuf = reinterpret_cast<float2*>(smem + 2 * kPairBytes);  // 8192 complex64
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t r = uint32_t(tid) & 127u, chunk = uint32_t(tid) >> 7;

  if (tid < 16) ibits[tid] = g.ibits[tid];
  {
    const uint4* s1 = reinterpret_cast<const uint4*>(bmats + g.b1_offset);
    const uint4* s2 = reinterpret_cast<const uint4*>(bmats + g.b2_offset);
    uint4* d1 = reinterpret_cast<uint4*>(bmat1);
    uint4* d2 = reinterpret_cast<uint4*>(bmat2);
    for (uint32_t i = tid; i < kPairBytes / 16; i += kThreads) {
      d1[i] = s1[i];
      d2[i] = s2[i];
    }
  }
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar1[b])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar2[b])));
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

  // This thread's group r and member chunk, for either gate: HBM offset of
  // its group and chunk, and its position (swizzled) in the transpose
  // buffer; member i adds lo*[i] / XORs llo*[i].
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
  uint32_t lo1[16], lo2[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    lo1[i] = g.lo1[i];
    lo2[i] = g.lo2[i];
  }
  const uint64_t my_iters = blockIdx.x < g.iters ? (g.iters - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // Iteration bases (the bits outside I), advanced by a running deposit.
  const uint64_t dstep = insert_zeros(gridDim.x, ibits, 13);
  uint64_t dload = insert_zeros(blockIdx.x, ibits, 13), dstore = dload;
  const uint32_t lanes = (uint32_t(warp & 3) * 32u) << 16;
  int failed = 0;

  auto load = [&](float2 (&x)[16]) {
    load16<VW1>(psi, dload + gb1, lo1, x);
    dload = dep_add(dload, dstep, g.imask);
  };
  // Step li: gate 1 of iteration li from registers into A and its products
  // issued; iteration li - 1 (gate 2's products, issued in the last step)
  // stored; iteration li's products transposed into gate 2's groups and
  // its second products issued. Returns whether another step follows.
  auto step = [&](uint64_t li, float2 (&x)[16]) -> bool {
    const bool have = li < my_iters;
    const uint32_t b = uint32_t(li & 1);
    const uint32_t acol = kTmemA + b * 128, dcol = b * 128;
    const uint32_t parity = uint32_t((li >> 1) & 1);
    if (have) {
      write_a8_tmem<6>(x, tmem + lanes + acol, chunk, 0);
      write_a8_tmem<6>(x + 8, tmem + lanes + acol, chunk, 1);
      if (li + 2 < my_iters) load(x);
      tmem_wait_st();
    }
    tc_fence_before();
    if (__syncthreads_or(failed)) return false;
    if (have && tid == 0) issue_products_tmem_a<6>(tmem + acol, bmat1, tmem + dcol, smem_addr(&bar1[b]));
    if (li > 0) {
      // Store iteration li - 1: gate 2's products in the other buffers.
      const uint32_t pb = b ^ 1u;
      const uint32_t pparity = uint32_t(((li - 1) >> 1) & 1);
      const uint64_t base = dstore + gb2;
      dstore = dep_add(dstore, dstep, g.imask);
      // Warp-uniform outcome: tcgen05.ld below is a warp-wide instruction.
      if (!__all_sync(0xffffffffu, wait_products(smem_addr(&bar2[pb]), pparity))) {
        failed = 1;
        atomicExch(status, 1);
      } else {
        tc_fence_after();
        const uint32_t taddr = tmem + lanes + pb * 128 + 16 * chunk;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          float re[8], im[8];
          tmem_ld8(taddr + 8 * hh, re);
          tmem_ld8(taddr + D + 8 * hh, im);
          tmem_wait_ld();
          store8<VW2>(psi, base, lo2, hh, re, im);
        }
      }
    }
    if (have && !failed) {
      // Gate 1's products of iteration li into the transpose buffer.
      if (!__all_sync(0xffffffffu, wait_products(smem_addr(&bar1[b]), parity))) {
        failed = 1;
        atomicExch(status, 1);
      } else {
        tc_fence_after();
        const uint32_t taddr = tmem + lanes + dcol + 16 * chunk;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          float re[8], im[8];
          tmem_ld8(taddr + 8 * hh, re);
          tmem_ld8(taddr + D + 8 * hh, im);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 8; ++i) xbuf[lb1 ^ g.llo1[8 * hh + i]] = make_float2(re[i], im[i]);
        }
      }
    }
    tc_fence_before();
    if (__syncthreads_or(failed)) return false;
    if (have) {
      // Gate 2's groups from the transpose buffer into A.
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        float2 m[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) m[i] = xbuf[lb2 ^ g.llo2[8 * q + i]];
        write_a8_tmem<6>(m, tmem + lanes + acol, chunk, q);
      }
      tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    if (have && tid == 0) issue_products_tmem_a<6>(tmem + acol, bmat2, tmem + dcol, smem_addr(&bar2[b]));
    return have;
  };
  // Two register sets in flight, so each iteration's loads are issued two
  // iterations ahead of their use; the step after the last iteration only
  // stores it.
  float2 xa[16], xb[16];
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
    configured = true;
  }
  const unsigned grid = unsigned(std::min<uint64_t>(g.iters, uint64_t(s.sms)));
  k_dense_tc_pair<VW1, VW2><<<grid, kThreads, smem, s.stream>>>(static_cast<float2*>(s.amp), g, bmats, s.status);
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
// runs of at least 16 amplitudes (128 bytes), or of at least 4 within 1024
// amplitudes. Elsewhere a warp touches many scattered sectors and the pass
// runs several times slower than two single passes (measured at 30 qubits).
bool pair_gate_coalesced(const std::vector<uint32_t>& t, const std::vector<uint32_t>& ibits) {
  const uint32_t vw = t[0] == 0 ? (t[1] == 1 ? 4u : 2u) : 1u;
  std::vector<uint32_t> lanes;
  for (uint32_t q : ibits)
    if (lanes.size() < 5 && std::find(t.begin(), t.end(), q) == t.end()) lanes.push_back(q);
  uint32_t run = vw, next = vw == 4 ? 2u : (vw == 2 ? 1u : 0u);
  for (uint32_t q : lanes) {
    if (q != next) break;
    run *= 2;
    ++next;
  }
  return run >= 16 || (run >= 4 && lanes.back() <= 9);
}

}  // namespace

bool dense_tc_pair_ok(uint32_t n, int bits, const std::vector<uint32_t>& t1, const std::vector<uint32_t>& t2) {
  if (bits != 32 || n < 14 || t1.size() != 6 || t2.size() != 6) return false;
  if (!dense_tc_ok(n, bits, t1, 0) || !dense_tc_ok(n, bits, t2, 0)) return false;
  std::vector<uint32_t> a(t1), b(t2);
  std::sort(a.begin(), a.end());
  std::sort(b.begin(), b.end());
  const std::vector<uint32_t> ibits = pair_bits(a, b);
  return pair_gate_coalesced(a, ibits) && pair_gate_coalesced(b, ibits);
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
    uint16_t* lgrp = k == 0 ? g.lgrp1 : g.lgrp2;
    for (int j = 0; j < 7; ++j) {
      grp_off[j] = uint64_t(1) << grp[k][j];
      lgrp[j] = uint16_t(swz(1u << local(grp[k][j])));
    }
    uint64_t* hi = k == 0 ? g.hi1 : g.hi2;
    uint16_t* lhi = k == 0 ? g.lhi1 : g.lhi2;
    for (uint32_t c = 0; c < 4; ++c) {
      uint64_t o = 0;
      uint32_t l = 0;
      for (int j = 0; j < 2; ++j)
        if ((c >> j) & 1) {
          o |= uint64_t(1) << t[4 + j];
          l |= 1u << local(t[4 + j]);
        }
      hi[c] = o;
      lhi[c] = uint16_t(swz(l));
    }
    uint32_t* lo = k == 0 ? g.lo1 : g.lo2;
    uint16_t* llo = k == 0 ? g.llo1 : g.llo2;
    for (uint32_t i = 0; i < 16; ++i) {
      uint64_t o = 0;
      uint32_t l = 0;
      for (int j = 0; j < 4; ++j)
        if ((i >> j) & 1) {
          o |= uint64_t(1) << t[j];
          l |= 1u << local(t[j]);
        }
      lo[i] = uint32_t(o);
      llo[i] = uint16_t(swz(l));
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
