// Device building blocks shared by the plain tensor-core kernels
// (dense_tc.cu, dense_tc_pair.cu): the persistent CTA shape, tensor-memory
// columns, the products with A in tensor memory, the bf16 split into
// tensor memory, running deposits and bounded completion waits.
#pragma once

#include <stdint.h>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace qvdg {
namespace {

constexpr int kThreads = 512;
constexpr uint32_t kIterAmps = 8192;
// Tensor memory of the direct kernel: two product buffers of 128 fp32
// columns (D), then two operand buffers of 128 columns (A, bf16 pairs).
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kTmemA = 256;  // first A column

// The direct kernel's products, A in tensor memory: for each of the T
// blocks of 128 groups, D = A_hi B_hi + A_hi B_lo + A_lo B_hi into columns
// `dcol` + t * 2^(K+1), A_hi of block t at `acol` + t * 2^(K+1) and A_lo
// 2^K columns after it (each 16-element K slice is 8 columns), B in shared
// memory; then one commit to `bar`.
template <int K, uint32_t T = 4 / ((1u << K) / 16)>
__device__ __forceinline__ void issue_products_tmem_a(uint32_t acol, const unsigned char* bmat, uint32_t dcol,
                                                      uint32_t bar) {
  constexpr uint32_t D = 1u << K, kd = 2u * D;
  constexpr uint32_t SBO = kd * 16, BPART = kd * kd * 2;
  tc_fence_after();
  const uint32_t idesc = umma_idesc(kd);
  const uint64_t dbh = umma_desc(smem_addr(bmat), 128, SBO), dbl = umma_desc(smem_addr(bmat + BPART), 128, SBO);
#pragma unroll
  for (uint32_t t = 0; t < T; ++t) {
    const uint32_t d = dcol + t * kd;
    uint32_t acc = 0;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const uint32_t a0 = acol + t * kd + (p == 2 ? D : 0);
      const uint64_t b0 = p == 1 ? dbl : dbh;
#pragma unroll
      for (uint32_t s = 0; s < kd / 16; ++s) {
        umma_bf16_tmem_a(d, a0 + 8 * s, b0 + 16 * s, idesc, acc);
        acc = 1;
      }
    }
  }
  umma_commit(bar);
}

// Running deposit: with `cur` the deposit of an index into the positions
// outside `mask` and `step` that of an increment, the deposit of the sum
// (the carry skips the masked positions).
__device__ __forceinline__ uint64_t dep_add(uint64_t cur, uint64_t step, uint64_t mask) {
  return ((cur | mask) + step) & ~mask;
}

// Bounded wait for a completion barrier phase (about two seconds).
__device__ __forceinline__ bool wait_products(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  bool done = mbar_try_wait(bar, parity);
  while (!done && clock64() - t0 <= kWaitCycles) done = mbar_try_wait(bar, parity);
  return done;
}

// Split 8 members (x[0..7], members 16 * chunk + 8 * q + i) of one group
// into bf16 parts in this thread's tensor-memory lane: `acol` is the lane
// base plus the block's first A column; real parts go to the columns of K
// elements 16 * chunk + 8 * q.., imaginary parts 2^K elements later, low
// parts 2^K columns after the high ones.
template <int K>
__device__ __forceinline__ void write_a8_tmem(const float2* x, uint32_t acol, uint32_t chunk, int q) {
  constexpr uint32_t D = 1u << K;
  float re[8], im[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    re[i] = x[i].x;
    im[i] = x[i].y;
  }
  uint4 h, l;
  const uint32_t cre = acol + 8 * chunk + 4 * q, cim = cre + D / 2;
  split8(re, h, l);
  tmem_st4(cre, h);
  tmem_st4(cre + D, l);
  split8(im, h, l);
  tmem_st4(cim, h);
  tmem_st4(cim + D, l);
}


}  // namespace
}  // namespace qvdg
