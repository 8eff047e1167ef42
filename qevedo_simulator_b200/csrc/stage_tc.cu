// Staged tile kernel with fused dense gates on the 5th-generation tensor
// cores (tcgen05), complex64 state.
//
// One CTA per SM, 128 threads, persistent over tiles. A tile T of 2^L
// amplitudes lives in shared memory as complex64. For a dense gate on k
// tile-local qubits (3 <= k <= L - 7) the tile is a batch of 2^(L-k) groups,
// and the gate is one real matrix product per block of 128 groups:
//
//     D[g][n] = sum_kk A[g][kk] * B[kk][n],   kk, n in [0, 2^(k+1))
//
// where row g of A holds group g's amplitudes (2^k real parts, then 2^k
// imaginary parts) and B is the gate as the real 2^(k+1) x 2^(k+1) matrix
// [[Re M, Im M], [-Im M, Re M]]^T. A and B are stored in shared memory as
// bf16 high and low parts (x = hi + lo to 16 significant bits), and D, in
// tensor memory (fp32), accumulates the compensated sum
// A_hi B_hi + A_hi B_lo + A_lo B_hi (issued by one thread, M = 128,
// N = K = 2^(k+1), K-major operands in the canonical no-swizzle core-matrix
// layout: 8 rows x 16 bytes per core matrix, K-adjacent cores 128 bytes
// apart, row-group-adjacent cores 16 * 2^(k+1) bytes apart). Each thread
// then reads its own row of D (its group) back with tcgen05.ld and writes
// the group into T. Diagonal gates and one- and two-qubit gates stay on the
// CUDA cores (tile_ops.cuh). Every wait on the MMA completion barrier is
// bounded: on timeout the kernel records an error, frees its tensor memory
// and returns.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "program.hpp"
#include "stage.hpp"
#include "stage_kernel.hpp"
#include "tile_ops.cuh"

namespace qvdg {

namespace {

constexpr int kTcThreads = 128;
constexpr uint32_t kTmemCols = 128;  // 2^(L+1) fp32 columns / 128 lanes for L = 13

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle, K-major canonical layout).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;  // descriptor version for this architecture
  return d;
}

// Instruction descriptor: D fp32, A and B bf16, both K-major, M = 128.
__device__ __forceinline__ uint32_t umma_idesc(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(phase)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Pack 8 floats' bf16 high parts and low parts into two 16-byte vectors.
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * i]);
    const __nv_bfloat16 h1 = __float2bfloat16_rn(x[2 * i + 1]);
    const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * i] - __bfloat162float(h0));
    const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * i + 1] - __bfloat162float(h1));
    h[i] = uint32_t(__bfloat16_as_ushort(h0)) | (uint32_t(__bfloat16_as_ushort(h1)) << 16);
    l[i] = uint32_t(__bfloat16_as_ushort(l0)) | (uint32_t(__bfloat16_as_ushort(l1)) << 16);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Bounded wait: about two seconds of SM clocks.
constexpr long long kWaitCycles = 4000000000LL;

__global__ void __launch_bounds__(kTcThreads, 1) k_stage_tc(float2* __restrict__ psi, const TileGeom geo,
                                                            const TileGate* __restrict__ gates,
                                                            const float2* __restrict__ mats,
                                                            const uint8_t* __restrict__ tc_blob,
                                                            int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint8_t tile_bits[48];
  __shared__ uint64_t hi_lo[32], hi_hi[32];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_run;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int L = geo.L, B = geo.B;
  const uint32_t n_el = 1u << L;
  float2* tile = reinterpret_cast<float2*>(smem);
  unsigned char* a_hi = smem + (size_t(8) << L);
  unsigned char* a_lo = a_hi + (size_t(4) << L);
  unsigned char* gmem = a_lo + (size_t(4) << L);  // the pass's gate matrices (bf16 hi, lo)

  if (tid < 48) tile_bits[tid] = geo.tile_bits[tid];
  if (tid == 0) {
    abort_run = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // The gate matrices of this pass stay resident for every tile.
  {
    const uint4* src = reinterpret_cast<const uint4*>(tc_blob + geo.tc_offset);
    uint4* dst = reinterpret_cast<uint4*>(gmem);
    for (uint32_t i = tid; i < geo.tc_bytes / 16; i += kTcThreads) dst[i] = src[i];
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  // Address tables: tile element e -> physical bits, split in two lookups
  // of the (L - B) non-contiguous bits.
  const int nfree = L - B, nlo = nfree < 5 ? nfree : 5;
  if (tid < 32) {
    uint64_t a = 0, b = 0;
    for (int j = 0; j < nlo; ++j)
      if ((tid >> j) & 1) a |= uint64_t(1) << tile_bits[B + j];
    for (int j = nlo; j < nfree; ++j)
      if ((tid >> (j - nlo)) & 1) b |= uint64_t(1) << tile_bits[B + j];
    hi_lo[tid] = a;
    hi_hi[tid] = b;
  }
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t barp = smem_addr(&bar);
  const uint32_t lowmask = (1u << B) - 1u;
  uint32_t phase = 0;

  for (uint64_t t = blockIdx.x; t < geo.num_tiles && !abort_run; t += gridDim.x) {
    const uint64_t base = insert_zeros(t, tile_bits, L);
    for (uint32_t e = tid * 2; e < n_el; e += kTcThreads * 2) {
      const uint32_t r = e >> B;
      const uint64_t a = base | hi_lo[r & 31] | hi_hi[r >> nlo] | (e & lowmask);
      *reinterpret_cast<float4*>(&tile[e]) = *reinterpret_cast<const float4*>(&psi[a]);
    }
    __syncthreads();
    for (int gi = 0; gi < geo.num_gates; ++gi) {
      const TileGate& g = gates[gi];
      if ((base & g.gcm) != g.gcv) continue;  // global controls: the same for the whole tile
      if (g.kind == 1) {
        tile_diag<float>(tile, L, g, mats + g.mat, base);
      } else if (g.kind == 0) {
        switch (g.k) {
          case 1: tile_dense<float, 1>(tile, L, g, mats + g.mat); break;
          case 2: tile_dense<float, 2>(tile, L, g, mats + g.mat); break;
          case 3: tile_dense<float, 3>(tile, L, g, mats + g.mat); break;
          case 4: tile_dense<float, 4>(tile, L, g, mats + g.mat); break;
          case 5: tile_dense_rows<float, 5>(tile, L, g, mats + g.mat); break;
          default: tile_dense_rows<float, 6>(tile, L, g, mats + g.mat); break;
        }
      } else {
        // ---- dense gate on the tensor cores
        const int k = g.k;
        const uint32_t half = 1u << k, kd = 2u << k;
        const uint32_t sbo = kd * 16;                    // bytes between 8-row core groups
        const uint32_t block_bytes = 128u * kd * 2u;     // one 128-group block of A (bf16)
        const uint32_t nblocks = 1u << (L - k - 7);
        uint8_t tg[8];
        for (int j = 0; j < k; ++j) tg[j] = g.tgt[j];
        // Gather: this thread's row in every block.
        for (uint32_t b = 0; b < nblocks; ++b) {
          const uint32_t eb = insert_zeros32(b * 128u + tid, g.fixed, k);
          const uint32_t row = b * block_bytes + (tid >> 3) * sbo + (tid & 7) * 16;
          for (uint32_t c0 = 0; c0 < half; c0 += 8) {
            float re[8], im[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              uint32_t off = 0;
              const uint32_t c = c0 + q;
              for (int j = 0; j < k; ++j) off |= ((c >> j) & 1u) << tg[j];
              const float2 v = tile[eb | off];
              re[q] = v.x;
              im[q] = v.y;
            }
            uint4 h, l;
            split8(re, h, l);
            *reinterpret_cast<uint4*>(a_hi + row + (c0 / 8) * 128) = h;
            *reinterpret_cast<uint4*>(a_lo + row + (c0 / 8) * 128) = l;
            split8(im, h, l);
            *reinterpret_cast<uint4*>(a_hi + row + ((half + c0) / 8) * 128) = h;
            *reinterpret_cast<uint4*>(a_lo + row + ((half + c0) / 8) * 128) = l;
          }
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
          tc_fence_after();
          const uint32_t idesc = umma_idesc(kd);
          const uint32_t g_hi = smem_addr(gmem + g.mat), g_lo = g_hi + kd * kd * 2;
          const uint32_t ah = smem_addr(a_hi), al = smem_addr(a_lo);
          for (uint32_t b = 0; b < nblocks; ++b) {
            const uint32_t d = tmem + b * kd;
            uint32_t acc = 0;
            for (int p = 0; p < 3; ++p) {
              const uint32_t abase = (p == 2 ? al : ah) + b * block_bytes;
              const uint32_t bbase = p == 1 ? g_lo : g_hi;
              for (uint32_t s = 0; s < kd / 16; ++s) {
                umma_bf16(d, umma_desc(abase + s * 256, 128, sbo), umma_desc(bbase + s * 256, 128, sbo), idesc, acc);
                acc = 1;
              }
            }
          }
          umma_commit(barp);
        }
        // Bounded wait for the products.
        const long long t0 = clock64();
        bool ok = true;
        while (!mbar_try_wait(barp, phase)) {
          if (clock64() - t0 > kWaitCycles) {
            ok = false;
            break;
          }
        }
        phase ^= 1u;
        if (!ok) {
          atomicExch(status, 1);
          abort_run = 1;
        }
        __syncthreads();
        if (abort_run) break;
        tc_fence_after();
        // Scatter: row tid of each block back to its group in T.
        for (uint32_t b = 0; b < nblocks; ++b) {
          const uint32_t eb = insert_zeros32(b * 128u + tid, g.fixed, k);
          const uint32_t lane_base = tmem + (uint32_t(warp * 32) << 16) + b * kd;
          if (half == 8) {
            // 16 columns: 8 real parts then 8 imaginary parts.
            float v[16];
            tmem_ld16(lane_base, v);
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              uint32_t off = 0;
              for (int j = 0; j < k; ++j) off |= ((uint32_t(q) >> j) & 1u) << tg[j];
              tile[eb | off] = make_float2(v[q], v[8 + q]);
            }
            continue;
          }
          for (uint32_t c0 = 0; c0 < half; c0 += 16) {
            float re[16], im[16];
            tmem_ld16(lane_base + c0, re);
            tmem_ld16(lane_base + half + c0, im);
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              uint32_t off = 0;
              const uint32_t c = c0 + q;
              for (int j = 0; j < k; ++j) off |= ((c >> j) & 1u) << tg[j];
              tile[eb | off] = make_float2(re[q], im[q]);
            }
          }
        }
        tc_fence_before();
      }
      __syncthreads();
    }
    if (abort_run) break;
    for (uint32_t e = tid * 2; e < n_el; e += kTcThreads * 2) {
      const uint32_t r = e >> B;
      const uint64_t a = base | hi_lo[r & 31] | hi_hi[r >> nlo] | (e & lowmask);
      *reinterpret_cast<float4*>(&psi[a]) = *reinterpret_cast<const float4*>(&tile[e]);
    }
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

}  // namespace

size_t tc_smem_bytes(const TileGeom& geo) { return (size_t(16) << geo.L) + geo.tc_bytes; }

// At least 116 KiB of dynamic shared memory: with more than half of the
// SM's shared memory per CTA, one CTA (and one 128-column TMEM allocation)
// is resident per SM.
static size_t tc_launch_smem(const TileGeom& geo) { return std::max(tc_smem_bytes(geo), size_t(116 * 1024)); }

void launch_stage_tc(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  const size_t smem = tc_launch_smem(lp.geo);
  static size_t configured = 0;
  if (smem > configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_stage_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    configured = smem;
  }
  const uint64_t grid = std::min<uint64_t>(lp.geo.num_tiles, uint64_t(s.sms));
  k_stage_tc<<<unsigned(grid), kTcThreads, smem, s.stream>>>(static_cast<float2*>(s.amp), lp.geo,
                                                            dev.gates + lp.gate_offset,
                                                            static_cast<const float2*>(dev.mats), dev.tc, s.status);
  QVDG_LAUNCH_CHECK();
}

}  // namespace qvdg
