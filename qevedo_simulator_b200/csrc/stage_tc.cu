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
#include "tc_ptx.cuh"
#include "tile_ops.cuh"

namespace qvdg {

namespace {

constexpr int kTcThreads = 256;
constexpr uint32_t kTmemCols = 64;  // 2^(L+1) fp32 columns / 128 lanes for L = 12

// Apply the tile-active one-phase gates sg[a0, a1) to n elements with tile
// indices e[] (values re[], im[]): a phase of -1 toggles a sign bit, any
// other phase is one complex multiply.
template <int N>
__device__ __forceinline__ void apply_phases(const TileGate* sg, int a0, int a1, uint64_t base,
                                             const unsigned char* blob, const uint32_t* e, float* re, float* im) {
  uint32_t sign = 0;
  for (int a = a0; a < a1; ++a) {
    const TileGate& p = sg[a];
    if ((base & p.gcm) != p.gcv) continue;
    const uint32_t m = p.lcm, v = p.lcv;
    if (p.absorb & 1) {
#pragma unroll
      for (int q = 0; q < N; ++q) sign ^= uint32_t((e[q] & m) == v) << q;
    } else {
      const float2 ph = *reinterpret_cast<const float2*>(blob + p.mat);
#pragma unroll
      for (int q = 0; q < N; ++q)
        if ((e[q] & m) == v) {
          const float r = fmaf(ph.x, re[q], -ph.y * im[q]);
          im[q] = fmaf(ph.x, im[q], ph.y * re[q]);
          re[q] = r;
        }
    }
  }
#pragma unroll
  for (int q = 0; q < N; ++q)
    if ((sign >> q) & 1) {
      re[q] = -re[q];
      im[q] = -im[q];
    }
}

// Per-thread share of one tile in flight: 2^L amplitudes / (2 per 16-byte
// access) / kTcThreads threads.
constexpr int kTileVecs = (1 << kTcTileBits) / 2 / kTcThreads;

__global__ void __launch_bounds__(kTcThreads, 2) k_stage_tc(float2* __restrict__ psi, const TileGeom geo,
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
  __shared__ TileGate sgates[kTcMaxGates];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int L = geo.L, B = geo.B;
  const uint32_t n_el = 1u << L;
  const uint32_t nvec = n_el / 2;  // 16-byte accesses per tile
  float2* tile = reinterpret_cast<float2*>(smem);
  unsigned char* a_hi = smem + (size_t(8) << L);
  unsigned char* a_lo = a_hi + (size_t(4) << L);
  unsigned char* gmem = a_lo + (size_t(4) << L);  // the pass's gate matrices (bf16 hi, lo)

  if (tid < 48) tile_bits[tid] = geo.tile_bits[tid];
  for (int i = tid; i < geo.num_gates * int(sizeof(TileGate) / 8); i += kTcThreads)
    reinterpret_cast<uint64_t*>(sgates)[i] = reinterpret_cast<const uint64_t*>(gates)[i];
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
  auto vec_addr = [&](uint64_t base, uint32_t e) -> uint64_t {
    const uint32_t r = e >> B;
    return base | hi_lo[r & 31] | hi_hi[r >> nlo] | (e & lowmask);
  };

  // Tile loads run one tile ahead: the next tile's 16-byte vectors are in
  // flight in registers while this tile is computed.
  float4 pre[kTileVecs];
  uint64_t t = blockIdx.x;
  if (t < geo.num_tiles) {
    const uint64_t base = insert_zeros(t, tile_bits, L);
#pragma unroll
    for (int i = 0; i < kTileVecs; ++i) {
      const uint32_t v = uint32_t(i) * kTcThreads + tid;
      if (v < nvec) pre[i] = ld_early(&psi[vec_addr(base, 2 * v)]);
    }
  }
  for (; t < geo.num_tiles; t += gridDim.x) {
#pragma unroll
    for (int i = 0; i < kTileVecs; ++i) {
      const uint32_t v = uint32_t(i) * kTcThreads + tid;
      if (v < nvec) {
        // elements 2v, 2v+1 land at the swizzled pair slot, swapped when the
        // swizzle flips bit 0
        const uint32_t hs = tc_swizzle(2 * v);
        const float4 x = pre[i];
        reinterpret_cast<float4*>(tile)[v ^ (hs >> 1)] = (hs & 1) ? make_float4(x.z, x.w, x.x, x.y) : x;
      }
    }
    __syncthreads();
    const uint64_t base = insert_zeros(t, tile_bits, L);
    const uint64_t next = t + gridDim.x;
    if (next < geo.num_tiles) {
      const uint64_t nbase = insert_zeros(next, tile_bits, L);
#pragma unroll
      for (int i = 0; i < kTileVecs; ++i) {
        const uint32_t v = uint32_t(i) * kTcThreads + tid;
        if (v < nvec) pre[i] = ld_early(&psi[vec_addr(nbase, 2 * v)]);
      }
    }
    for (int gi = 0; gi < geo.num_gates; ++gi) {
      // Gate scalars (uniform across the CTA); tables and data are in the
      // shared-memory blob.
      const TileGate* gp = sgates + gi;
      if (gp->kind == 3 && (gp->absorb & 2)) continue;  // applied by the next gather or the final store
      const uint64_t gcm = gp->gcm, gcv = gp->gcv;
      if ((base & gcm) != gcv) continue;  // global predicate: the same for the whole tile
      const int kind = gp->kind, k = gp->k;
      const uint32_t lcv = tc_swz_bytes(gp->lcv);  // swizzled byte units
      const uint32_t count = 1u << (L - gp->nfixed);
      const unsigned char* data = gmem + gp->mat;
      const uint32_t* ebl = reinterpret_cast<const uint32_t*>(gmem + gp->tab);  // byte offsets
      const uint32_t* ebh = ebl + 64;
      const uint32_t* aux = ebl + 192;  // member byte offsets, or diagonal index parts
      unsigned char* tb = reinterpret_cast<unsigned char*>(tile);
      if (kind == 3) {
        const float2 ph = *reinterpret_cast<const float2*>(data);
        for (uint32_t i = tid; i < count; i += kTcThreads) {
          float2* p = reinterpret_cast<float2*>(tb + (ebl[i & 63] ^ ebh[i >> 6] ^ lcv));
          const float2 x = *p;
          *p = make_float2(fmaf(ph.x, x.x, -ph.y * x.y), fmaf(ph.x, x.y, ph.y * x.x));
        }
      } else if (kind == 1) {
        uint32_t dglob = 0;
        for (int j = 0; j < k; ++j) {
          const uint32_t tj = gp->tgt[j];
          if (tj & 0x80) dglob |= uint32_t((base >> (tj & 0x7f)) & 1) << j;
        }
        const float2* d = reinterpret_cast<const float2*>(data);
        for (uint32_t i = tid; i < count; i += kTcThreads) {
          const uint32_t eb = ebl[i & 63] ^ ebh[i >> 6] ^ lcv;
          const uint32_t e = tc_swz(eb >> 3);  // logical index for the diagonal
          const float2 f = d[aux[e & 127] | aux[128 + (e >> 7)] | dglob];
          float2* p = reinterpret_cast<float2*>(tb + eb);
          const float2 x = *p;
          *p = make_float2(fmaf(f.x, x.x, -f.y * x.y), fmaf(f.x, x.y, f.y * x.x));
        }
      } else if (kind == 0) {
        const float2* m = reinterpret_cast<const float2*>(data);
        if (k == 1) {
          const float2 m00 = m[0], m01 = m[1], m10 = m[2], m11 = m[3];
          const uint32_t o1 = aux[1];
          for (uint32_t i = tid; i < count; i += kTcThreads) {
            const uint32_t b = ebl[i & 63] ^ ebh[i >> 6] ^ lcv;
            float2* p0 = reinterpret_cast<float2*>(tb + b);
            float2* p1 = reinterpret_cast<float2*>(tb + (b ^ o1));
            const float2 x0 = *p0, x1 = *p1;
            float2 y0 = make_float2(0.f, 0.f), y1 = make_float2(0.f, 0.f);
            cmac<float>(y0, m00, x0);
            cmac<float>(y0, m01, x1);
            cmac<float>(y1, m10, x0);
            cmac<float>(y1, m11, x1);
            *p0 = y0;
            *p1 = y1;
          }
        } else {
          // k = 2 (wider gates go to the tensor cores)
          for (uint32_t i = tid; i < count; i += kTcThreads) {
            const uint32_t b = ebl[i & 63] ^ ebh[i >> 6] ^ lcv;
            float2 x[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) x[h] = *reinterpret_cast<const float2*>(tb + (b ^ aux[h]));
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              float2 y = make_float2(0.f, 0.f);
#pragma unroll
              for (int c = 0; c < 4; ++c) cmac<float>(y, m[r * 4 + c], x[c]);
              *reinterpret_cast<float2*>(tb + (b ^ aux[r])) = y;
            }
          }
        }
      } else {
        // ---- dense gate on the tensor cores
        const uint32_t half = 1u << k, kd = 2u << k;
        const uint32_t sbo = kd * 16;                 // bytes between 8-row core groups
        const uint32_t block_bytes = 128u * kd * 2u;  // one 128-group block of A (bf16)
        const uint32_t groups = count, nblocks = groups >> 7;
        // Gather: unit = (group, 8 consecutive members); consecutive
        // threads take consecutive groups.
        const uint32_t units = groups * (half / 8);
        const int absorb = gp->absorb;
#pragma unroll 2
        for (uint32_t u = tid; u < units; u += kTcThreads) {
          const uint32_t grp = u & (groups - 1), c0 = (u >> (L - k)) * 8;
          const uint32_t eb = ebl[grp & 63] ^ ebh[grp >> 6];
          const uint4 o0 = *reinterpret_cast<const uint4*>(aux + c0);
          const uint4 o1 = *reinterpret_cast<const uint4*>(aux + c0 + 4);
          uint32_t e[8] = {eb ^ o0.x, eb ^ o0.y, eb ^ o0.z, eb ^ o0.w, eb ^ o1.x, eb ^ o1.y, eb ^ o1.z, eb ^ o1.w};
          float re[8], im[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float2 v = *reinterpret_cast<const float2*>(tb + e[q]);
            re[q] = v.x;
            im[q] = v.y;
          }
          if (absorb) {
            uint32_t le[8];  // logical byte offsets for the phase tests
#pragma unroll
            for (int q = 0; q < 8; ++q) le[q] = tc_swz_bytes(e[q]);
            apply_phases<8>(sgates, gi - absorb, gi, base, gmem, le, re, im);
          }
          const uint32_t r = grp & 127;
          const uint32_t row = (grp >> 7) * block_bytes + (r >> 3) * sbo + (r & 7) * 16;
          uint4 h, l;
          split8(re, h, l);
          *reinterpret_cast<uint4*>(a_hi + row + (c0 / 8) * 128) = h;
          *reinterpret_cast<uint4*>(a_lo + row + (c0 / 8) * 128) = l;
          split8(im, h, l);
          *reinterpret_cast<uint4*>(a_hi + row + ((half + c0) / 8) * 128) = h;
          *reinterpret_cast<uint4*>(a_lo + row + ((half + c0) / 8) * 128) = l;
        }
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
          tc_fence_after();
          const uint32_t idesc = umma_idesc(kd);
          const uint32_t g_hi = smem_addr(data), g_lo = g_hi + kd * kd * 2;
          // Descriptors differ only in the start-address field (16-byte units).
          const uint64_t dah = umma_desc(smem_addr(a_hi), 128, sbo), dal = umma_desc(smem_addr(a_lo), 128, sbo);
          const uint64_t dbh = umma_desc(g_hi, 128, sbo), dbl = umma_desc(g_lo, 128, sbo);
          const uint32_t ksteps = kd / 16;
          for (uint32_t b = 0; b < nblocks; ++b) {
            const uint32_t d = tmem + b * kd;
            const uint64_t boff = (b * block_bytes) >> 4;
            uint32_t acc = 0;
#pragma unroll
            for (int p = 0; p < 3; ++p) {
              const uint64_t a0 = (p == 2 ? dal : dah) + boff, b0 = p == 1 ? dbl : dbh;
              for (uint32_t s = 0; s < ksteps; ++s) {
                umma_bf16(d, a0 + 16 * s, b0 + 16 * s, idesc, acc);
                acc = 1;
              }
            }
          }
          umma_commit(barp);
          // Bounded wait for the products by this thread alone (suspended in
          // hardware); the other warps wait at the barrier below.
          const long long t0 = clock64();
          while (!mbar_try_wait(barp, phase)) {
            if (clock64() - t0 > kWaitCycles) {
              atomicExch(status, 1);
              abort_run = 1;
              break;
            }
          }
        }
        phase ^= 1u;
        __syncthreads();
        if (abort_run) break;
        tc_fence_after();
        // Read-back: warp w reads TMEM lanes 32*(w%4).. of the columns of
        // work unit w/4 + 2 j, a unit being 16 real and 16 imaginary
        // columns of one block (or the 16 columns of one block for k = 3).
        const uint32_t quarter = uint32_t(warp & 3), wg = uint32_t(warp >> 2);
        const uint32_t chunks = half >= 16 ? half / 16 : 1;
        const uint32_t nunits = nblocks * chunks;
        for (uint32_t unit = wg; unit < nunits; unit += kTcThreads / 128) {
          const uint32_t b = unit / chunks, c0 = (unit % chunks) * 16;
          const uint32_t grp = b * 128u + quarter * 32u + uint32_t(tid & 31);
          const uint32_t eb = ebl[grp & 63] ^ ebh[grp >> 6];
          const uint32_t lane_base = tmem + ((quarter * 32u) << 16) + b * kd;
          if (half == 8) {
            float v[16];
            tmem_ld16(lane_base, v);
            const uint4 o0 = *reinterpret_cast<const uint4*>(aux);
            const uint4 o1 = *reinterpret_cast<const uint4*>(aux + 4);
            const uint32_t o[8] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y, o1.z, o1.w};
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 8; ++q) *reinterpret_cast<float2*>(tb + (eb ^ o[q])) = make_float2(v[q], v[8 + q]);
          } else {
            float re[16], im[16];
            tmem_ld16(lane_base + c0, re);
            tmem_ld16(lane_base + half + c0, im);
            uint32_t o[16];
#pragma unroll
            for (int q = 0; q < 16; q += 4) {
              const uint4 oo = *reinterpret_cast<const uint4*>(aux + c0 + q);
              o[q] = oo.x;
              o[q + 1] = oo.y;
              o[q + 2] = oo.z;
              o[q + 3] = oo.w;
            }
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; ++q) *reinterpret_cast<float2*>(tb + (eb ^ o[q])) = make_float2(re[q], im[q]);
          }
        }
        tc_fence_before();
      }
      __syncthreads();
    }
    if (abort_run) break;
    // Store this tile (the next tile's loads are already in flight),
    // applying the trailing one-phase gates.
    const int tail0 = geo.num_gates - geo.tail_absorb;
#pragma unroll
    for (int i = 0; i < kTileVecs; ++i) {
      const uint32_t v = uint32_t(i) * kTcThreads + tid;
      if (v < nvec) {
        const uint32_t hs = tc_swizzle(2 * v);
        float4 x = reinterpret_cast<const float4*>(tile)[v ^ (hs >> 1)];
        if (hs & 1) x = make_float4(x.z, x.w, x.x, x.y);
        if (geo.tail_absorb) {
          const uint32_t e[2] = {16 * v, 16 * v + 8};  // byte offsets
          float re[2] = {x.x, x.z}, im[2] = {x.y, x.w};
          apply_phases<2>(sgates, tail0, geo.num_gates, base, gmem, e, re, im);
          x = make_float4(re[0], im[0], re[1], im[1]);
        }
        *reinterpret_cast<float4*>(&psi[vec_addr(base, 2 * v)]) = x;
      }
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

// Registers limit the kernel to two CTAs per SM (256 threads x 128
// registers each); two 64-column TMEM allocations always fit.
static size_t tc_launch_smem(const TileGeom& geo) { return tc_smem_bytes(geo); }

void launch_stage_tc(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  const size_t smem = tc_launch_smem(lp.geo);
  static size_t configured = 0;
  if (smem > configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_stage_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    configured = smem;
  }
  const uint64_t grid = std::min<uint64_t>(lp.geo.num_tiles, uint64_t(s.sms) * 2);
  k_stage_tc<<<unsigned(grid), kTcThreads, smem, s.stream>>>(static_cast<float2*>(s.amp), lp.geo,
                                                            dev.gates + lp.gate_offset,
                                                            static_cast<const float2*>(dev.mats), dev.tc, s.status);
  QVDG_LAUNCH_CHECK();
}

}  // namespace qvdg
