// Measurement on the device: FP64 reductions and the two-pass sampler.
//
// Reductions (norm, per-bit probabilities) accumulate in double precision in
// a fixed order per launch shape, so repeated calls give identical results.
//
// The sampler restates StateVector::sample_unordered (src/measure.rs:104-174)
// so that, for the same amplitudes and the same uniforms, every outcome is
// bit-identical to the reference's:
//   - the state is cut into chunks of CHUNK_BLOCKS * LANES amplitudes
//     (4096 * 8 = 32768 for complex64, 4096 * 4 = 16384 for complex128,
//     src/measure.rs:13 and src/simd.rs:71-97), in physical index order;
//   - p = re*re + im*im in f64 without contraction (__dmul_rn/__dadd_rn);
//   - each chunk sum is one sequential left fold in index order (one lane
//     owns a chunk; a warp streams 32 chunks' data through shared memory);
//   - the chunk prefix is sequential; targets = u * total are sorted in f64
//     total order; bounds are partition points of the prefix;
//   - the walk adds nonzero p in index order from prefix[chunk] and emits an
//     index while target < cumulative, pads with the last nonzero index.

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "engine.hpp"
#include "qvdg.h"

namespace qvdg {

namespace {

constexpr int kThreads = 256;

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

template <typename T>
__device__ __forceinline__ double prob(const cplx_t<T>& a) {
  const double re = double(a.x), im = double(a.y);
  return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum (result valid in thread 0).
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_sumsq(const cplx_t<T>* __restrict__ psi, uint64_t len,
                                                    double* __restrict__ partials) {
  __shared__ double red[32];
  double acc = 0.0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    const cplx_t<T> a = psi[i];
    acc += double(a.x) * double(a.x) + double(a.y) * double(a.y);
  }
  const double t = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// Sums `count` vectors of `width` doubles (vector i at partials + i*width)
// into out[0..width), each component in index order.
__global__ void k_sum_columns(const double* __restrict__ partials, int count, int width, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= width) return;
  double t = 0.0;
  for (int i = 0; i < count; ++i) t += partials[size_t(i) * width + j];
  out[j] = t;
}

// Per-bit probabilities. A segment is 1024 consecutive amplitudes: bits 0-1
// inside a thread (4 elements), bits 2-9 from the thread index. Each block
// takes `per_block` consecutive segments (a power of two), so the low
// log2(per_block) segment bits vary inside the block and the others are fixed
// by the block index. Each block writes P(bit = 1) for every bit, then the
// total, to partials[block * (n + 1) + ...].
constexpr int kMaxVarBits = 16;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_bit_probs(const cplx_t<T>* __restrict__ psi, int n,
                                                        uint64_t per_block, int var_bits,
                                                        double* __restrict__ partials) {
  __shared__ double red[32];
  const uint64_t len = uint64_t(1) << n;
  double tot = 0.0, lo0 = 0.0, lo1 = 0.0;
  double hv[kMaxVarBits];
#pragma unroll
  for (int b = 0; b < kMaxVarBits; ++b) hv[b] = 0.0;
  for (uint64_t i = 0; i < per_block; ++i) {
    const uint64_t first = ((uint64_t(blockIdx.x) * per_block + i) << 10) + uint64_t(threadIdx.x) * 4;
    double st = 0.0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (first + e < len) {
        const double p = prob<T>(psi[first + e]);
        st += p;
        if (e & 1) lo0 += p;
        if (e & 2) lo1 += p;
      }
    }
    tot += st;
#pragma unroll
    for (int b = 0; b < kMaxVarBits; ++b)
      if ((i >> b) & 1) hv[b] += st;
  }
  double* out = partials + size_t(blockIdx.x) * (n + 1);
  for (int bit = 0; bit < n; ++bit) {
    double v = 0.0;
    if (bit == 0) {
      v = lo0;
    } else if (bit == 1) {
      v = lo1;
    } else if (bit < 10) {
      v = ((threadIdx.x >> (bit - 2)) & 1) ? tot : 0.0;
    } else if (bit < 10 + var_bits) {
#pragma unroll
      for (int b = 0; b < kMaxVarBits; ++b)
        if (b == bit - 10) v = hv[b];
    } else {
      v = ((uint64_t(blockIdx.x) >> (bit - 10 - var_bits)) & 1) ? tot : 0.0;
    }
    const double s = block_sum(v, red);
    if (threadIdx.x == 0) out[bit] = s;
  }
  const double s = block_sum(tot, red);
  if (threadIdx.x == 0) out[n] = s;
}

template <typename T>
__global__ void k_probs(const cplx_t<T>* __restrict__ psi, double* __restrict__ out, uint64_t first, uint64_t count,
                        const uint64_t* __restrict__ tables, int ntables) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += stride) {
    uint64_t i = first + t, p = i;
    if (ntables) {
      p = 0;
      for (int b = 0; b < ntables; ++b) p |= tables[b * 256 + ((i >> (8 * b)) & 255)];
    }
    const cplx_t<T> a = psi[p];
    out[t] = double(a.x) * double(a.x) + double(a.y) * double(a.y);
  }
}

// ---------------------------------------------------------------- sampler
// Pass 1: sequential f64 sum of p over each chunk (src/measure.rs:110-118).
// A warp owns 32 consecutive chunks and lane c folds chunk c, in index
// order. The chunks stream through shared memory in windows of 256 bytes
// per chunk, copied with cp.async (16 bytes a lane, lanes 0-15 on one chunk
// and 16-31 on the next) kSumStages - 1 windows ahead of the fold, so each
// warp keeps 16 KB of loads in flight. Rows are padded by 16 bytes: the
// fold's 16-byte reads (one row per lane) then hit distinct banks.
constexpr int kSumStages = 3;
constexpr int kSumWindow = 256;             // bytes per chunk per window
constexpr int kSumRow = kSumWindow + 16;    // padded row in shared memory
constexpr int kSumStageBytes = 32 * kSumRow;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async16_s(uint32_t smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem), "l"(gmem) : "memory");
}

// prob<T> in fewer instructions: for a complex64 amplitude re*re and im*im
// are exact in f64 (24-bit significands), so re*re + im*im rounded once, as
// one fused multiply-add, equals the sum of the two rounded products.
template <typename T>
__device__ __forceinline__ double prob_fast(const cplx_t<T>& a) {
  if constexpr (sizeof(T) == 4) {
    const double re = double(a.x), im = double(a.y);
    return __fma_rn(re, re, __dmul_rn(im, im));
  } else {
    return prob<T>(a);
  }
}

// p of the amplitudes of one 16-byte read, in index order.
template <typename T>
__device__ __forceinline__ void probs16(const float4& v, double* p) {
  if constexpr (sizeof(T) == 4) {
    p[0] = prob_fast<float>(make_float2(v.x, v.y));
    p[1] = prob_fast<float>(make_float2(v.z, v.w));
  } else {
    p[0] = prob<double>(*reinterpret_cast<const double2*>(&v));
  }
}

template <typename T>
__global__ void __launch_bounds__(32) k_chunk_sums(const cplx_t<T>* __restrict__ psi, uint64_t len,
                                                   uint64_t chunk_len, uint64_t nchunks,
                                                   double* __restrict__ sums) {
  constexpr int kAmp = int(sizeof(cplx_t<T>));  // 8 or 16 bytes
  constexpr int kPerWin = kSumWindow / kAmp;     // amplitudes per chunk per window
  constexpr int kPerRead = 16 / kAmp;            // amplitudes per 16-byte read
  __shared__ __align__(16) unsigned char sbuf[kSumStages][kSumStageBytes];
  const int lane = threadIdx.x;
  const uint64_t chunk0 = uint64_t(blockIdx.x) * 32;
  if (chunk0 >= nchunks) return;
  const int live = int(umin64(32, nchunks - chunk0));
  // Windows of the warp's first chunk (no later chunk is longer).
  const uint64_t windows = (umin64(chunk_len, len - chunk0 * chunk_len) + kPerWin - 1) / kPerWin;
  const unsigned char* src0 = reinterpret_cast<const unsigned char*>(psi);
  const int half = lane >> 4, sub = lane & 15;
  // Every chunk of the warp whole (all but a state shorter than one chunk):
  // a lane's copies are then one pointer and one shared address apart.
  const bool whole = (chunk0 + uint64_t(live)) * chunk_len <= len;
  const unsigned char* lane_src = src0 + (chunk0 + uint64_t(half)) * chunk_len * kAmp + sub * 16;
  const uint64_t lane_step = 2 * chunk_len * kAmp;
  const uint32_t lane_dst = static_cast<uint32_t>(__cvta_generic_to_shared(&sbuf[0][half * kSumRow + sub * 16]));
  auto issue = [&](uint64_t w, int stage) {
    if (whole) {
      const unsigned char* src = lane_src + w * kSumWindow;
      uint32_t dst = lane_dst + uint32_t(stage) * kSumStageBytes;
      if (live == 32) {
#pragma unroll
        for (int r = 0; r < 16; ++r) cp_async16_s(dst + uint32_t(r) * 2 * kSumRow, src + r * lane_step);
      } else {
        for (int r = 0; 2 * r + half < live; ++r) cp_async16_s(dst + uint32_t(r) * 2 * kSumRow, src + r * lane_step);
      }
      return;
    }
    for (int r = 0; r < 16; ++r) {
      const int c = 2 * r + half;
      if (c >= live) break;
      const uint64_t chunk = chunk0 + c;
      const uint64_t end_b = umin64(chunk_len, len - chunk * chunk_len) * kAmp;
      const uint64_t off_b = w * kSumWindow + uint64_t(sub) * 16;
      unsigned char* dst = &sbuf[stage][c * kSumRow + sub * 16];
      const unsigned char* src = src0 + chunk * chunk_len * kAmp + off_b;
      if (off_b + 16 <= end_b)
        cp_async16(dst, src);
      else if (off_b < end_b)  // one complex64 left (a state of one amplitude)
        *reinterpret_cast<cplx_t<T>*>(dst) = *reinterpret_cast<const cplx_t<T>*>(src);
    }
  };
  for (int st = 0; st < kSumStages - 1; ++st) {
    if (uint64_t(st) < windows) issue(uint64_t(st), st);
    cp_async_commit();
  }
  double s = 0.0;
  const uint64_t my_end = lane < live ? umin64(chunk_len, len - (chunk0 + lane) * chunk_len) : 0;
  for (uint64_t w = 0; w < windows; ++w) {
    const uint64_t ahead = w + kSumStages - 1;
    if (ahead < windows) issue(ahead, int(ahead % kSumStages));
    cp_async_commit();
    cp_async_wait<kSumStages - 1>();  // window w has landed
    __syncwarp();
    const uint64_t pos = w * kPerWin;
    if (pos < my_end) {
      const float4* row = reinterpret_cast<const float4*>(&sbuf[w % kSumStages][lane * kSumRow]);
      const uint64_t n = umin64(kPerWin, my_end - pos);
      if (n == uint64_t(kPerWin)) {
        // The probabilities first (independent of the sum), then the chain.
        double p[kPerWin];
#pragma unroll
        for (int j = 0; j < kPerWin / kPerRead; ++j) probs16<T>(row[j], p + j * kPerRead);
#pragma unroll
        for (int j = 0; j < kPerWin; ++j) s = __dadd_rn(s, p[j]);
      } else {
        const cplx_t<T>* amps = reinterpret_cast<const cplx_t<T>*>(row);
        for (uint64_t j = 0; j < n; ++j) s = __dadd_rn(s, prob_fast<T>(amps[j]));
      }
    }
    __syncwarp();
  }
  if (lane < live) sums[chunk0 + lane] = s;
}

// prefix[0] = 0, prefix[c + 1] = prefix[c] + sums[c], sequentially
// (src/measure.rs:119-124).
__global__ void __launch_bounds__(256) k_prefix(const double* __restrict__ sums, uint64_t nchunks,
                                                double* __restrict__ prefix) {
  constexpr int kTile = 2048;
  __shared__ double tile[kTile];
  double p = 0.0;
  if (threadIdx.x == 0) prefix[0] = 0.0;
  for (uint64_t t0 = 0; t0 < nchunks; t0 += kTile) {
    const int n = int(umin64(kTile, nchunks - t0));
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) tile[i] = sums[t0 + i];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < n; ++i) {
        p = __dadd_rn(p, tile[i]);
        prefix[t0 + i + 1] = p;
      }
  }
}

// Total-order key of a double (f64::total_cmp order as unsigned integers).
__device__ __forceinline__ uint64_t order_key(double x) {
  const uint64_t b = uint64_t(__double_as_longlong(x));
  return (b >> 63) ? ~b : (b | (uint64_t(1) << 63));
}
__device__ __forceinline__ double from_key(uint64_t k) {
  const uint64_t b = (k >> 63) ? (k & ~(uint64_t(1) << 63)) : ~k;
  return __longlong_as_double((long long)b);
}

// targets = u * total (src/measure.rs:125), as sort keys.
__global__ void k_target_keys(const double* __restrict__ uniforms, size_t shots, const double* __restrict__ total,
                              uint64_t* __restrict__ keys) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < shots) keys[i] = order_key(__dmul_rn(uniforms[i], *total));
}

__global__ void k_keys_to_targets(const uint64_t* __restrict__ keys, size_t shots, double* __restrict__ targets) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < shots) targets[i] = from_key(keys[i]);
}

// bounds[c] = number of targets < prefix[c] (partition_point,
// src/measure.rs:128-131); chunks that hold shots are appended to `active`.
__global__ void k_bounds(const double* __restrict__ targets, size_t shots, const double* __restrict__ prefix,
                         uint64_t nchunks, uint64_t* __restrict__ bounds) {
  const uint64_t c = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c > nchunks) return;
  const double p = prefix[c];
  size_t lo = 0, hi = shots;
  while (lo < hi) {
    const size_t mid = (lo + hi) >> 1;
    if (targets[mid] < p)
      lo = mid + 1;
    else
      hi = mid;
  }
  bounds[c] = lo;
}

__global__ void k_active(const uint64_t* __restrict__ bounds, uint64_t nchunks, size_t shots,
                         uint32_t* __restrict__ active, uint32_t* __restrict__ count) {
  const uint64_t c = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  const uint64_t lo = bounds[c], hi = umin64(bounds[c + 1], shots);
  if (lo < hi) active[atomicAdd(count, 1u)] = uint32_t(c);
}

// Pass 2: one warp per chunk that holds shots (src/measure.rs:134-167). The
// warp streams the chunk's amplitudes through shared memory with cp.async
// (windows of 2 KB, two ahead of the fold). For each window the lanes
// compute the probabilities, eight each, with each block of eight's last
// nonzero position; lane 0 then folds them in index order exactly as the
// reference does: one sequential f64 sum from prefix[chunk], emitting an
// index while the next target is below the running sum. Lane 0 adds eight
// probabilities at a time and checks the target once against the eighth
// sum: the running sum never decreases (p >= +0, and adding +0 changes
// nothing), so a target at or above it emits nothing in those eight, and
// only a block that emits is redone one probability at a time (the same
// additions, so the same sums). Lane 0's work per amplitude is then one
// addition of the chain.
constexpr int kWalkWarps = 4;
constexpr int kWalkStages = 3;
constexpr int kWalkBytes = 2048;  // per window

template <typename T>
__global__ void __launch_bounds__(32 * kWalkWarps) k_walk(const cplx_t<T>* __restrict__ psi, uint64_t len,
                                                          uint64_t chunk_len, const uint32_t* __restrict__ active,
                                                          const uint32_t* __restrict__ num_active,
                                                          const double* __restrict__ prefix,
                                                          const uint64_t* __restrict__ bounds, size_t shots,
                                                          const double* __restrict__ targets,
                                                          uint64_t* __restrict__ out) {
  constexpr int kAmp = int(sizeof(cplx_t<T>));
  constexpr int kPerWin = kWalkBytes / kAmp;  // 256 or 128 amplitudes
  constexpr int kBlocks = kPerWin / 8;        // blocks of eight per window
  __shared__ __align__(16) unsigned char raw[kWalkWarps][kWalkStages][kWalkBytes];
  __shared__ __align__(16) double pw[kWalkWarps][kPerWin];
  __shared__ int8_t last_in[kWalkWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t a = blockIdx.x * kWalkWarps + warp;
  if (a >= *num_active) return;
  const uint64_t chunk = active[a];
  const uint64_t base = chunk * chunk_len;
  const uint64_t end = umin64(chunk_len, len - base);
  const uint64_t hi = umin64(bounds[chunk + 1], shots);
  uint64_t shot = bounds[chunk];
  if (shot >= hi) return;  // the whole warp: no shot lands here
  uint64_t last_nonzero = base;
  double cumulative = prefix[chunk];
  const uint64_t windows = (end + kPerWin - 1) / kPerWin;
  const uint64_t end_b = end * kAmp;
  const unsigned char* src0 = reinterpret_cast<const unsigned char*>(psi + base);
  auto issue = [&](uint64_t w, int stage) {
#pragma unroll
    for (int i = 0; i < kWalkBytes / 512; ++i) {
      const uint64_t off_b = w * kWalkBytes + uint64_t(i * 32 + lane) * 16;
      unsigned char* dst = &raw[warp][stage][(i * 32 + lane) * 16];
      if (off_b + 16 <= end_b)
        cp_async16(dst, src0 + off_b);
      else if (off_b < end_b)  // one complex64 left (a state of one amplitude)
        *reinterpret_cast<cplx_t<T>*>(dst) = *reinterpret_cast<const cplx_t<T>*>(src0 + off_b);
    }
  };
  for (int st = 0; st < kWalkStages - 1; ++st) {
    if (uint64_t(st) < windows) issue(uint64_t(st), st);
    cp_async_commit();
  }
  for (uint64_t w = 0; w < windows; ++w) {
    const uint64_t ahead = w + kWalkStages - 1;
    if (ahead < windows) issue(ahead, int(ahead % kWalkStages));
    cp_async_commit();
    cp_async_wait<kWalkStages - 1>();  // window w has landed
    __syncwarp();
    const uint64_t pos = w * kPerWin;
    const int n = int(umin64(kPerWin, end - pos));
    // Lane b: the probabilities of block b (0 past the window's end) and the
    // position of its last nonzero one (-1: none).
    if (lane < kBlocks) {
      const cplx_t<T>* amps = reinterpret_cast<const cplx_t<T>*>(&raw[warp][w % kWalkStages][0]);
      const int j0 = lane * 8;
      double p[8];
      if (j0 + 8 <= n) {
        const float4* v = reinterpret_cast<const float4*>(amps + j0);
#pragma unroll
        for (int r = 0; r < 8 * kAmp / 16; ++r) probs16<T>(v[r], p + r * (16 / kAmp));
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) p[j] = j0 + j < n ? prob_fast<T>(amps[j0 + j]) : 0.0;
      }
      int last = -1;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        pw[warp][j0 + j] = p[j];
        last = p[j] != 0.0 ? j : last;
      }
      last_in[warp][lane] = int8_t(last);
    }
    __syncwarp();
    if (lane == 0) {
      double next = targets[shot];  // shot < hi here
      for (int j0 = 0; j0 < n && shot < hi; j0 += 8) {
        double p[8];
        const double2* v = reinterpret_cast<const double2*>(&pw[warp][j0]);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const double2 x = v[r];
          p[2 * r] = x.x;
          p[2 * r + 1] = x.y;
        }
        double c8 = cumulative;
#pragma unroll
        for (int j = 0; j < 8; ++j) c8 = __dadd_rn(c8, p[j]);
        if (!(next < c8)) {  // no emission among these eight
          cumulative = c8;
          const int last = last_in[warp][j0 >> 3];
          if (last >= 0) last_nonzero = base + pos + uint64_t(j0 + last);
          continue;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (p[j] == 0.0 || shot == hi) continue;
          const uint64_t index = base + pos + uint64_t(j0 + j);
          last_nonzero = index;
          cumulative = __dadd_rn(cumulative, p[j]);
          while (next < cumulative) {
            out[shot++] = index;
            if (shot == hi) break;
            next = targets[shot];
          }
        }
      }
    }
    const bool walking = __shfl_sync(0xffffffffu, shot < hi ? 1 : 0, 0) != 0;
    __syncwarp();
    if (!walking) break;
  }
  cp_async_wait<0>();  // no copy outlives the kernel's shared memory
  if (lane == 0)
    for (; shot < hi; ++shot) out[shot] = umin64(last_nonzero, len - 1);
}

// Physical -> logical index through byte tables.
__global__ void k_remap(uint64_t* __restrict__ out, size_t count, const uint64_t* __restrict__ tables, int ntables) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t x = out[i];
  uint64_t l = 0;
  for (int b = 0; b < ntables; ++b) l |= tables[b * 256 + ((x >> (8 * b)) & 255)];
  out[i] = l;
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(kThreads) k_max_diff(const cplx_t<TA>* __restrict__ a,
                                                       const cplx_t<TB>* __restrict__ b, uint64_t len,
                                                       const uint64_t* __restrict__ ta, int nta,
                                                       const uint64_t* __restrict__ tb, int ntb,
                                                       double* __restrict__ partials) {
  __shared__ double red[32];
  double m = 0.0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    uint64_t pa = i, pb = i;
    if (nta) {
      pa = 0;
      for (int k = 0; k < nta; ++k) pa |= ta[k * 256 + ((i >> (8 * k)) & 255)];
    }
    if (ntb) {
      pb = 0;
      for (int k = 0; k < ntb; ++k) pb |= tb[k * 256 + ((i >> (8 * k)) & 255)];
    }
    const cplx_t<TA> x = a[pa];
    const cplx_t<TB> y = b[pb];
    const double dr = double(x.x) - double(y.x), di = double(x.y) - double(y.y);
    m = fmax(m, sqrt(dr * dr + di * di));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
    partials[blockIdx.x] = t;
  }
}

unsigned blocks_for(uint64_t items, int threads) { return unsigned(std::max<uint64_t>(1, (items + threads - 1) / threads)); }

template <typename T>
double norm_t(StateImpl& s) {
  const unsigned blocks = unsigned(umin64(uint64_t(s.sms) * 8, std::max<uint64_t>(1, s.size() / kThreads)));
  double* d = static_cast<double*>(s.work.get((blocks + 1) * sizeof(double)));
  k_sumsq<T><<<blocks, kThreads, 0, s.stream>>>(static_cast<const cplx_t<T>*>(s.amp), s.size(), d);
  QVDG_LAUNCH_CHECK();
  k_sum_columns<<<1, 32, 0, s.stream>>>(d, int(blocks), 1, d + blocks);
  QVDG_LAUNCH_CHECK();
  double* h = static_cast<double*>(s.host.get(sizeof(double)));
  QVDG_CUDA(cudaMemcpyAsync(h, d + blocks, sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  return *h;
}

template <typename T>
void bit_probs_t(StateImpl& s, std::vector<double>& p1, double& total) {
  const int n = int(s.n);
  const uint64_t segments = (s.size() + 1023) >> 10;  // a power of two
  uint64_t blocks = 1;
  while (blocks * 2 <= segments && blocks * 2 <= uint64_t(s.sms) * 4) blocks *= 2;
  while (segments / blocks > (uint64_t(1) << kMaxVarBits)) blocks *= 2;
  const uint64_t per_block = segments / blocks;
  int var_bits = 0;
  while ((uint64_t(1) << var_bits) < per_block) ++var_bits;
  const size_t width = size_t(n) + 1;
  double* d = static_cast<double*>(s.work.get((size_t(blocks) + 1) * width * sizeof(double)));
  k_bit_probs<T><<<unsigned(blocks), kThreads, 0, s.stream>>>(static_cast<const cplx_t<T>*>(s.amp), n, per_block,
                                                              var_bits, d);
  QVDG_LAUNCH_CHECK();
  double* sum = d + size_t(blocks) * width;
  k_sum_columns<<<blocks_for(width, 64), 64, 0, s.stream>>>(d, int(blocks), int(width), sum);
  QVDG_LAUNCH_CHECK();
  double* h = static_cast<double*>(s.host.get(width * sizeof(double)));
  QVDG_CUDA(cudaMemcpyAsync(h, sum, width * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  p1.assign(h, h + n);
  total = h[n];
}

// Byte tables mapping an index through a bit permutation: table bit q of
// the input -> bit perm[q] of the output.
int permutation_tables(StateImpl& s, const std::vector<uint32_t>& perm, uint64_t* dev) {
  const int ntables = int((s.n + 7) / 8);
  std::vector<uint64_t> t(size_t(std::max(ntables, 1)) * 256, 0);
  for (int b = 0; b < ntables; ++b)
    for (int v = 0; v < 256; ++v) {
      uint64_t p = 0;
      for (int bit = 0; bit < 8; ++bit) {
        const uint32_t q = uint32_t(8 * b + bit);
        if (q < s.n && ((v >> bit) & 1)) p |= uint64_t(1) << perm[q];
      }
      t[size_t(b) * 256 + v] = p;
    }
  QVDG_CUDA(cudaMemcpyAsync(dev, t.data(), t.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  return ntables;
}

template <typename T>
void probabilities_t(StateImpl& s, double* out_host) {
  uint64_t* tables = nullptr;
  int nt = 0;
  if (!s.identity_layout()) {
    tables = static_cast<uint64_t*>(s.work2.get(size_t((s.n + 7) / 8) * 256 * sizeof(uint64_t)));
    nt = permutation_tables(s, s.layout, tables);
  }
  const uint64_t chunk = uint64_t(1) << 24;
  const uint64_t len = s.size();
  double* d = static_cast<double*>(s.work.get(std::min(chunk, len) * sizeof(double)));
  for (uint64_t first = 0; first < len; first += chunk) {
    const uint64_t count = std::min(chunk, len - first);
    k_probs<T><<<unsigned(umin64(blocks_for(count, kThreads), uint64_t(s.sms) * 16)), kThreads, 0,
                 s.stream>>>(static_cast<const cplx_t<T>*>(s.amp), d, first, count, tables, nt);
    QVDG_LAUNCH_CHECK();
    QVDG_CUDA(cudaMemcpyAsync(out_host + first, d, count * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    QVDG_CUDA(cudaStreamSynchronize(s.stream));
  }
}

// The sampler's outcomes (logical indices) left in the workspace at *out_dev;
// returns their number. The workspace's `keys` and `tmp` regions (shots
// entries each) are free afterwards and returned for reuse.
template <typename T>
size_t sample_device_t(StateImpl& s, size_t shots, const double* uniforms_host, uint64_t** out_dev,
                       uint64_t** keys_dev, uint64_t** tmp_dev) {
  const uint64_t len = s.size();
  // CHUNK_BLOCKS (4096) blocks of LANES amplitudes (8 for f32, 4 for f64).
  const uint64_t chunk_len = sizeof(T) == 4 ? 32768 : 16384;
  const uint64_t nchunks = (len + chunk_len - 1) / chunk_len;
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_sums = 0;
  const size_t o_prefix = o_sums + align(nchunks * 8);
  const size_t o_bounds = o_prefix + align((nchunks + 1) * 8);
  const size_t o_active = o_bounds + align((nchunks + 1) * 8);
  const size_t o_count = o_active + align(nchunks * 4);
  const size_t o_uni = o_count + 256;
  const size_t o_keys = o_uni + align(shots * 8);
  const size_t o_tmp = o_keys + align(shots * 8);
  const size_t o_targets = o_tmp + align(shots * 8);
  const size_t o_out = o_targets + align(shots * 8);
  const size_t o_tables = o_out + align(shots * 8);
  const size_t total_bytes = o_tables + align(size_t((s.n + 7) / 8 + 1) * 256 * 8);
  char* w = static_cast<char*>(s.work.get(total_bytes));
  double* sums = reinterpret_cast<double*>(w + o_sums);
  double* prefix = reinterpret_cast<double*>(w + o_prefix);
  uint64_t* bounds = reinterpret_cast<uint64_t*>(w + o_bounds);
  uint32_t* active = reinterpret_cast<uint32_t*>(w + o_active);
  uint32_t* count = reinterpret_cast<uint32_t*>(w + o_count);
  double* uni = reinterpret_cast<double*>(w + o_uni);
  uint64_t* keys = reinterpret_cast<uint64_t*>(w + o_keys);
  uint64_t* tmp = reinterpret_cast<uint64_t*>(w + o_tmp);
  double* targets = reinterpret_cast<double*>(w + o_targets);
  uint64_t* out = reinterpret_cast<uint64_t*>(w + o_out);
  uint64_t* tables = reinterpret_cast<uint64_t*>(w + o_tables);
  const cplx_t<T>* psi = static_cast<const cplx_t<T>*>(s.amp);

  QVDG_CUDA(cudaMemcpyAsync(uni, uniforms_host, shots * 8, cudaMemcpyHostToDevice, s.stream));
  static bool carveout = false;  // per instantiation
  if (!carveout) {
    // Eight one-warp blocks per SM (26 KB of shared memory each): all of the
    // unified L1/shared storage as shared memory.
    QVDG_CUDA(cudaFuncSetAttribute(k_chunk_sums<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   int(cudaSharedmemCarveoutMaxShared)));
    carveout = true;
  }
  k_chunk_sums<T><<<unsigned((nchunks + 31) / 32), 32, 0, s.stream>>>(psi, len, chunk_len, nchunks, sums);
  QVDG_LAUNCH_CHECK();
  k_prefix<<<1, 256, 0, s.stream>>>(sums, nchunks, prefix);
  QVDG_LAUNCH_CHECK();
  k_target_keys<<<blocks_for(shots, kThreads), kThreads, 0, s.stream>>>(uni, shots, prefix + nchunks, keys);
  QVDG_LAUNCH_CHECK();
  DeviceScratch& sort_work = s.work2;
  radix_sort_u64(keys, tmp, shots, sort_work, s.stream);
  k_keys_to_targets<<<blocks_for(shots, kThreads), kThreads, 0, s.stream>>>(keys, shots, targets);
  QVDG_LAUNCH_CHECK();
  k_bounds<<<blocks_for(nchunks + 1, kThreads), kThreads, 0, s.stream>>>(targets, shots, prefix, nchunks, bounds);
  QVDG_LAUNCH_CHECK();
  QVDG_CUDA(cudaMemsetAsync(count, 0, sizeof(uint32_t), s.stream));
  k_active<<<blocks_for(nchunks, kThreads), kThreads, 0, s.stream>>>(bounds, nchunks, shots, active, count);
  QVDG_LAUNCH_CHECK();
  // Shots that land in chunks: min(bounds[nchunks], shots).
  uint64_t* hb = static_cast<uint64_t*>(s.host.get(16));
  QVDG_CUDA(cudaMemcpyAsync(hb, bounds + nchunks, 8, cudaMemcpyDeviceToHost, s.stream));
  uint32_t* hc = reinterpret_cast<uint32_t*>(hb + 1);
  QVDG_CUDA(cudaMemcpyAsync(hc, count, 4, cudaMemcpyDeviceToHost, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  const size_t found = size_t(umin64(hb[0], shots));
  const uint32_t num_active = *hc;
  if (num_active > 0) {
    const unsigned walk_blocks = unsigned((num_active + kWalkWarps - 1) / kWalkWarps);
    k_walk<T><<<walk_blocks, 32 * kWalkWarps, 0, s.stream>>>(psi, len, chunk_len, active, count, prefix, bounds,
                                                            shots, targets, out);
    QVDG_LAUNCH_CHECK();
  }
  if (!s.identity_layout() && found > 0) {
    // physical bit p holds logical qubit q: inverse of the layout
    std::vector<uint32_t> inverse(s.n);
    for (uint32_t q = 0; q < s.n; ++q) inverse[s.layout[q]] = q;
    const int nt = permutation_tables(s, inverse, tables);
    k_remap<<<blocks_for(found, kThreads), kThreads, 0, s.stream>>>(out, found, tables, nt);
    QVDG_LAUNCH_CHECK();
  }
  *out_dev = out;
  *keys_dev = keys;
  *tmp_dev = tmp;
  return found;
}

template <typename T>
size_t sample_t(StateImpl& s, size_t shots, const double* uniforms_host, uint64_t* out_host) {
  if (shots == 0) return 0;
  uint64_t *out = nullptr, *keys = nullptr, *tmp = nullptr;
  const size_t found = sample_device_t<T>(s, shots, uniforms_host, &out, &keys, &tmp);
  if (found > 0) QVDG_CUDA(cudaMemcpyAsync(out_host, out, found * 8, cudaMemcpyDeviceToHost, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  return found;
}

// Classical keys of outcomes: bit c of key i = bit q of outcome i for each
// (q, c) measurement (count_outcomes, src/simulator.rs:187-230).
struct MeasureMap {
  uint8_t q[64], c[64];
  int32_t n;
};

__global__ void k_outcome_keys(const uint64_t* __restrict__ out, size_t found, const MeasureMap m,
                               uint64_t* __restrict__ keys) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= found) return;
  const uint64_t o = out[i];
  uint64_t k = 0;
  for (int j = 0; j < m.n; ++j) k |= ((o >> m.q[j]) & 1ull) << m.c[j];
  keys[i] = k;
}

template <typename T>
size_t counts_t(StateImpl& s, size_t shots, const double* uniforms_host, const MeasureMap& m,
                std::vector<uint64_t>& keys_out, std::vector<uint64_t>& counts_out) {
  keys_out.clear();
  counts_out.clear();
  if (shots == 0) return 0;
  uint64_t *out = nullptr, *keys = nullptr, *tmp = nullptr;
  const size_t found = sample_device_t<T>(s, shots, uniforms_host, &out, &keys, &tmp);
  if (found == 0) return 0;
  k_outcome_keys<<<blocks_for(found, kThreads), kThreads, 0, s.stream>>>(out, found, m, keys);
  QVDG_LAUNCH_CHECK();
  radix_sort_u64(keys, tmp, found, s.work2, s.stream);
  std::vector<uint64_t> sorted(found);
  QVDG_CUDA(cudaMemcpyAsync(sorted.data(), keys, found * 8, cudaMemcpyDeviceToHost, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  for (size_t i = 0; i < found;) {
    size_t j = i + 1;
    while (j < found && sorted[j] == sorted[i]) ++j;
    keys_out.push_back(sorted[i]);
    counts_out.push_back(j - i);
    i = j;
  }
  return found;
}

// <psi|P|psi> for a Pauli string with X/Y on the bits of x, Z/Y on the bits of
// z (physical): P|j> = i^nY (-1)^popc(j & z) |j ^ x>, so the value is
// i^nY * sum_j conj(psi[j ^ x]) psi[j] (-1)^popc(j & z). Per-block partial
// sums (re, im) in double precision, summed in order.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pauli(const cplx_t<T>* __restrict__ psi, uint64_t len, uint64_t x,
                                                    uint64_t z, double* __restrict__ partials) {
  __shared__ double red[32];
  double re = 0.0, im = 0.0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < len; j += stride) {
    const cplx_t<T> a = psi[j], b = psi[j ^ x];
    // conj(b) * a
    const double pr = double(b.x) * double(a.x) + double(b.y) * double(a.y);
    const double pi = double(b.x) * double(a.y) - double(b.y) * double(a.x);
    const double sgn = (__popcll(j & z) & 1) ? -1.0 : 1.0;
    re += sgn * pr;
    im += sgn * pi;
  }
  const double tr = block_sum(re, red);
  __syncthreads();
  const double ti = block_sum(im, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = tr;
    partials[2 * blockIdx.x + 1] = ti;
  }
}

template <typename T>
double pauli_t(StateImpl& s, uint64_t x, uint64_t z, int ny) {
  const unsigned blocks = unsigned(umin64(uint64_t(s.sms) * 8, std::max<uint64_t>(1, s.size() / kThreads)));
  double* d = static_cast<double*>(s.work.get((2 * size_t(blocks) + 2) * sizeof(double)));
  k_pauli<T><<<blocks, kThreads, 0, s.stream>>>(static_cast<const cplx_t<T>*>(s.amp), s.size(), x, z, d);
  QVDG_LAUNCH_CHECK();
  k_sum_columns<<<1, 32, 0, s.stream>>>(d, int(blocks), 2, d + 2 * blocks);
  QVDG_LAUNCH_CHECK();
  double* h = static_cast<double*>(s.host.get(2 * sizeof(double)));
  QVDG_CUDA(cudaMemcpyAsync(h, d + 2 * blocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  const double re = h[0], im = h[1];
  switch (ny & 3) {
    case 0: return re;
    case 1: return -im;
    case 2: return -re;
    default: return im;
  }
}

}  // namespace

double max_abs_diff(StateImpl& a, StateImpl& b) {
  if (a.n != b.n) throw Error(1, "states of different sizes");
  const int nt = int((a.n + 7) / 8);
  const size_t tbytes = size_t(nt) * 256 * sizeof(uint64_t);
  uint64_t* ta = static_cast<uint64_t*>(a.work2.get(tbytes));
  uint64_t* tb = static_cast<uint64_t*>(b.work2.get(tbytes));
  const int nta = a.identity_layout() ? 0 : permutation_tables(a, a.layout, ta);
  const int ntb = b.identity_layout() ? 0 : permutation_tables(b, b.layout, tb);
  QVDG_CUDA(cudaStreamSynchronize(b.stream));
  const unsigned blocks = unsigned(umin64(uint64_t(a.sms) * 8, std::max<uint64_t>(1, a.size() / kThreads)));
  double* d = static_cast<double*>(a.work.get(blocks * sizeof(double)));
  if (a.bits == 32 && b.bits == 32)
    k_max_diff<float, float><<<blocks, kThreads, 0, a.stream>>>(static_cast<const float2*>(a.amp),
        static_cast<const float2*>(b.amp), a.size(), ta, nta, tb, ntb, d);
  else if (a.bits == 32)
    k_max_diff<float, double><<<blocks, kThreads, 0, a.stream>>>(static_cast<const float2*>(a.amp),
        static_cast<const double2*>(b.amp), a.size(), ta, nta, tb, ntb, d);
  else if (b.bits == 32)
    k_max_diff<double, float><<<blocks, kThreads, 0, a.stream>>>(static_cast<const double2*>(a.amp),
        static_cast<const float2*>(b.amp), a.size(), ta, nta, tb, ntb, d);
  else
    k_max_diff<double, double><<<blocks, kThreads, 0, a.stream>>>(static_cast<const double2*>(a.amp),
        static_cast<const double2*>(b.amp), a.size(), ta, nta, tb, ntb, d);
  QVDG_LAUNCH_CHECK();
  std::vector<double> h(blocks);
  QVDG_CUDA(cudaMemcpyAsync(h.data(), d, blocks * sizeof(double), cudaMemcpyDeviceToHost, a.stream));
  QVDG_CUDA(cudaStreamSynchronize(a.stream));
  double m = 0.0;
  for (double x : h) m = std::max(m, x);
  return m;
}

double norm_sqr(StateImpl& s) { return s.bits == 32 ? norm_t<float>(s) : norm_t<double>(s); }

void bit_probabilities(StateImpl& s, std::vector<double>& p1, double& total) {
  if (s.bits == 32)
    bit_probs_t<float>(s, p1, total);
  else
    bit_probs_t<double>(s, p1, total);
}

double probability_one(StateImpl& s, uint32_t physical_bit) {
  std::vector<double> p1;
  double total;
  bit_probabilities(s, p1, total);
  return p1[physical_bit];
}

void probabilities(StateImpl& s, double* out_host) {
  if (s.bits == 32)
    probabilities_t<float>(s, out_host);
  else
    probabilities_t<double>(s, out_host);
}

size_t sample_counts(StateImpl& s, size_t shots, const double* uniforms_host, const uint32_t* qubits,
                     const uint32_t* clbits, size_t nm, std::vector<uint64_t>& keys, std::vector<uint64_t>& counts) {
  MeasureMap m{};
  // Every pair ORs its bit into the key, as the reference's keyed counting
  // does (src/simulator.rs:204-210); pairs repeated exactly are kept once.
  for (size_t i = 0; i < nm && m.n < 64; ++i) {
    bool dup = false;
    for (int j = 0; j < m.n; ++j) dup = dup || (m.q[j] == qubits[i] && m.c[j] == clbits[i]);
    if (dup) continue;
    m.q[m.n] = uint8_t(qubits[i]);
    m.c[m.n] = uint8_t(clbits[i]);
    ++m.n;
  }
  return s.bits == 32 ? counts_t<float>(s, shots, uniforms_host, m, keys, counts)
                      : counts_t<double>(s, shots, uniforms_host, m, keys, counts);
}

double expect_pauli(StateImpl& s, uint64_t x, uint64_t z, int ny) {
  return s.bits == 32 ? pauli_t<float>(s, x, z, ny) : pauli_t<double>(s, x, z, ny);
}

size_t sample_unordered(StateImpl& s, size_t shots, const double* uniforms_host, uint64_t* out_host) {
  return s.bits == 32 ? sample_t<float>(s, shots, uniforms_host, out_host)
                      : sample_t<double>(s, shots, uniforms_host, out_host);
}


// ---------------------------------------------------------------------------
// Per-bit probabilities with no allocation (qvdg_bit_probabilities_noalloc).
//
// For callers that cannot allocate device memory: the k_bit_probs partials
// and their column sums live in one file-scope device array instead of the
// state's workspace. At most kNoAllocMaxBlocks blocks of k_bit_probs, each
// writing kNoAllocMaxQubits + 1 doubles, plus one row of totals:
// (512 + 1) * 36 doubles = 147,744 bytes, held on every device that loads
// this library until the process exits. Every row the kernels read is
// written earlier in the same call, so nothing needs clearing; calls that
// overlap on the GPU share the array and race.
constexpr uint32_t kNoAllocMaxQubits = 35;
constexpr uint64_t kNoAllocMaxBlocks = 512;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_noalloc_scratch[(kNoAllocMaxBlocks + 1) * (kNoAllocMaxQubits + 1)];

namespace {

std::mutex g_noalloc_mutex;
double* g_noalloc_address[kNoAllocMaxDevices] = {};

// The device address of g_noalloc_scratch on `device` (the current device).
// In host code g_noalloc_scratch only names the symbol; its address on a
// device comes from cudaGetSymbolAddress, looked up once per device.
double* noalloc_scratch(int device) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_address[device] == nullptr) {
    void* p = nullptr;
    QVDG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_address[device] = static_cast<double*>(p);
  }
  return g_noalloc_address[device];
}

template <typename T>
void bit_probs_noalloc_t(const void* amplitudes, uint32_t n, cudaStream_t stream, double* p1, double* total) {
  int device = 0;
  QVDG_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kNoAllocMaxDevices)
    throw Error(QVDG_ERR_UNSUPPORTED, "device index beyond the no-allocation limit of 64 devices");
  double* d = noalloc_scratch(device);
  int sms = 0;
  QVDG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const uint64_t segments = ((uint64_t(1) << n) + 1023) >> 10;
  uint64_t blocks = 1;
  while (blocks * 2 <= segments && blocks * 2 <= uint64_t(sms) * 4 && blocks * 2 <= kNoAllocMaxBlocks) blocks *= 2;
  while (segments / blocks > (uint64_t(1) << kMaxVarBits)) blocks *= 2;
  if (blocks > kNoAllocMaxBlocks) throw Error(QVDG_ERR_UNSUPPORTED, "state too large for the no-allocation scratch");
  const uint64_t per_block = segments / blocks;
  int var_bits = 0;
  while ((uint64_t(1) << var_bits) < per_block) ++var_bits;
  const size_t width = size_t(n) + 1;
  k_bit_probs<T><<<unsigned(blocks), kThreads, 0, stream>>>(static_cast<const cplx_t<T>*>(amplitudes), int(n),
                                                            per_block, var_bits, d);
  QVDG_LAUNCH_CHECK();
  double* sum = d + size_t(blocks) * width;
  k_sum_columns<<<blocks_for(width, 64), 64, 0, stream>>>(d, int(blocks), int(width), sum);
  QVDG_LAUNCH_CHECK();
  QVDG_CUDA(cudaMemcpyAsync(p1, sum, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
  QVDG_CUDA(cudaMemcpyAsync(total, sum + n, sizeof(double), cudaMemcpyDeviceToHost, stream));
  QVDG_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace

void bit_probabilities_noalloc(const void* amplitudes, uint32_t num_qubits, uint32_t precision_bits,
                               cudaStream_t stream, double* p1, double* total) {
  if (num_qubits > kNoAllocMaxQubits)
    throw Error(QVDG_ERR_UNSUPPORTED, "num_qubits " + std::to_string(num_qubits) +
                                          " exceeds the no-allocation limit of 35 qubits");
  if (precision_bits == 32)
    bit_probs_noalloc_t<float>(amplitudes, num_qubits, stream, p1, total);
  else
    bit_probs_noalloc_t<double>(amplitudes, num_qubits, stream, p1, total);
}

}  // namespace qvdg
