// Register-blocked stage kernel: the staged tile pass on the CUDA cores,
// gate by gate without fusing matrices.
//
// A stage (the reference's cache-blocked stage, src/blocking.rs:57-302) runs
// over tiles of 2^L amplitudes held in shared memory. Within a tile the
// stage's gates are cut into *register passes*: each names four tile bits G;
// a thread loads the 16 amplitudes of one G-subcube into registers, applies
// every gate of the pass there and stores them back. A register pass takes
// the gates, in dependency order, whose dense targets lie in G (controls may
// be anywhere: outside G they are a per-thread or per-tile predicate, inside
// a mask of active register groups) and every diagonal gate that is ready
// (a diagonal reads bits inside G per register and bits outside G from the
// thread's subcube base). So one shared-memory round trip serves several
// gates, and no matrix is ever multiplied out: a 1-qubit gate costs 4 to 8
// FMAs per amplitude (real and RX-type matrices take the cheaper forms), a
// +-1 diagonal (CZ and the like) only toggles sign bits.
//
// Tiles are double-buffered: the next tile's 16-byte cp.async copies are in
// flight while the current one is computed, and a finished tile is stored
// from shared memory straight to HBM.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "program.hpp"
#include "stage_kernel.hpp"

namespace qvdg {

namespace {

constexpr int kRegThreads = 512;
constexpr size_t kRegBlobBudget = 64 * 1024;

enum : uint8_t { kRegDense1 = 0, kRegDense2 = 1, kRegSign = 2, kRegPhase = 3, kRegSign2 = 4 };
enum : uint8_t { kSpecGeneral = 0, kSpecReal = 1, kSpecRx = 2, kSpecDiagReal = 3 };

// Shared-memory position of tile element e: bits 1-3 XORed with bits 5-7,
// 9-11 and 13-15 (bit 0 is kept, so element pairs 2v, 2v+1 stay one 16-byte
// slot for cp.async). XOR-linear and an involution.
__host__ __device__ __forceinline__ uint32_t reg_swz(uint32_t e) {
  return e ^ (((e >> 4) ^ (e >> 8) ^ (e >> 12)) & 14u);
}

struct RegPassHdr {
  uint8_t g[4];         // tile bits held in registers, ascending: register index bit i <-> tile bit g[i]
  uint16_t num_gates;
  uint16_t pair;        // g[0] == 0: registers j, j^1 are one 16-byte slot (complex64)
  uint32_t first_gate;  // index of the pass's first gate
  uint32_t pad;
  uint16_t off[16];     // tile element offset of register j (j deposited over g)
};
static_assert(sizeof(RegPassHdr) == 48, "header layout");

// Dispatch codes of the register kernel (one switch per gate).
enum : uint16_t {
  kOpDense1 = 0,         // + 4 * spec + target register bit (16 codes), no register controls
  kOpDense1Masked = 16,  // any matrix, register controls
  kOpDense2 = 17,        // + index of (t0, t1) in (0,1) (0,2) (0,3) (1,2) (1,3) (2,3)
  kOpDense2Masked = 23,
  kOpSign2 = 24,
  kOpSign = 25,
  kOpPhase = 26,
};

struct RegGate {
  // Hot: the first 16 bytes, read with one 16-byte load per gate.
  uint16_t op;        // kOp* dispatch code
  uint16_t pmask;     // dense: register bases j (target bits clear) whose group is active (0xffff: all)
  uint8_t t0, t1;     // dense: register bits of matrix bits 0 and 1; kOpSign2: bit of index bits 0, 1 in the
                      // word (tile base | subcube base << 48), 63: none
  uint8_t pred;       // 1 when the gate has controls outside the registers (gcm/lcm)
  uint8_t k;          // diagonal: targets
  uint32_t data;      // byte offset in the pass blob: matrix, diagonal entries or sign masks
  uint32_t table;     // diagonal: byte offset of the 16 register index parts (uint16)
  // Cold.
  uint32_t lcm, lcv;  // controls on tile bits outside the registers (per-thread predicate)
  uint64_t gcm, gcv;  // controls on global bits (per-tile predicate)
  uint8_t tgt[16];    // diagonal target i: 0x40|j register bit j, l < 0x40 tile bit, 0x80|p global bit p
  uint8_t kind, spec; // host bookkeeping
  uint8_t pad1[6];
};
static_assert(sizeof(RegGate) == 64, "gate layout");

// ---------------------------------------------------------------------------
// Device side.

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ cplx_t<T> neg_c(cplx_t<T> a) {
  return make_c<T>(-a.x, -a.y);
}

template <typename T>
__device__ __forceinline__ cplx_t<T> mul_c(cplx_t<T> m, cplx_t<T> x) {
  return make_c<T>(fma(m.x, x.x, -m.y * x.y), fma(m.x, x.y, m.y * x.x));
}

// y = m0 * x0 + m1 * x1 for complex m (general), real m (spec real: the
// imaginary parts are zero) or the RX form (m0 real, m1 imaginary).
template <typename T, int SPEC>
__device__ __forceinline__ cplx_t<T> row2(cplx_t<T> m0, cplx_t<T> m1, cplx_t<T> x0, cplx_t<T> x1) {
  if (SPEC == kSpecReal) return make_c<T>(fma(m0.x, x0.x, m1.x * x1.x), fma(m0.x, x0.y, m1.x * x1.y));
  if (SPEC == kSpecRx) return make_c<T>(fma(m0.x, x0.x, -m1.y * x1.y), fma(m0.x, x0.y, m1.y * x1.x));
  if (SPEC == kSpecDiagReal)
    return make_c<T>(fma(m0.x, x0.x, fma(m1.x, x1.x, -m1.y * x1.y)), fma(m0.x, x0.y, fma(m1.x, x1.y, m1.y * x1.x)));
  return make_c<T>(fma(m0.x, x0.x, fma(-m0.y, x0.y, fma(m1.x, x1.x, -m1.y * x1.y))),
                   fma(m0.x, x0.y, fma(m0.y, x0.x, fma(m1.x, x1.y, m1.y * x1.x))));
}
// Second rows: the RX form has an imaginary first entry and a real second;
// the real-diagonal form a complex first entry and a real second.
template <typename T, int SPEC>
__device__ __forceinline__ cplx_t<T> row2b(cplx_t<T> m0, cplx_t<T> m1, cplx_t<T> x0, cplx_t<T> x1) {
  if (SPEC == kSpecRx) return make_c<T>(fma(m1.x, x1.x, -m0.y * x0.y), fma(m1.x, x1.y, m0.y * x0.x));
  if (SPEC == kSpecDiagReal)
    return make_c<T>(fma(m1.x, x1.x, fma(m0.x, x0.x, -m0.y * x0.y)), fma(m1.x, x1.y, fma(m0.x, x0.y, m0.y * x0.x)));
  return row2<T, SPEC>(m0, m1, x0, x1);
}

// Sign flip of a complex value where `bit` is 1, on the sign bits.
// (bit 31 of `t` set: negate).
__device__ __forceinline__ void flip(float2& x, uint32_t t) {
  const uint32_t s = t & 0x80000000u;
  x.x = __uint_as_float(__float_as_uint(x.x) ^ s);
  x.y = __uint_as_float(__float_as_uint(x.y) ^ s);
}
__device__ __forceinline__ void flip(double2& x, uint32_t t) {
  const unsigned long long s = (unsigned long long)(t & 0x80000000u) << 32;
  x.x = __longlong_as_double(__double_as_longlong(x.x) ^ s);
  x.y = __longlong_as_double(__double_as_longlong(x.y) ^ s);
}

template <typename T, int TB, int SPEC, bool MASKED>
__device__ __forceinline__ void apply1(cplx_t<T> (&a)[16], const cplx_t<T>* m, uint32_t pmask) {
  const cplx_t<T> m00 = m[0], m01 = m[1], m10 = m[2], m11 = m[3];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << TB)) continue;
    const cplx_t<T> x0 = a[j], x1 = a[j | (1 << TB)];
    const cplx_t<T> y0 = row2<T, SPEC>(m00, m01, x0, x1);
    const cplx_t<T> y1 = row2b<T, SPEC>(m10, m11, x0, x1);
    if (MASKED) {
      const bool on = (pmask >> j) & 1u;
      a[j] = on ? y0 : x0;
      a[j | (1 << TB)] = on ? y1 : x1;
    } else {
      a[j] = y0;
      a[j | (1 << TB)] = y1;
    }
  }
}

template <typename T, int SPEC, bool MASKED>
__device__ __forceinline__ void apply1_bit(cplx_t<T> (&a)[16], int tb, const cplx_t<T>* m, uint32_t pmask) {
  switch (tb) {
    case 0: apply1<T, 0, SPEC, MASKED>(a, m, pmask); break;
    case 1: apply1<T, 1, SPEC, MASKED>(a, m, pmask); break;
    case 2: apply1<T, 2, SPEC, MASKED>(a, m, pmask); break;
    default: apply1<T, 3, SPEC, MASKED>(a, m, pmask); break;
  }
}

// Dense 2-qubit gate on register bits B0 < B1 (matrix bit 0 <-> B0).
template <typename T, int B0, int B1, bool MASKED>
__device__ __forceinline__ void apply2(cplx_t<T> (&a)[16], const cplx_t<T>* m, uint32_t pmask) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & ((1 << B0) | (1 << B1))) continue;
    const int i[4] = {j, j | (1 << B0), j | (1 << B1), j | (1 << B0) | (1 << B1)};
    cplx_t<T> x[4] = {a[i[0]], a[i[1]], a[i[2]], a[i[3]]};
    cplx_t<T> y[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      cplx_t<T> acc = make_c<T>(T(0), T(0));
#pragma unroll
      for (int c = 0; c < 4; ++c) cmac<T>(acc, m[r * 4 + c], x[c]);
      y[r] = acc;
    }
    const bool on = !MASKED || ((pmask >> j) & 1u);
#pragma unroll
    for (int r = 0; r < 4; ++r) a[i[r]] = on ? y[r] : x[r];
  }
}

template <typename T, bool MASKED>
__device__ __forceinline__ void apply2_any(cplx_t<T> (&a)[16], const RegGate& g, const cplx_t<T>* m) {
  switch (g.t0 * 4 + g.t1) {
    case 1: apply2<T, 0, 1, MASKED>(a, m, g.pmask); break;
    case 2: apply2<T, 0, 2, MASKED>(a, m, g.pmask); break;
    case 3: apply2<T, 0, 3, MASKED>(a, m, g.pmask); break;
    case 6: apply2<T, 1, 2, MASKED>(a, m, g.pmask); break;
    case 7: apply2<T, 1, 3, MASKED>(a, m, g.pmask); break;
    default: apply2<T, 2, 3, MASKED>(a, m, g.pmask); break;
  }
}

template <typename T>
__device__ __forceinline__ void flip_mask(cplx_t<T> (&a)[16], uint32_t mask) {
#pragma unroll
  for (int j = 0; j < 16; ++j) flip(a[j], mask << (31 - j));
}

// Index bits of a diagonal gate that do not come from the registers.
__device__ __forceinline__ uint32_t diag_fixed(const RegGate& g, uint32_t eb, uint64_t tile_base) {
  uint32_t idx = 0;
  for (int i = 0; i < g.k; ++i) {
    const uint32_t t = g.tgt[i];
    if (t & 0x80)
      idx |= uint32_t((tile_base >> (t & 0x7f)) & 1u) << i;
    else if (!(t & 0x40))
      idx |= ((eb >> t) & 1u) << i;
  }
  return idx;
}

template <typename T>
__device__ void run_register_pass(cplx_t<T>* tile, const RegPassHdr& h, const RegGate* gates,
                                  const unsigned char* blob, int L, uint64_t tile_base) {
  using C2 = cplx_t<T>;
  const uint32_t nsub = 1u << (L - 4);
  for (uint32_t s = threadIdx.x; s < nsub; s += blockDim.x) {
    uint32_t eb = s;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t p = h.g[i];
      eb = ((eb >> p) << (p + 1)) | (eb & ((1u << p) - 1u));
    }
    C2 a[16];
    if (sizeof(C2) == 8 && h.pair) {
#pragma unroll
      for (int j = 0; j < 16; j += 2) {
        const float4 v = *reinterpret_cast<const float4*>(tile + reg_swz(eb | h.off[j]));
        a[j] = make_c<T>(T(v.x), T(v.y));
        a[j + 1] = make_c<T>(T(v.z), T(v.w));
      }
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) a[j] = tile[reg_swz(eb | h.off[j])];
    }
    // Bits a sign gate reads outside the registers: the tile's global bits
    // and the subcube's tile bits (at 48 and up).
    const uint64_t where = tile_base | (uint64_t(eb) << 48);
    for (uint32_t gi = h.first_gate; gi < h.first_gate + h.num_gates; ++gi) {
      const RegGate& g = gates[gi];
      const uint4 hot = *reinterpret_cast<const uint4*>(&g);
      const uint32_t op = hot.x & 0xffffu, pmask = hot.x >> 16;
      const uint32_t t0 = hot.y & 0xffu, t1 = (hot.y >> 8) & 0xffu;
      if ((hot.y >> 16) & 0xffu)
        if ((tile_base & g.gcm) != g.gcv || (eb & g.lcm) != g.lcv) continue;
      const unsigned char* data = blob + hot.z;
      const C2* m = reinterpret_cast<const C2*>(data);
      switch (op >= kOpSign2 ? op : (op >= kOpDense2 ? 1u : 0u)) {
        case 0:  // dense 1-qubit
          if (op == kOpDense1Masked) {
            apply1_bit<T, kSpecGeneral, true>(a, int(t0), m, pmask);
          } else {
            const int tb = int(op & 3u);
            switch ((op - kOpDense1) >> 2) {
              case kSpecReal: apply1_bit<T, kSpecReal, false>(a, tb, m, 0); break;
              case kSpecRx: apply1_bit<T, kSpecRx, false>(a, tb, m, 0); break;
              case kSpecDiagReal: apply1_bit<T, kSpecDiagReal, false>(a, tb, m, 0); break;
              default: apply1_bit<T, kSpecGeneral, false>(a, tb, m, 0); break;
            }
          }
          break;
        case 1: {  // dense 2-qubit
          RegGate gg;
          gg.t0 = uint8_t(t0);
          gg.t1 = uint8_t(t1);
          gg.pmask = uint16_t(pmask);
          if (op == kOpDense2Masked)
            apply2_any<T, true>(a, gg, m);
          else
            apply2_any<T, false>(a, gg, m);
          break;
        }
        case kOpSign2: {
          const uint16_t* masks = reinterpret_cast<const uint16_t*>(data);
          flip_mask<T>(a, masks[uint32_t((where >> t0) & 1u) | (uint32_t((where >> t1) & 1u) << 1)]);
          break;
        }
        case kOpSign: {
          const uint16_t* masks = reinterpret_cast<const uint16_t*>(data);
          flip_mask<T>(a, masks[diag_fixed(g, eb, tile_base)]);
          break;
        }
        default: {  // kOpPhase
          const uint16_t* ridx = reinterpret_cast<const uint16_t*>(blob + hot.w);
          const uint32_t f = diag_fixed(g, eb, tile_base);
#pragma unroll
          for (int j = 0; j < 16; ++j) a[j] = mul_c<T>(m[f | ridx[j]], a[j]);
          break;
        }
      }
    }
    if (sizeof(C2) == 8 && h.pair) {
#pragma unroll
      for (int j = 0; j < 16; j += 2)
        *reinterpret_cast<float4*>(tile + reg_swz(eb | h.off[j])) =
            make_float4(float(a[j].x), float(a[j].y), float(a[j + 1].x), float(a[j + 1].y));
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) tile[reg_swz(eb | h.off[j])] = a[j];
    }
  }
  __syncthreads();
}

// complex128 tiles are 2^12 amplitudes (256 subcubes): 256 threads, which
// leaves room for twice the registers.
template <typename T>
constexpr int reg_threads() {
  return sizeof(T) == 4 ? kRegThreads : kRegThreads / 2;
}

template <typename T>
__global__ void __launch_bounds__(reg_threads<T>(), 1)
    k_stage_reg(cplx_t<T>* __restrict__ psi, const TileGeom geo, const unsigned char* __restrict__ blob_all) {
  using C2 = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint8_t tile_bits[48];
  __shared__ uint64_t map_lo[32], map_hi[32];
  const int tid = threadIdx.x;
  const int L = geo.L, B = geo.B;
  const uint32_t n_el = 1u << L;
  C2* const buf0 = reinterpret_cast<C2*>(smem);  // tiles at buf0 and buf0 + n_el
  unsigned char* blob = smem + 2 * sizeof(C2) * n_el;

  for (int i = tid; i < 48; i += blockDim.x) tile_bits[i] = geo.tile_bits[i];
  {
    const uint4* src = reinterpret_cast<const uint4*>(blob_all + geo.tc_offset);
    uint4* dst = reinterpret_cast<uint4*>(blob);
    for (uint32_t i = tid; i < geo.tc_bytes / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  // Tile element e -> physical index offset: the low B bits are physical
  // bits 0..B-1; the others go through two tables of their set bits.
  const int nfree = L - B, nlo = nfree < 5 ? nfree : 5;
  for (int i = tid; i < 32; i += blockDim.x) {
    uint64_t a = 0, b = 0;
    for (int j = 0; j < nlo; ++j)
      if ((i >> j) & 1) a |= uint64_t(1) << tile_bits[B + j];
    for (int j = nlo; j < nfree; ++j)
      if ((i >> (j - nlo)) & 1) b |= uint64_t(1) << tile_bits[B + j];
    map_lo[i] = a;
    map_hi[i] = b;
  }
  __syncthreads();
  const uint32_t lowmask = (1u << B) - 1u;
  auto phys = [&](uint64_t base, uint32_t e) -> uint64_t {
    const uint32_t r = e >> B;
    return base | map_lo[r & 31] | map_hi[r >> nlo] | (e & lowmask);
  };
  constexpr uint32_t per16 = 16 / sizeof(C2);  // elements per 16-byte copy
  const uint32_t units = n_el / per16;
  const RegPassHdr* hdrs = reinterpret_cast<const RegPassHdr*>(blob);
  const RegGate* gates = reinterpret_cast<const RegGate*>(blob + sizeof(RegPassHdr) * geo.num_gates);

  auto issue = [&](uint64_t t, C2* dst) {
    const uint64_t base = insert_zeros(t, tile_bits, L);
    for (uint32_t u = tid; u < units; u += blockDim.x) {
      const uint32_t e = u * per16;
      cp_async16(smem_u32(dst + reg_swz(e)), psi + phys(base, e));
    }
  };

  uint64_t t = blockIdx.x;
  int cur = 0;
  if (t < geo.num_tiles) issue(t, buf0);
  cp_async_commit();
  for (; t < geo.num_tiles; t += gridDim.x) {
    const uint64_t next = t + gridDim.x;
    if (next < geo.num_tiles) issue(next, buf0 + (cur ^ 1) * n_el);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    C2* tile = buf0 + cur * n_el;
    const uint64_t base = insert_zeros(t, tile_bits, L);
    for (int p = 0; p < geo.num_gates; ++p) run_register_pass<T>(tile, hdrs[p], gates, blob, L, base);
    for (uint32_t u = tid; u < units; u += blockDim.x) {
      const uint32_t e = u * per16;
      *reinterpret_cast<uint4*>(psi + phys(base, e)) = *reinterpret_cast<const uint4*>(tile + reg_swz(e));
    }
    __syncthreads();
    cur ^= 1;
  }
  cp_async_wait0();
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side: lowering a stage to register passes.

namespace {

struct RegOp {
  bool dense = false;
  std::vector<int> tgt;                      // dense: tile bits; diagonal: encoded as RegGate::tgt (before registers)
  std::vector<int> dtgt_local;               // diagonal: tile bit of target i, or -1
  std::vector<int> dtgt_global;              // diagonal: physical bit of target i, or -1
  uint32_t local_ctl_mask = 0, local_ctl_val = 0;
  uint64_t gcm = 0, gcv = 0;
  uint32_t qmask = 0;                        // tile bits touched (dependencies)
  std::vector<C> entries;                    // dense matrix (row-major) or diagonal entries
};

bool is_pm_one(const C& c) { return c.im == 0.0 && (c.re == 1.0 || c.re == -1.0); }

template <typename V>
size_t put(std::vector<uint8_t>& blob, const V* p, size_t n) {
  blob.resize((blob.size() + 15) & ~size_t(15), 0);
  const size_t off = blob.size();
  blob.resize(off + n * sizeof(V));
  std::memcpy(blob.data() + off, p, n * sizeof(V));
  return off;
}

size_t put_complex(std::vector<uint8_t>& blob, const std::vector<C>& v, int bits) {
  if (bits == 32) {
    std::vector<float> f;
    for (const C& c : v) {
      f.push_back(float(c.re));
      f.push_back(float(c.im));
    }
    return put(blob, f.data(), f.size());
  }
  std::vector<double> d;
  for (const C& c : v) {
    d.push_back(c.re);
    d.push_back(c.im);
  }
  return put(blob, d.data(), d.size());
}

}  // namespace

bool register_pass_ok(const Target& s, const PlannedPass& p) {
  if (!p.staged || p.tile_bits.size() < 5 || p.tile_bits.size() > 14) return false;
  for (const HOp& op : p.ops) {
    if (op.diagonal) {
      if (op.targets.size() + op.controls.size() > QVDG_MAX_DIAGONAL_QUBITS) return false;
    } else if (op.targets.size() > 2) {
      return false;
    }
  }
  (void)s;
  return true;
}

LoweredPass lower_register_pass(const Target& s, const PlannedPass& p, const StageConfig& cfg, StageUpload& up) {
  LoweredPass lp;
  lp.staged = true;
  TileGeom& geo = lp.geo;
  const int L = int(p.tile_bits.size());
  geo.L = L;
  geo.B = int(cfg.low_bits);
  geo.num_tiles = uint64_t(1) << (s.n - uint32_t(L));
  geo.tensor = 2;
  for (size_t j = 0; j < p.tile_bits.size(); ++j) geo.tile_bits[j] = uint8_t(p.tile_bits[j]);
  std::vector<int> local(s.n, -1);
  for (size_t j = 0; j < p.tile_bits.size(); ++j) local[p.tile_bits[j]] = int(j);

  // Ops on tile bits. A controlled diagonal becomes a diagonal on its
  // controls and targets.
  std::vector<RegOp> ops;
  for (const HOp& op : p.ops) {
    RegOp r;
    if (op.diagonal) {
      std::vector<uint32_t> qs;
      HMatrix full;
      op.full(qs, full);  // qs = controls then targets
      r.entries = full.diagonal_entries();
      for (uint32_t q : qs) {
        const uint32_t ph = s.layout[q];
        r.dtgt_local.push_back(local[ph]);
        r.dtgt_global.push_back(local[ph] >= 0 ? -1 : int(ph));
        if (local[ph] >= 0) r.qmask |= 1u << local[ph];
      }
    } else {
      r.dense = true;
      for (uint32_t q : op.targets) {
        const int l = local[s.layout[q]];
        if (l < 0) throw Error(QVDG_ERR_INVALID, "internal: dense stage gate with a global target");
        r.tgt.push_back(l);
        r.qmask |= 1u << l;
      }
      for (auto& c : op.controls) {
        const uint32_t ph = s.layout[c.first];
        if (local[ph] >= 0) {
          r.local_ctl_mask |= 1u << local[ph];
          if (c.second) r.local_ctl_val |= 1u << local[ph];
          r.qmask |= 1u << local[ph];
        } else {
          r.gcm |= uint64_t(1) << ph;
          if (c.second) r.gcv |= uint64_t(1) << ph;
        }
      }
      r.entries = op.matrix.a;
    }
    ops.push_back(std::move(r));
  }

  // Register passes: one scan in program order takes every op that commutes
  // with all ops skipped before it and, if dense, whose targets fit in the
  // pass's four register bits (grown from the first dense ops).
  struct Pass {
    uint32_t gmask = 0;
    std::vector<size_t> ops;
  };
  std::vector<Pass> passes;
  std::vector<bool> done(ops.size(), false);
  size_t remaining = ops.size();
  while (remaining > 0) {
    Pass ps;
    uint32_t block_dense = 0, block_any = 0;
    for (size_t i = 0; i < ops.size(); ++i) {
      if (done[i]) continue;
      const RegOp& r = ops[i];
      if (r.dense) {
        uint32_t want = ps.gmask;
        for (int b : r.tgt) want |= 1u << b;
        if ((r.qmask & block_any) == 0 && __builtin_popcount(want) <= 4) {
          ps.gmask = want;
          ps.ops.push_back(i);
        } else {
          block_any |= r.qmask;
          block_dense |= r.qmask;
        }
      } else if ((r.qmask & block_dense) == 0) {
        ps.ops.push_back(i);
      } else {
        block_any |= r.qmask;
      }
    }
    for (size_t i : ps.ops) done[i] = true;
    remaining -= ps.ops.size();
    // Fill the register bits up to four with the lowest free tile bits.
    for (int b = 0; b < L && __builtin_popcount(ps.gmask) < 4; ++b) ps.gmask |= 1u << b;
    passes.push_back(std::move(ps));
  }

  // The pass blob: headers, gates, data.
  std::vector<uint8_t> blob(sizeof(RegPassHdr) * passes.size(), 0);
  std::vector<RegGate> gates;
  std::vector<uint8_t> data;  // appended after the gates; offsets fixed up below
  struct Fix {
    size_t gate;
    size_t data_off, table_off;
    bool has_table;
  };
  std::vector<Fix> fixes;
  for (size_t pi = 0; pi < passes.size(); ++pi) {
    const Pass& ps = passes[pi];
    RegPassHdr h{};
    int reg_of[64];
    std::fill(reg_of, reg_of + 64, -1);
    int gi = 0;
    for (int b = 0; b < L; ++b)
      if ((ps.gmask >> b) & 1u) {
        h.g[gi] = uint8_t(b);
        reg_of[b] = gi++;
      }
    h.pair = h.g[0] == 0 ? 1 : 0;
    for (uint32_t j = 0; j < 16; ++j) {
      uint32_t o = 0;
      for (int i = 0; i < 4; ++i)
        if ((j >> i) & 1u) o |= 1u << h.g[i];
      h.off[j] = uint16_t(o);
    }
    h.first_gate = uint32_t(gates.size());
    h.num_gates = uint16_t(ps.ops.size());
    std::memcpy(blob.data() + pi * sizeof(RegPassHdr), &h, sizeof(h));
    for (size_t oi : ps.ops) {
      const RegOp& r = ops[oi];
      RegGate g{};
      Fix fx{gates.size(), 0, 0, false};
      g.gcm = r.gcm;
      g.gcv = r.gcv;
      if (r.dense) {
        g.kind = r.tgt.size() == 1 ? kRegDense1 : kRegDense2;
        // Register controls become the mask of active bases, outside ones a predicate.
        uint32_t rcm = 0, rcv = 0;
        for (int b = 0; b < L; ++b) {
          if (!((r.local_ctl_mask >> b) & 1u)) continue;
          const bool v = (r.local_ctl_val >> b) & 1u;
          if (reg_of[b] >= 0) {
            rcm |= 1u << reg_of[b];
            if (v) rcv |= 1u << reg_of[b];
          } else {
            g.lcm |= 1u << b;
            if (v) g.lcv |= 1u << b;
          }
        }
        std::vector<C> m = r.entries;
        int t0 = reg_of[r.tgt[0]], t1 = r.tgt.size() > 1 ? reg_of[r.tgt[1]] : -1;
        if (t1 >= 0 && t1 < t0) {
          // Swap matrix bits 0 and 1 so that t0 < t1.
          std::vector<C> w(16);
          auto sw = [](int x) { return ((x & 1) << 1) | ((x >> 1) & 1); };
          for (int rr = 0; rr < 4; ++rr)
            for (int cc = 0; cc < 4; ++cc) w[sw(rr) * 4 + sw(cc)] = m[rr * 4 + cc];
          m = w;
          std::swap(t0, t1);
        }
        g.t0 = uint8_t(t0);
        g.t1 = uint8_t(t1 < 0 ? 0 : t1);
        const uint32_t tmask = (1u << t0) | (t1 >= 0 ? 1u << t1 : 0u);
        uint32_t pm = 0;
        for (uint32_t j = 0; j < 16; ++j)
          if (!(j & tmask) && (j & rcm) == rcv) pm |= 1u << j;
        g.pmask = rcm == 0 ? uint16_t(0xffffu) : uint16_t(pm);  // 0xffff: no register controls
        if (g.kind == kRegDense1) {
          const bool real = m[0].im == 0 && m[1].im == 0 && m[2].im == 0 && m[3].im == 0;
          const bool rx = m[0].im == 0 && m[3].im == 0 && m[1].re == 0 && m[2].re == 0;
          const bool diag_real = m[0].im == 0 && m[3].im == 0;
          g.spec = real ? kSpecReal : (rx ? kSpecRx : (diag_real ? kSpecDiagReal : kSpecGeneral));
        }
        fx.data_off = put_complex(data, m, s.bits);
      } else {
        const size_t k = r.dtgt_local.size();
        g.k = uint8_t(k);
        uint32_t reg_idx_mask = 0;
        for (size_t i = 0; i < k; ++i) {
          if (r.dtgt_local[i] >= 0) {
            const int b = r.dtgt_local[i];
            if (reg_of[b] >= 0) {
              g.tgt[i] = uint8_t(0x40 | reg_of[b]);
              reg_idx_mask |= 1u << i;
            } else {
              g.tgt[i] = uint8_t(b);
            }
          } else {
            g.tgt[i] = uint8_t(0x80 | r.dtgt_global[i]);
          }
        }
        // Register part of the diagonal index for each register j.
        uint16_t ridx[16];
        for (uint32_t j = 0; j < 16; ++j) {
          uint32_t idx = 0;
          for (size_t i = 0; i < k; ++i)
            if ((reg_idx_mask >> i) & 1u)
              if ((j >> (g.tgt[i] & 0x3f)) & 1u) idx |= 1u << i;
          ridx[j] = uint16_t(idx);
        }
        const bool sign = k <= 4 && std::all_of(r.entries.begin(), r.entries.end(), is_pm_one);
        if (sign) {
          g.kind = kRegSign;
          if (k <= 2 && s.n <= 48) {
            // Index bits from two shifts of (tile base | subcube base << 48);
            // register bits read bit 63, which is always 0.
            auto where = [&](size_t i) -> uint8_t {
              if (i >= k || (g.tgt[i] & 0x40)) return 63;
              if (g.tgt[i] & 0x80) return uint8_t(g.tgt[i] & 0x7f);
              return uint8_t(48 + g.tgt[i]);
            };
            g.kind = kRegSign2;
            g.t0 = where(0);
            g.t1 = where(1);
          }
          // For each value of the non-register index bits: the registers to negate.
          std::vector<uint16_t> masks(size_t(1) << k, 0);
          for (uint32_t f = 0; f < (1u << k); ++f) {
            if (f & reg_idx_mask) continue;
            uint16_t mk = 0;
            for (uint32_t j = 0; j < 16; ++j)
              if (r.entries[f | ridx[j]].re < 0) mk |= uint16_t(1u << j);
            masks[f] = mk;
          }
          fx.data_off = put(data, masks.data(), masks.size());
        } else {
          g.kind = kRegPhase;
          fx.data_off = put_complex(data, r.entries, s.bits);
          fx.table_off = put(data, ridx, 16);
          fx.has_table = true;
        }
      }
      g.pred = (g.gcm != 0 || g.lcm != 0) ? 1 : 0;
      if (g.kind == kRegDense1)
        g.op = g.pmask == 0xffffu ? uint16_t(kOpDense1 + 4 * g.spec + g.t0) : uint16_t(kOpDense1Masked);
      else if (g.kind == kRegDense2)
        g.op = g.pmask == 0xffffu ? uint16_t(kOpDense2 + (g.t0 == 0 ? g.t1 - 1 : (g.t0 == 1 ? g.t1 + 1 : 5)))
                                  : uint16_t(kOpDense2Masked);
      else if (g.kind == kRegSign2)
        g.op = kOpSign2;
      else if (g.kind == kRegSign)
        g.op = kOpSign;
      else
        g.op = kOpPhase;
      gates.push_back(g);
      fixes.push_back(fx);
    }
  }
  const size_t gates_off = blob.size();  // a multiple of 48, so of 16
  const size_t data_base = gates_off + gates.size() * sizeof(RegGate);
  for (const Fix& fx : fixes) {
    gates[fx.gate].data = uint32_t(data_base + fx.data_off);
    if (fx.has_table) gates[fx.gate].table = uint32_t(data_base + fx.table_off);
  }
  blob.resize(data_base);
  std::memcpy(blob.data() + gates_off, gates.data(), gates.size() * sizeof(RegGate));
  blob.insert(blob.end(), data.begin(), data.end());
  blob.resize((blob.size() + 15) & ~size_t(15), 0);
  if (blob.size() > kRegBlobBudget) throw Error(QVDG_ERR_UNSUPPORTED, "internal: register stage program too large");

  up.tc.resize((up.tc.size() + 15) & ~size_t(15), 0);
  geo.tc_offset = up.tc.size();
  geo.tc_bytes = uint32_t(blob.size());
  geo.num_gates = int(passes.size());
  up.tc.insert(up.tc.end(), blob.begin(), blob.end());
  lp.gate_offset = up.gates.size();
  return lp;
}

size_t register_blob_budget() { return kRegBlobBudget; }

void launch_stage_reg(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  const size_t tile_bytes = (s.bits == 32 ? 8 : 16) << lp.geo.L;
  const size_t smem = 2 * tile_bytes + lp.geo.tc_bytes;
  // One thread per register subcube, at least one full warp (the set-up
  // loops are strided, so any count works).
  const int cap = s.bits == 32 ? reg_threads<float>() : reg_threads<double>();
  const int threads = std::max(32, std::min(cap, 1 << (lp.geo.L - 4)));
  const uint64_t grid = std::min<uint64_t>(lp.geo.num_tiles, uint64_t(s.sms));
  if (s.bits == 32) {
    static size_t configured = 0;
    if (smem > configured) {
      QVDG_CUDA(cudaFuncSetAttribute(k_stage_reg<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      configured = smem;
    }
    k_stage_reg<float><<<unsigned(grid), threads, smem, s.stream>>>(static_cast<float2*>(s.amp), lp.geo, dev.tc);
  } else {
    static size_t configured = 0;
    if (smem > configured) {
      QVDG_CUDA(cudaFuncSetAttribute(k_stage_reg<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      configured = smem;
    }
    k_stage_reg<double><<<unsigned(grid), threads, smem, s.stream>>>(static_cast<double2*>(s.amp), lp.geo, dev.tc);
  }
  QVDG_LAUNCH_CHECK();
}

}  // namespace qvdg
