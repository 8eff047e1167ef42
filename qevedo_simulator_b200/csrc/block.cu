// Plain passes that apply a fused group gate by gate: one pass over the
// state per fused group (the reference's one sweep per fused op,
// src/simulator.rs:136-143), but instead of the group's 2^K x 2^K product
// matrix (4^K complex multiply-adds per 2^K amplitudes) each thread applies
// the group's member gates to its 2^K amplitudes in registers: a 1-qubit
// gate costs 4-8 FMAs per amplitude, runs of diagonal gates are merged on
// the host into one phase vector (or, when every entry is +-1, one mask of
// sign flips). For the 5- and 6-qubit groups of layered circuits this is a
// fraction of the dense product's arithmetic, so wide groups stay
// memory-bound and fewer passes are needed.
//
// Eligible groups: complex64 or complex128, K = 4 or 5 qubits, every dense
// member with one target (controls anywhere in the group), and at most two
// targets among index bits 0-3 (wider low runs would make a warp's loads
// stride); other groups use the dense fused kernel.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "program.hpp"
#include "stage_kernel.hpp"

namespace qvdg {

namespace {

enum : uint8_t { kBlk1 = 0, kBlkSign = 1, kBlkPhase = 2 };
enum : uint8_t { kBSpecGeneral = 0, kBSpecReal = 1, kBSpecRx = 2, kBSpecDiagReal = 3 };
constexpr int kBlockThreads = 256;
constexpr int kBlockMaxOps = 1024;

struct BlockOp {
  uint8_t kind;
  uint8_t bit;        // 1-qubit gate: register bit of the target
  uint8_t spec;       // 1-qubit gate: matrix form
  uint8_t masked;     // 1-qubit gate: 1 when some pairs are inactive (controls)
  uint32_t data;      // byte offset of the matrix / phase vector in the program
  uint64_t mask;      // 1-qubit: active pair bases j (target bit clear); sign: registers to negate
};
static_assert(sizeof(BlockOp) == 16, "block op layout");

// ---------------------------------------------------------------------------
// Device side.

template <typename T, int SPEC>
__device__ __forceinline__ cplx_t<T> brow(cplx_t<T> m0, cplx_t<T> m1, cplx_t<T> x0, cplx_t<T> x1) {
  if (SPEC == kBSpecReal) return make_c<T>(fma(m0.x, x0.x, m1.x * x1.x), fma(m0.x, x0.y, m1.x * x1.y));
  if (SPEC == kBSpecRx) return make_c<T>(fma(m0.x, x0.x, -m1.y * x1.y), fma(m0.x, x0.y, m1.y * x1.x));
  if (SPEC == kBSpecDiagReal)
    return make_c<T>(fma(m0.x, x0.x, fma(m1.x, x1.x, -m1.y * x1.y)), fma(m0.x, x0.y, fma(m1.x, x1.y, m1.y * x1.x)));
  return make_c<T>(fma(m0.x, x0.x, fma(-m0.y, x0.y, fma(m1.x, x1.x, -m1.y * x1.y))),
                   fma(m0.x, x0.y, fma(m0.y, x0.x, fma(m1.x, x1.y, m1.y * x1.x))));
}
template <typename T, int SPEC>
__device__ __forceinline__ cplx_t<T> brow2(cplx_t<T> m0, cplx_t<T> m1, cplx_t<T> x0, cplx_t<T> x1) {
  if (SPEC == kBSpecRx) return make_c<T>(fma(m1.x, x1.x, -m0.y * x0.y), fma(m1.x, x1.y, m0.y * x0.x));
  if (SPEC == kBSpecDiagReal)
    return make_c<T>(fma(m1.x, x1.x, fma(m0.x, x0.x, -m0.y * x0.y)), fma(m1.x, x1.y, fma(m0.x, x0.y, m0.y * x0.x)));
  return brow<T, SPEC>(m0, m1, x0, x1);
}

template <typename T, int S, int TB, int SPEC, bool MASKED>
__device__ __forceinline__ void b1(cplx_t<T> (&a)[S], const cplx_t<T>* m, uint64_t mask) {
  const cplx_t<T> m00 = m[0], m01 = m[1], m10 = m[2], m11 = m[3];
#pragma unroll
  for (int j = 0; j < S; ++j) {
    if (j & (1 << TB)) continue;
    const cplx_t<T> x0 = a[j], x1 = a[j | (1 << TB)];
    const cplx_t<T> y0 = brow<T, SPEC>(m00, m01, x0, x1);
    const cplx_t<T> y1 = brow2<T, SPEC>(m10, m11, x0, x1);
    if (MASKED) {
      const bool on = (mask >> j) & 1u;
      a[j] = on ? y0 : x0;
      a[j | (1 << TB)] = on ? y1 : x1;
    } else {
      a[j] = y0;
      a[j | (1 << TB)] = y1;
    }
  }
}

template <typename T, int S, int SPEC, bool MASKED>
__device__ __forceinline__ void b1_bit(cplx_t<T> (&a)[S], int bit, const cplx_t<T>* m, uint64_t mask) {
  switch (bit) {
    case 0: b1<T, S, 0, SPEC, MASKED>(a, m, mask); break;
    case 1: b1<T, S, 1, SPEC, MASKED>(a, m, mask); break;
    case 2: b1<T, S, 2, SPEC, MASKED>(a, m, mask); break;
    case 3: b1<T, S, 3, SPEC, MASKED>(a, m, mask); break;
    default:
      if constexpr (S > 16) b1<T, S, 4, SPEC, MASKED>(a, m, mask);
      break;
  }
}

__device__ __forceinline__ void bflip(float2& x, uint32_t t) {
  const uint32_t s = t & 0x80000000u;
  x.x = __uint_as_float(__float_as_uint(x.x) ^ s);
  x.y = __uint_as_float(__float_as_uint(x.y) ^ s);
}
__device__ __forceinline__ void bflip(double2& x, uint32_t t) {
  const unsigned long long s = (unsigned long long)(t & 0x80000000u) << 32;
  x.x = __longlong_as_double(__double_as_longlong(x.x) ^ s);
  x.y = __longlong_as_double(__double_as_longlong(x.y) ^ s);
}

template <typename T, int K>
__global__ void __launch_bounds__(kBlockThreads) k_block(cplx_t<T>* __restrict__ psi, const uint64_t n_groups,
                                                         const TileGeom geo, const unsigned char* __restrict__ blob_all) {
  using C2 = cplx_t<T>;
  constexpr int S = 1 << K;
  extern __shared__ __align__(16) unsigned char prog[];
  __shared__ uint8_t fixed[8];
  __shared__ uint64_t off[S];
  {
    const uint4* src = reinterpret_cast<const uint4*>(blob_all + geo.tc_offset);
    uint4* dst = reinterpret_cast<uint4*>(prog);
    for (uint32_t i = threadIdx.x; i < geo.tc_bytes / 16; i += blockDim.x) dst[i] = src[i];
  }
  if (threadIdx.x < K) fixed[threadIdx.x] = geo.tile_bits[threadIdx.x];
  if (threadIdx.x < S) {
    uint64_t o = 0;
    for (int i = 0; i < K; ++i)
      if ((threadIdx.x >> i) & 1) o |= uint64_t(1) << geo.tile_bits[i];
    off[threadIdx.x] = o;
  }
  __syncthreads();
  const BlockOp* ops = reinterpret_cast<const BlockOp*>(prog);
  const int nops = geo.num_gates;
  const bool pairs = sizeof(C2) == 8 && fixed[0] == 0;  // registers j, j^1 adjacent: 16-byte accesses
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t it = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; it < n_groups; it += stride) {
    const uint64_t base = insert_zeros(it, fixed, K);
    C2 a[S];
    if (pairs) {
#pragma unroll
      for (int j = 0; j < S; j += 2) {
        const float4 v = *reinterpret_cast<const float4*>(psi + base + off[j]);
        a[j] = make_c<T>(T(v.x), T(v.y));
        a[j + 1] = make_c<T>(T(v.z), T(v.w));
      }
    } else {
#pragma unroll
      for (int j = 0; j < S; ++j) a[j] = psi[base + off[j]];
    }
    for (int i = 0; i < nops; ++i) {
      const BlockOp op = ops[i];
      const C2* m = reinterpret_cast<const C2*>(prog + op.data);
      if (op.kind == kBlk1) {
        if (op.masked) {
          b1_bit<T, S, kBSpecGeneral, true>(a, op.bit, m, op.mask);
        } else {
          switch (op.spec) {
            case kBSpecReal: b1_bit<T, S, kBSpecReal, false>(a, op.bit, m, 0); break;
            case kBSpecRx: b1_bit<T, S, kBSpecRx, false>(a, op.bit, m, 0); break;
            case kBSpecDiagReal: b1_bit<T, S, kBSpecDiagReal, false>(a, op.bit, m, 0); break;
            default: b1_bit<T, S, kBSpecGeneral, false>(a, op.bit, m, 0); break;
          }
        }
      } else if (op.kind == kBlkSign) {
        const uint32_t lo = uint32_t(op.mask), hi = uint32_t(op.mask >> 32);
#pragma unroll
        for (int j = 0; j < S; ++j) bflip(a[j], (j < 32 ? lo << (31 - j) : hi << (63 - j)));
      } else {
#pragma unroll
        for (int j = 0; j < S; ++j) {
          const C2 p = m[j];
          a[j] = make_c<T>(fma(p.x, a[j].x, -p.y * a[j].y), fma(p.x, a[j].y, p.y * a[j].x));
        }
      }
    }
    if (pairs) {
#pragma unroll
      for (int j = 0; j < S; j += 2)
        *reinterpret_cast<float4*>(psi + base + off[j]) =
            make_float4(float(a[j].x), float(a[j].y), float(a[j + 1].x), float(a[j + 1].y));
    } else {
#pragma unroll
      for (int j = 0; j < S; ++j) psi[base + off[j]] = a[j];
    }
  }
}

// ---------------------------------------------------------------------------
// Host side.

template <typename V>
size_t bput(std::vector<uint8_t>& blob, const V* p, size_t n) {
  blob.resize((blob.size() + 15) & ~size_t(15), 0);
  const size_t o = blob.size();
  blob.resize(o + n * sizeof(V));
  std::memcpy(blob.data() + o, p, n * sizeof(V));
  return o;
}

size_t bput_complex(std::vector<uint8_t>& blob, const std::vector<C>& v, int bits) {
  if (bits == 32) {
    std::vector<float> f;
    for (const C& c : v) {
      f.push_back(float(c.re));
      f.push_back(float(c.im));
    }
    return bput(blob, f.data(), f.size());
  }
  std::vector<double> d;
  for (const C& c : v) {
    d.push_back(c.re);
    d.push_back(c.im);
  }
  return bput(blob, d.data(), d.size());
}

C cmul_h(const C& a, const C& b) { return C{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

}  // namespace

bool block_pass_ok(const Target& t, const std::vector<HOp>& members, const std::vector<uint32_t>& qubits) {
  const size_t k = qubits.size();
  if (k < 4 || k > 5 || members.size() < 2) return false;
  int low = 0;
  for (uint32_t q : qubits)
    if (t.layout[q] < 4) ++low;
  if (low > 2) return false;
  for (const HOp& op : members)
    if (!op.diagonal && op.targets.size() != 1) return false;
  return true;
}

LoweredPass lower_block_pass(const Target& t, const PlannedPass& p, StageUpload& up) {
  LoweredPass lp;
  lp.staged = false;
  lp.block = true;
  TileGeom& geo = lp.geo;
  std::vector<uint32_t> phys;
  for (uint32_t q : p.block_qubits) phys.push_back(t.layout[q]);
  std::sort(phys.begin(), phys.end());
  const int K = int(phys.size());
  const uint32_t S = 1u << K;
  geo.L = K;
  for (int i = 0; i < K; ++i) geo.tile_bits[i] = uint8_t(phys[size_t(i)]);
  auto reg_of = [&](uint32_t logical) {
    return int(std::find(phys.begin(), phys.end(), t.layout[logical]) - phys.begin());
  };
  std::vector<BlockOp> ops;
  std::vector<uint8_t> data;
  struct Fix {
    size_t op, off;
  };
  std::vector<Fix> fixes;
  std::vector<C> phase;  // pending merged diagonal over the registers
  auto flush_phase = [&]() {
    if (phase.empty()) return;
    bool sign = true;
    for (const C& c : phase) sign = sign && c.im == 0.0 && (c.re == 1.0 || c.re == -1.0);
    BlockOp o{};
    if (sign) {
      o.kind = kBlkSign;
      for (uint32_t j = 0; j < S; ++j)
        if (phase[j].re < 0) o.mask |= uint64_t(1) << j;
      ops.push_back(o);
    } else {
      o.kind = kBlkPhase;
      fixes.push_back({ops.size(), bput_complex(data, phase, t.bits)});
      ops.push_back(o);
    }
    phase.clear();
  };
  for (const HOp& op : p.ops) {
    if (op.diagonal) {
      std::vector<uint32_t> qs;
      HMatrix full;
      op.full(qs, full);
      const std::vector<C> d = full.diagonal_entries();
      if (phase.empty()) phase.assign(S, C{1.0, 0.0});
      for (uint32_t j = 0; j < S; ++j) {
        uint32_t idx = 0;
        for (size_t i = 0; i < qs.size(); ++i)
          if ((j >> reg_of(qs[i])) & 1u) idx |= 1u << i;
        phase[j] = cmul_h(phase[j], d[idx]);
      }
      continue;
    }
    flush_phase();
    BlockOp o{};
    o.kind = kBlk1;
    o.bit = uint8_t(reg_of(op.targets[0]));
    uint32_t cm = 0, cv = 0;
    for (auto& c : op.controls) {
      cm |= 1u << reg_of(c.first);
      if (c.second) cv |= 1u << reg_of(c.first);
    }
    for (uint32_t j = 0; j < S; ++j)
      if (!((j >> o.bit) & 1u) && (j & cm) == cv) o.mask |= uint64_t(1) << j;
    o.masked = cm != 0 ? 1 : 0;
    const std::vector<C>& m = op.matrix.a;
    const bool real = m[0].im == 0 && m[1].im == 0 && m[2].im == 0 && m[3].im == 0;
    const bool rx = m[0].im == 0 && m[3].im == 0 && m[1].re == 0 && m[2].re == 0;
    const bool dreal = m[0].im == 0 && m[3].im == 0;
    o.spec = real ? kBSpecReal : (rx ? kBSpecRx : (dreal ? kBSpecDiagReal : kBSpecGeneral));
    fixes.push_back({ops.size(), bput_complex(data, m, t.bits)});
    ops.push_back(o);
  }
  flush_phase();
  if (ops.size() > size_t(kBlockMaxOps)) throw Error(QVDG_ERR_UNSUPPORTED, "internal: block program too long");
  const size_t data_base = (ops.size() * sizeof(BlockOp) + 15) & ~size_t(15);
  for (const Fix& f : fixes) ops[f.op].data = uint32_t(data_base + f.off);
  std::vector<uint8_t> blob(data_base, 0);
  std::memcpy(blob.data(), ops.data(), ops.size() * sizeof(BlockOp));
  blob.insert(blob.end(), data.begin(), data.end());
  blob.resize((blob.size() + 15) & ~size_t(15), 0);
  up.tc.resize((up.tc.size() + 15) & ~size_t(15), 0);
  geo.tc_offset = up.tc.size();
  geo.tc_bytes = uint32_t(blob.size());
  geo.num_gates = int(ops.size());
  geo.num_tiles = uint64_t(1) << (t.n - uint32_t(K));  // groups
  up.tc.insert(up.tc.end(), blob.begin(), blob.end());
  return lp;
}

void launch_block(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  const size_t smem = lp.geo.tc_bytes;
  const uint64_t groups = lp.geo.num_tiles;
  const unsigned grid = unsigned(std::max<uint64_t>(
      1, std::min<uint64_t>((groups + kBlockThreads - 1) / kBlockThreads, uint64_t(s.sms) * 8)));
  auto go = [&](auto kernel, auto* psi) {
    if (smem > 48 * 1024)
      QVDG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    kernel<<<grid, kBlockThreads, smem, s.stream>>>(psi, groups, lp.geo, dev.tc);
  };
  if (s.bits == 32) {
    auto* psi = static_cast<float2*>(s.amp);
    if (lp.geo.L == 4)
      go(k_block<float, 4>, psi);
    else
      go(k_block<float, 5>, psi);
  } else {
    auto* psi = static_cast<double2*>(s.amp);
    if (lp.geo.L == 4)
      go(k_block<double, 4>, psi);
    else
      go(k_block<double, 5>, psi);
  }
  QVDG_LAUNCH_CHECK();
}

}  // namespace qvdg
