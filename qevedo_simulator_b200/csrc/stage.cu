// Staged tile kernel: a CTA loads a tile of 2^L amplitudes (the low B
// physical bits plus L - B chosen bits) into shared memory with 16-byte
// coalesced loads, applies the stage's whole gate program in place, and
// stores it back. CTAs are persistent over tiles. The tile is the GPU form of
// the reference's region (src/blocking.rs:228-302): one pass over HBM per
// stage instead of one per gate.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "program.hpp"
#include "dense_tc.hpp"
#include "stage.hpp"
#include "stage_kernel.hpp"
#include "tile_ops.cuh"

namespace qvdg {

namespace {

constexpr int kStageThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kStageThreads) k_stage(cplx_t<T>* __restrict__ psi, const TileGeom geo,
                                                         const TileGate* __restrict__ gates,
                                                         const cplx_t<T>* __restrict__ mats) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint8_t tile_bits[48];
  if (threadIdx.x < 48) tile_bits[threadIdx.x] = geo.tile_bits[threadIdx.x];
  __syncthreads();  // every thread reads tile_bits below
  const int L = geo.L, B = geo.B;
  cplx_t<T>* tile = reinterpret_cast<cplx_t<T>*>(smem);
  uint64_t* hi = reinterpret_cast<uint64_t*>(smem + (sizeof(cplx_t<T>) << L));
  const int nhi = 1 << (L - B);
  for (int r = threadIdx.x; r < nhi; r += blockDim.x) {
    uint64_t a = 0;
    for (int j = 0; j < L - B; ++j)
      if ((r >> j) & 1) a |= uint64_t(1) << tile_bits[B + j];
    hi[r] = a;
  }
  __syncthreads();
  const uint32_t n_el = 1u << L;
  const uint32_t lowmask = (1u << B) - 1u;
  // 16-byte accesses: two complex64 per access when runs have >= 2 amplitudes.
  const bool pairs = sizeof(T) == 4 && B >= 1;
  for (uint64_t t = blockIdx.x; t < geo.num_tiles; t += gridDim.x) {
    const uint64_t base = insert_zeros(t, tile_bits, L);
    if (pairs) {
      for (uint32_t e = threadIdx.x * 2; e < n_el; e += blockDim.x * 2) {
        const uint64_t a = base | hi[e >> B] | (e & lowmask);
        *reinterpret_cast<float4*>(&tile[e]) = *reinterpret_cast<const float4*>(&psi[a]);
      }
    } else {
      for (uint32_t e = threadIdx.x; e < n_el; e += blockDim.x) tile[e] = psi[base | hi[e >> B] | (e & lowmask)];
    }
    __syncthreads();
    for (int gi = 0; gi < geo.num_gates; ++gi) {
      const TileGate& g = gates[gi];
      if ((base & g.gcm) != g.gcv) continue;  // global controls: same for the whole tile
      const cplx_t<T>* m = mats + g.mat;
      if (g.kind == 1) {
        tile_diag<T>(tile, L, g, m, base);
      } else {
        switch (g.k) {
          case 1: tile_dense<T, 1>(tile, L, g, m); break;
          case 2: tile_dense<T, 2>(tile, L, g, m); break;
          case 3: tile_dense<T, 3>(tile, L, g, m); break;
          case 4: tile_dense<T, 4>(tile, L, g, m); break;
          case 5: tile_dense_rows<T, 5>(tile, L, g, m); break;
          default: tile_dense_rows<T, 6>(tile, L, g, m); break;
        }
      }
      __syncthreads();
    }
    if (pairs) {
      for (uint32_t e = threadIdx.x * 2; e < n_el; e += blockDim.x * 2) {
        const uint64_t a = base | hi[e >> B] | (e & lowmask);
        *reinterpret_cast<float4*>(&psi[a]) = *reinterpret_cast<const float4*>(&tile[e]);
      }
    } else {
      for (uint32_t e = threadIdx.x; e < n_el; e += blockDim.x) psi[base | hi[e >> B] | (e & lowmask)] = tile[e];
    }
    __syncthreads();
  }
}

template <typename T>
void stage_launch(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  const int L = lp.geo.L, B = lp.geo.B;
  const size_t smem = (sizeof(cplx_t<T>) << L) + (sizeof(uint64_t) << (L - B));
  static size_t configured = 0;
  if (smem > configured) {
    QVDG_CUDA(cudaFuncSetAttribute(k_stage<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    configured = smem;
  }
  const size_t per_sm = std::max<size_t>(1, std::min<size_t>(8, (220 * 1024) / smem));
  const uint64_t grid = std::min<uint64_t>(lp.geo.num_tiles, uint64_t(s.sms) * per_sm);
  k_stage<T><<<unsigned(grid), kStageThreads, smem, s.stream>>>(
      static_cast<cplx_t<T>*>(s.amp), lp.geo, dev.gates + lp.gate_offset, static_cast<const cplx_t<T>*>(dev.mats));
  QVDG_LAUNCH_CHECK();
}

}  // namespace

namespace {

uint16_t to_bf16(float f) {  // round to nearest even
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;
  return uint16_t((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

float from_bf16(uint16_t h) {
  const uint32_t u = uint32_t(h) << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// A gate as the real matrix B^T = [[Re M, -Im M], [Im M, Re M]] (row n =
// output component, column kk = input component), split into bf16 high and
// low parts, each in the canonical K-major core-matrix layout.
void append_tc_gate(const HMatrix& m, std::vector<uint8_t>& blob) {
  const size_t half = m.dim, kd = 2 * half;
  const size_t base = blob.size();
  blob.resize(base + 4 * kd * kd, 0);
  uint8_t* hi = blob.data() + base;
  uint8_t* lo = hi + 2 * kd * kd;
  auto split = [](double v, uint16_t& h, uint16_t& l) {
    h = to_bf16(float(v));
    l = to_bf16(float(v - double(from_bf16(h))));
  };
  auto put = [&](size_t n, size_t kk, uint16_t h, uint16_t l) {
    const size_t off = (n / 8) * (kd * 16) + (kk / 8) * 128 + (n % 8) * 16 + (kk % 8) * 2;
    std::memcpy(hi + off, &h, 2);
    std::memcpy(lo + off, &l, 2);
  };
  // Entry (r, c) of M fills one element of each quadrant.
  for (size_t r = 0; r < half; ++r)
    for (size_t c = 0; c < half; ++c) {
      const C e = m.at(r, c);
      uint16_t h, l;
      split(e.re, h, l);
      put(r, c, h, l);
      put(r + half, c + half, h, l);
      split(-e.im, h, l);
      put(r, c + half, h, l);
      split(e.im, h, l);
      put(r + half, c, h, l);
    }
}

}  // namespace

// Fold one-phase gates into the neighbouring tensor-core gathers (see
// lower_tensor_pass).
constexpr bool kAbsorbPhases = false;

// Spread the low bits of `x` over the set bits of `mask` (ascending).
uint32_t spread_bits(uint32_t x, uint32_t mask) {
  uint32_t out = 0;
  for (uint32_t bit = 0; mask; mask &= mask - 1, ++bit)
    if ((x >> bit) & 1) out |= mask & (~mask + 1);
  return out;
}

void blob_align(std::vector<uint8_t>& blob) { blob.resize((blob.size() + 15) & ~size_t(15), 0); }

template <class V>
size_t blob_put(std::vector<uint8_t>& blob, const std::vector<V>& v) {
  blob_align(blob);
  const size_t off = blob.size();
  blob.resize(off + v.size() * sizeof(V));
  std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(V));
  return off;
}

size_t blob_put_c64(std::vector<uint8_t>& blob, const std::vector<C>& v) {
  std::vector<float> f;
  for (const C& c : v) {
    f.push_back(float(c.re));
    f.push_back(float(c.im));
  }
  return blob_put(blob, f);
}

// Index tables of one gate in a tensor pass, as 32-bit byte offsets into
// the complex64 tile (element index * 8): the spread of an enumeration index
// over the tile bits not in `fixed` (64 low + 128 high entries), then the
// member offsets of the targets (64 entries), or the local part of a
// diagonal's index (128 + 64 entries, plain indices).
size_t blob_tables(std::vector<uint8_t>& blob, uint32_t L, uint32_t fixed_mask, const std::vector<int>& tgt_local,
                   bool diagonal) {
  const uint32_t free_mask = ((1u << L) - 1u) & ~fixed_mask;
  // Swizzled positions (tc_swz): XOR-linear, so the kernel combines
  // entries with XOR.
  std::vector<uint32_t> t(64 + 128, 0);
  for (uint32_t x = 0; x < 64; ++x) t[x] = tc_swz(spread_bits(x, free_mask)) * 8;
  for (uint32_t x = 0; x < 128; ++x) t[64 + x] = tc_swz(spread_bits(x << 6, free_mask)) * 8;
  if (!diagonal) {
    for (uint32_t c = 0; c < 64; ++c) {
      uint32_t o = 0;
      for (size_t j = 0; j < tgt_local.size(); ++j)
        if ((c >> j) & 1) o |= 1u << tgt_local[j];
      t.push_back(c < (1u << tgt_local.size()) ? tc_swz(o) * 8 : 0);
    }
  } else {
    for (uint32_t part = 0; part < 2; ++part)
      for (uint32_t x = 0; x < (part ? 64u : 128u); ++x) {
        const uint32_t e = part ? (x << 7) : x;
        uint32_t idx = 0;
        for (size_t j = 0; j < tgt_local.size(); ++j)
          if (tgt_local[j] >= 0 && ((e >> tgt_local[j]) & 1)) idx |= 1u << j;
        t.push_back(idx);
      }
  }
  return blob_put(blob, t);
}

// Lower a pass for the tensor-core kernel: every gate's data and tables go
// into the pass blob, which the kernel keeps in shared memory.
LoweredPass lower_tensor_pass(const Target& s, const PlannedPass& p, const StageConfig& cfg, StageUpload& up) {
  LoweredPass lp;
  TileGeom& geo = lp.geo;
  geo.L = int(p.tile_bits.size());
  geo.B = int(cfg.low_bits);
  geo.num_tiles = uint64_t(1) << (s.n - uint32_t(geo.L));
  for (size_t j = 0; j < p.tile_bits.size(); ++j) geo.tile_bits[j] = uint8_t(p.tile_bits[j]);
  std::vector<int> local(s.n, -1);
  for (size_t j = 0; j < p.tile_bits.size(); ++j) local[p.tile_bits[j]] = int(j);
  const uint32_t L = uint32_t(geo.L);
  lp.gate_offset = up.gates.size();
  blob_align(up.tc);
  geo.tc_offset = up.tc.size();
  std::vector<uint8_t> blob;
  for (const HOp& src : p.ops) {
    HOp op = src;
    TileGate g{};
    // Global controls are tile predicates; local controls of a dense gate
    // are folded into its matrix (the gate then acts on them too).
    std::vector<std::pair<uint32_t, bool>> local_controls;
    for (auto& c : op.controls) {
      const uint32_t ph = s.layout[c.first];
      if (local[ph] >= 0) {
        local_controls.push_back(c);
      } else {
        g.gcm |= uint64_t(1) << ph;
        if (c.second) g.gcv |= uint64_t(1) << ph;
      }
    }
    if (!op.diagonal && !local_controls.empty()) {
      size_t state = 0;
      std::vector<uint32_t> qs;
      for (size_t i = 0; i < local_controls.size(); ++i) {
        state |= size_t(local_controls[i].second) << i;
        qs.push_back(local_controls[i].first);
      }
      qs.insert(qs.end(), op.targets.begin(), op.targets.end());
      op.matrix = op.matrix.controlled(local_controls.size(), state);
      op.targets = qs;
      local_controls.clear();
    }
    uint32_t fixed = 0;
    for (auto& c : local_controls) {
      const int l = local[s.layout[c.first]];
      fixed |= 1u << l;
      if (c.second) g.lcv |= 1u << l;
    }
    const size_t k = op.targets.size();
    g.k = uint8_t(k);
    std::vector<int> tl;
    for (uint32_t q : op.targets) tl.push_back(local[s.layout[q]]);
    if (op.diagonal) {
      if (k > QVDG_MAX_DIAGONAL_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "diagonal gates on more than 10 qubits are not supported");
      const std::vector<C> d = op.matrix.diagonal_entries();
      size_t odd = 0, count = 0;
      for (size_t i = 0; i < d.size(); ++i)
        if (!(d[i].re == 1.0 && d[i].im == 0.0)) {
          odd = i;
          ++count;
        }
      for (size_t j = 0; j < k; ++j) g.tgt[j] = tl[j] >= 0 ? uint8_t(tl[j]) : uint8_t(0x80 | s.layout[op.targets[j]]);
      if (count <= 1) {
        // One phase on the elements whose targets read `odd` (CZ, CP, S, T, ...).
        g.kind = 3;
        for (size_t j = 0; j < k; ++j) {
          const bool one = (odd >> j) & 1;
          if (tl[j] >= 0) {
            fixed |= 1u << tl[j];
            if (one) g.lcv |= 1u << tl[j];
          } else {
            const uint32_t ph = s.layout[op.targets[j]];
            g.gcm |= uint64_t(1) << ph;
            if (one) g.gcv |= uint64_t(1) << ph;
          }
        }
        const C ph = count ? d[odd] : C{1.0, 0.0};
        g.absorb = (ph.re == -1.0 && ph.im == 0.0) ? 1 : 0;
        g.mat = uint32_t(blob_put_c64(blob, {ph}));
        g.tab = uint32_t(blob_tables(blob, L, fixed, {}, false));
      } else {
        g.kind = 1;
        g.mat = uint32_t(blob_put_c64(blob, d));
        g.tab = uint32_t(blob_tables(blob, L, fixed, tl, true));
      }
    } else {
      if (k > QVDG_MAX_GATE_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "dense gates on more than 6 qubits are not supported");
      for (size_t j = 0; j < k; ++j) {
        if (tl[j] < 0) throw Error(QVDG_ERR_INVALID, "internal: dense stage gate with a global target");
        g.tgt[j] = uint8_t(tl[j]);
        fixed |= 1u << tl[j];
      }
      if (k >= 3 && k + 7 <= L) {
        g.kind = 2;
        blob_align(blob);
        g.mat = uint32_t(blob.size());
        append_tc_gate(op.matrix, blob);
      } else {
        g.kind = 0;
        g.mat = uint32_t(blob_put_c64(blob, op.matrix.a));
      }
      g.tab = uint32_t(blob_tables(blob, L, fixed, tl, false));
    }
    g.nfixed = uint8_t(__builtin_popcount(fixed));
    g.lcm = fixed * 8;  // byte units, like the tables
    g.lcv *= 8;
    up.gates.push_back(g);
  }
  // Runs of one-phase gates right before a tensor-core gate can be applied
  // in that gate's gather, and a run at the end of the pass in the final
  // store (kAbsorbPhases). Measured on the 30-qubit grid circuit this was
  // neither faster nor slower than separate phase steps, so it is off.
  if (kAbsorbPhases) {
    // kind 3: absorb bit 0 = the phase is -1, bit 1 = applied by a consumer.
    const size_t first = lp.gate_offset, last = up.gates.size();
    size_t run = 0;
    auto mark = [&](size_t end) {
      for (size_t j = end - run; j < end; ++j) up.gates[j].absorb |= 2;
    };
    for (size_t i = first; i < last; ++i) {
      TileGate& g = up.gates[i];
      if (g.kind == 3) {
        ++run;
      } else if (g.kind == 2 && g.gcm == 0) {  // runs on every tile, so it can carry the run
        mark(i);
        g.absorb = uint8_t(run);
        run = 0;
      } else {
        run = 0;
      }
    }
    mark(last);
    lp.geo.tail_absorb = int(run);
  }
  blob_align(blob);
  up.tc.insert(up.tc.end(), blob.begin(), blob.end());
  geo.num_gates = int(up.gates.size() - lp.gate_offset);
  geo.tc_bytes = uint32_t(blob.size());
  geo.tensor = 1;
  if (geo.L - geo.B > 10 || geo.L > int(kTcTileBits) || geo.tc_bytes > kTcBlobBytes ||
      geo.num_gates > kTcMaxGates)
    throw Error(QVDG_ERR_INVALID, "internal: tensor-core pass does not fit shared memory");
  return lp;
}

// Whether the tensor-core kernel can run every gate of a pass: dense gates
// (with local controls folded in) have at most 2 qubits or fit the
// tensor-core shape (3 <= k <= L - 7).
bool tensor_pass_ok(const Target& s, const PlannedPass& p) {
  const uint32_t L = uint32_t(p.tile_bits.size());
  if (L < 10 || L > kTcTileBits || p.ops.size() > size_t(kTcMaxGates)) return false;
  for (const HOp& op : p.ops) {
    if (op.diagonal) continue;
    size_t k = op.targets.size();
    for (auto& c : op.controls)
      if (std::find(p.tile_bits.begin(), p.tile_bits.end(), s.layout[c.first]) != p.tile_bits.end()) ++k;
    if (k >= 3 && (k + 7 > L || k > 6)) return false;
  }
  return true;
}

bool plain_tc_eligible(const Target& s, const PlannedPass& p, const StageConfig& cfg) {
  if (p.staged || p.block || !cfg.plain_tensor || p.ops[0].diagonal) return false;
  std::vector<uint32_t> targets;
  for (uint32_t q : p.ops[0].targets) targets.push_back(s.layout[q]);
  return dense_tc_ok(s.n, s.bits, targets, p.ops[0].controls.size());
}

PlainTcBlob plain_tc_blob(const Target& s, const HOp& op) {
  // Targets ascending, the matrix permuted to match: new index bit i is old
  // bit order[i].
  const size_t k = op.targets.size(), D = op.matrix.dim;
  std::vector<uint32_t> phys;
  for (uint32_t q : op.targets) phys.push_back(s.layout[q]);
  std::vector<size_t> order(k);
  for (size_t i = 0; i < k; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return phys[a] < phys[b]; });
  PlainTcBlob b;
  for (size_t i = 0; i < k; ++i) b.targets.push_back(phys[order[i]]);
  std::vector<size_t> old_index(D);
  for (size_t h = 0; h < D; ++h) {
    size_t o = 0;
    for (size_t i = 0; i < k; ++i) o |= ((h >> i) & 1) << order[i];
    old_index[h] = o;
  }
  HMatrix m(D);
  for (size_t r = 0; r < D; ++r)
    for (size_t c = 0; c < D; ++c) m.at(r, c) = op.matrix.at(old_index[r], old_index[c]);
  append_tc_gate(m, b.blob);
  return b;
}

LoweredPass lower_pass(const Target& s, const PlannedPass& p, const StageConfig& cfg, StageUpload& up,
                       PlainTcBlob* pre) {
  if (p.block) return lower_block_pass(s, p, up);
  if (p.staged && cfg.tensor && cfg.low_bits >= 1 && tensor_pass_ok(s, p)) return lower_tensor_pass(s, p, cfg, up);
  if (p.staged && cfg.reg && cfg.low_bits >= 1 && register_pass_ok(s, p)) return lower_register_pass(s, p, cfg, up);
  LoweredPass lp;
  lp.staged = p.staged;
  if (!p.staged) {
    const HOp& op = p.ops[0];
    PlainGate& g = lp.plain;
    g.diagonal = op.diagonal;
    for (uint32_t q : op.targets) g.targets.push_back(s.layout[q]);
    for (auto& c : op.controls) g.controls.push_back({s.layout[c.first], c.second});
    if (g.diagonal) {
      if (op.targets.size() > QVDG_MAX_DIAGONAL_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "diagonal gates on more than 10 qubits are not supported");
      g.matrix_offset = up.push_matrix(op.matrix.diagonal_entries());
    } else if (plain_tc_eligible(s, p, cfg)) {
      const PlainTcBlob b = pre ? std::move(*pre) : plain_tc_blob(s, op);
      g.targets = b.targets;
      g.tensor = true;
      blob_align(up.tc);
      g.tc_offset = up.tc.size();
      up.tc.insert(up.tc.end(), b.blob.begin(), b.blob.end());
    } else {
      if (op.targets.size() > QVDG_MAX_GATE_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "dense gates on more than 6 qubits are not supported");
      g.matrix_offset = up.push_matrix(op.matrix.a);
    }
    return lp;
  }
  TileGeom& geo = lp.geo;
  geo.L = int(p.tile_bits.size());
  geo.B = int(cfg.low_bits);
  geo.num_tiles = uint64_t(1) << (s.n - uint32_t(geo.L));
  for (size_t j = 0; j < p.tile_bits.size(); ++j) geo.tile_bits[j] = uint8_t(p.tile_bits[j]);
  std::vector<int> local(s.n, -1);
  for (size_t j = 0; j < p.tile_bits.size(); ++j) local[p.tile_bits[j]] = int(j);
  lp.gate_offset = up.gates.size();
  geo.tc_offset = up.tc.size();
  for (const HOp& op : p.ops) {
    TileGate g{};
    std::vector<uint8_t> fixed;
    for (auto& c : op.controls) {
      const uint32_t ph = s.layout[c.first];
      if (local[ph] >= 0) {
        g.lcm |= 1u << local[ph];
        if (c.second) g.lcv |= 1u << local[ph];
        fixed.push_back(uint8_t(local[ph]));
      } else {
        g.gcm |= uint64_t(1) << ph;
        if (c.second) g.gcv |= uint64_t(1) << ph;
      }
    }
    g.k = uint8_t(op.targets.size());
    if (op.diagonal) {
      if (op.targets.size() > QVDG_MAX_DIAGONAL_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "diagonal gates on more than 10 qubits are not supported");
      g.kind = 1;
      for (size_t j = 0; j < op.targets.size(); ++j) {
        const uint32_t ph = s.layout[op.targets[j]];
        g.tgt[j] = local[ph] >= 0 ? uint8_t(local[ph]) : uint8_t(0x80 | ph);
      }
      g.mat = uint32_t(up.push_matrix(op.matrix.diagonal_entries()));
    } else {
      if (op.targets.size() > QVDG_MAX_GATE_QUBITS)
        throw Error(QVDG_ERR_UNSUPPORTED, "dense gates on more than 6 qubits are not supported");
      g.kind = 0;
      for (size_t j = 0; j < op.targets.size(); ++j) {
        const int l = local[s.layout[op.targets[j]]];
        if (l < 0) throw Error(QVDG_ERR_INVALID, "internal: dense stage gate with a global target");
        g.tgt[j] = uint8_t(l);
        fixed.push_back(uint8_t(l));
      }
      if (op.targets.size() >= 5) {
        // transposed for the row-parallel kernel
        const size_t D = op.matrix.dim;
        std::vector<C> t(D * D);
        for (size_t r = 0; r < D; ++r)
          for (size_t c = 0; c < D; ++c) t[c * D + r] = op.matrix.at(r, c);
        g.mat = uint32_t(up.push_matrix(t));
      } else {
        g.mat = uint32_t(up.push_matrix(op.matrix.a));
      }
    }
    std::sort(fixed.begin(), fixed.end());
    g.nfixed = uint8_t(fixed.size());
    for (size_t i = 0; i < fixed.size(); ++i) g.fixed[i] = fixed[i];
    up.gates.push_back(g);
  }
  geo.num_gates = int(up.gates.size() - lp.gate_offset);
  return lp;
}

void launch_pass(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev) {
  if (lp.block) {
    launch_block(s, lp, dev);
    return;
  }
  if (!lp.staged) {
    if (lp.pair)
      launch_dense_tc_pair(s, *lp.pair, dev.tc);
    else if (lp.plain.tensor)
      launch_dense_tc(s, lp.plain, dev.tc);
    else
      launch_plain_gate(s, lp.plain, dev.mats);
    return;
  }
  if (lp.geo.tensor == 2)
    launch_stage_reg(s, lp, dev);
  else if (lp.geo.tensor == 1)
    launch_stage_tc(s, lp, dev);
  else if (s.bits == 32)
    stage_launch<float>(s, lp, dev);
  else
    stage_launch<double>(s, lp, dev);
}

}  // namespace qvdg
