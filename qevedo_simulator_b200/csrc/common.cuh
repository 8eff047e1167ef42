// Shared device/host helpers of the B200 state-vector engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace qvdg {

// Amplitudes are interleaved complex numbers (float2 / double2) in physical
// index order: 8-byte and 16-byte elements, so a warp's 32 consecutive
// amplitudes are one 256/512-byte coalesced access.
template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};
template <typename T>
using cplx_t = typename Cplx<T>::type;

template <typename T>
__host__ __device__ inline cplx_t<T> make_c(T re, T im) {
  cplx_t<T> c;
  c.x = re;
  c.y = im;
  return c;
}

// acc += m * x with four FMAs (the complex multiply-accumulate of the
// reference's dense rows, src/kernels.rs:330-344, written per element).
template <typename T>
__device__ __forceinline__ void cmac(cplx_t<T>& acc, const cplx_t<T>& m, const cplx_t<T>& x) {
  acc.x = fma(m.x, x.x, acc.x);
  acc.x = fma(-m.y, x.y, acc.x);
  acc.y = fma(m.x, x.y, acc.y);
  acc.y = fma(m.y, x.x, acc.y);
}

template <typename T>
__device__ __forceinline__ cplx_t<T> cmul(const cplx_t<T>& a, const cplx_t<T>& b) {
  cplx_t<T> r;
  r.x = fma(a.x, b.x, -a.y * b.y);
  r.y = fma(a.x, b.y, a.y * b.x);
  return r;
}

// Insert a zero bit at each of the `count` ascending positions in `pos`:
// enumerates the indices whose fixed bits are zero (the GPU form of the
// reference's BMI2 `deposit` over a free mask, src/kernels.rs:22-43).
__device__ __forceinline__ uint64_t insert_zeros(uint64_t x, const uint8_t* pos, int count) {
#pragma unroll 4
  for (int i = 0; i < count; ++i) {
    const uint64_t p = pos[i];
    const uint64_t low = x & ((uint64_t(1) << p) - 1);
    x = ((x >> p) << (p + 1)) | low;
  }
  return x;
}

// Error raised inside the library and turned into a status at the C ABI.
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define QVDG_CUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t err__ = (call);                                                            \
    if (err__ != cudaSuccess)                                                              \
      throw ::qvdg::Error(err__ == cudaErrorMemoryAllocation ? 2 : 3,                      \
                          std::string(#call) + ": " + cudaGetErrorString(err__));         \
  } while (0)

#define QVDG_LAUNCH_CHECK() QVDG_CUDA(cudaGetLastError())

inline int ceil_log2(uint64_t x) {
  int r = 0;
  while ((uint64_t(1) << r) < x) ++r;
  return r;
}

}  // namespace qvdg
