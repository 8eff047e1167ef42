// The learned cost model's network: an MLP with two hidden ReLU layers and
// one linear output, trained with mean squared error and Adam. Every step
// runs on this file's kernels (fp32, deterministic: no atomics, fixed
// reduction order), so training and inference need no other library.
//
// Layer l computes Z = X W^T + b (X: rows x in, W: out x in) and
// A = relu(Z) for the hidden layers. Backward, with dZ the gradient at Z:
//   dW = dZ^T X, db = column sums of dZ, dX = dZ W.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "common.cuh"
#include "qvdg.h"

struct qvdg_mlp {
  int device = 0;
  uint32_t in = 0, hid = 0;
  size_t nparams = 0;
  float* params = nullptr;  // W1 b1 W2 b2 W3 b3
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  uint64_t adam_step = 0;
  // Activations and gradients for `cap` rows.
  size_t cap = 0;
  float* buf = nullptr;
  cudaStream_t stream = nullptr;
};

namespace qvdg {

namespace {

constexpr int kTile = 16;

// Y[r][o] = sum_k X[r][k] W[o][k] + b[o], then relu when RELU.
template <bool RELU>
__global__ void k_dense_fwd(const float* __restrict__ X, int rows, int in, const float* __restrict__ W,
                            const float* __restrict__ b, int out, float* __restrict__ Y) {
  __shared__ float xs[kTile][kTile + 1], ws[kTile][kTile + 1];
  const int r = blockIdx.y * kTile + threadIdx.y, o = blockIdx.x * kTile + threadIdx.x;
  float acc = 0.f;
  for (int k0 = 0; k0 < in; k0 += kTile) {
    const int kx = k0 + threadIdx.x, kw = k0 + threadIdx.y;
    xs[threadIdx.y][threadIdx.x] = (r < rows && kx < in) ? X[size_t(r) * in + kx] : 0.f;
    const int ow = blockIdx.x * kTile + threadIdx.x;
    ws[threadIdx.y][threadIdx.x] = (ow < out && kw < in) ? W[size_t(ow) * in + kw] : 0.f;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kTile; ++k) acc = fmaf(xs[threadIdx.y][k], ws[k][threadIdx.x], acc);
    __syncthreads();
  }
  if (r < rows && o < out) {
    const float z = acc + b[o];
    Y[size_t(r) * out + o] = RELU ? fmaxf(z, 0.f) : z;
  }
}

// dW[o][k] = sum_r dZ[r][o] X[r][k]; db[o] = sum_r dZ[r][o] (column k == in).
__global__ void k_dense_dw(const float* __restrict__ dZ, const float* __restrict__ X, int rows, int in, int out,
                           float* __restrict__ dW, float* __restrict__ db) {
  __shared__ float zs[kTile][kTile + 1], xs[kTile][kTile + 1];
  const int o = blockIdx.y * kTile + threadIdx.y, k = blockIdx.x * kTile + threadIdx.x;
  float acc = 0.f, accb = 0.f;
  for (int r0 = 0; r0 < rows; r0 += kTile) {
    const int rz = r0 + threadIdx.x, oz = blockIdx.y * kTile + threadIdx.y;
    zs[threadIdx.y][threadIdx.x] = (rz < rows && oz < out) ? dZ[size_t(rz) * out + oz] : 0.f;
    const int rx = r0 + threadIdx.y;
    xs[threadIdx.y][threadIdx.x] = (rx < rows && k < in) ? X[size_t(rx) * in + k] : 0.f;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kTile; ++j) {
      acc = fmaf(zs[threadIdx.y][j], xs[j][threadIdx.x], acc);
      accb += zs[threadIdx.y][j];
    }
    __syncthreads();
  }
  if (o < out && k < in) dW[size_t(o) * in + k] = acc;
  if (o < out && blockIdx.x == 0 && threadIdx.x == 0) db[o] = accb;
}

// dX[r][k] = sum_o dZ[r][o] W[o][k], then times relu'(A[r][k]) (A > 0) when
// MASK: the gradient at the previous layer's pre-activation.
template <bool MASK>
__global__ void k_dense_dx(const float* __restrict__ dZ, const float* __restrict__ W, int rows, int in, int out,
                           const float* __restrict__ A, float* __restrict__ dX) {
  __shared__ float zs[kTile][kTile + 1], ws[kTile][kTile + 1];
  const int r = blockIdx.y * kTile + threadIdx.y, k = blockIdx.x * kTile + threadIdx.x;
  float acc = 0.f;
  for (int o0 = 0; o0 < out; o0 += kTile) {
    const int oz = o0 + threadIdx.x;
    zs[threadIdx.y][threadIdx.x] = (r < rows && oz < out) ? dZ[size_t(r) * out + oz] : 0.f;
    const int ow = o0 + threadIdx.y;
    ws[threadIdx.y][threadIdx.x] = (ow < out && k < in) ? W[size_t(ow) * in + k] : 0.f;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kTile; ++j) acc = fmaf(zs[threadIdx.y][j], ws[j][threadIdx.x], acc);
    __syncthreads();
  }
  if (r < rows && k < in) {
    const size_t i = size_t(r) * in + k;
    dX[i] = MASK ? (A[i] > 0.f ? acc : 0.f) : acc;
  }
}

// dY = 2 (y - t) / rows, and per-block partial sums of (y - t)^2.
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, int rows, float* __restrict__ dy,
                      float* __restrict__ partial) {
  __shared__ float red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float e = 0.f;
  if (i < rows) {
    const float d = y[i] - t[i];
    dy[i] = 2.f * d / float(rows);
    e = d * d;
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_gather_rows(const float* __restrict__ src, const float* __restrict__ tsrc,
                              const uint32_t* __restrict__ idx, int rows, int width, float* __restrict__ dst,
                              float* __restrict__ tdst) {
  const int r = blockIdx.x, c = threadIdx.x;
  if (r >= rows) return;
  const uint32_t s = idx[r];
  for (int k = c; k < width; k += blockDim.x) dst[size_t(r) * width + k] = src[size_t(s) * width + k];
  if (c == 0) tdst[r] = tsrc[s];
}

dim3 grid2(int cols, int rows) { return dim3(unsigned((cols + kTile - 1) / kTile), unsigned((rows + kTile - 1) / kTile)); }

struct Views {
  float *W1, *b1, *W2, *b2, *W3, *b3;
};

Views views(float* base, uint32_t in, uint32_t h) {
  Views v;
  v.W1 = base;
  v.b1 = v.W1 + size_t(h) * in;
  v.W2 = v.b1 + h;
  v.b2 = v.W2 + size_t(h) * h;
  v.W3 = v.b2 + h;
  v.b3 = v.W3 + h;
  return v;
}

// Activation buffers for `rows` rows: X, t, A1, A2, y, dA2, dA1, dy, partial.
struct Acts {
  float *X, *t, *A1, *A2, *y, *dZ2, *dZ1, *dy, *partial;
};

size_t acts_floats(size_t rows, uint32_t in, uint32_t h) {
  return rows * in + rows + 2 * rows * h + rows + 2 * rows * h + rows + (rows + 255) / 256 + 64;
}

Acts acts(float* base, size_t rows, uint32_t in, uint32_t h) {
  Acts a;
  a.X = base;
  a.t = a.X + rows * in;
  a.A1 = a.t + rows;
  a.A2 = a.A1 + rows * h;
  a.y = a.A2 + rows * h;
  a.dZ2 = a.y + rows;
  a.dZ1 = a.dZ2 + rows * h;
  a.dy = a.dZ1 + rows * h;
  a.partial = a.dy + rows;
  return a;
}

void ensure(qvdg_mlp* m, size_t rows) {
  if (rows <= m->cap) return;
  if (m->buf) cudaFree(m->buf);
  m->buf = nullptr;
  m->cap = 0;
  QVDG_CUDA(cudaMalloc(&m->buf, acts_floats(rows, m->in, m->hid) * sizeof(float)));
  m->cap = rows;
}

// Row-parallel launches take rows in the grid's y dimension (at most 65535
// blocks of kTile rows): larger row counts go in chunks.
constexpr int kChunkRows = 65535 * kTile;

void forward(qvdg_mlp* m, const Acts& a, int rows) {
  const Views p = views(m->params, m->in, m->hid);
  const dim3 blk(kTile, kTile);
  const int h = int(m->hid), in = int(m->in);
  for (int r0 = 0; r0 < rows; r0 += kChunkRows) {
    const int rc = std::min(kChunkRows, rows - r0);
    const size_t o = size_t(r0);
    k_dense_fwd<true><<<grid2(h, rc), blk, 0, m->stream>>>(a.X + o * in, rc, in, p.W1, p.b1, h, a.A1 + o * h);
    k_dense_fwd<true><<<grid2(h, rc), blk, 0, m->stream>>>(a.A1 + o * h, rc, h, p.W2, p.b2, h, a.A2 + o * h);
    k_dense_fwd<false><<<grid2(1, rc), blk, 0, m->stream>>>(a.A2 + o * h, rc, h, p.W3, p.b3, 1, a.y + o);
  }
  QVDG_LAUNCH_CHECK();
}

// Gradients of the mean squared error over the rows into m->grads; returns
// the loss (host sync).
float backward(qvdg_mlp* m, const Acts& a, int rows) {
  const Views p = views(m->params, m->in, m->hid);
  const Views g = views(m->grads, m->in, m->hid);
  const dim3 blk(kTile, kTile);
  const int h = int(m->hid), in = int(m->in);
  const int nb = (rows + 255) / 256;
  k_mse<<<nb, 256, 0, m->stream>>>(a.y, a.t, rows, a.dy, a.partial);
  // output layer: dZ3 = dy (rows x 1)
  k_dense_dw<<<grid2(h, 1), blk, 0, m->stream>>>(a.dy, a.A2, rows, h, 1, g.W3, g.b3);
  for (int r0 = 0; r0 < rows; r0 += kChunkRows) {
    const int rc = std::min(kChunkRows, rows - r0);
    const size_t o = size_t(r0);
    k_dense_dx<true><<<grid2(h, rc), blk, 0, m->stream>>>(a.dy + o, p.W3, rc, h, 1, a.A2 + o * h, a.dZ2 + o * h);
  }
  k_dense_dw<<<grid2(h, h), blk, 0, m->stream>>>(a.dZ2, a.A1, rows, h, h, g.W2, g.b2);
  for (int r0 = 0; r0 < rows; r0 += kChunkRows) {
    const int rc = std::min(kChunkRows, rows - r0);
    const size_t o = size_t(r0);
    k_dense_dx<true><<<grid2(h, rc), blk, 0, m->stream>>>(a.dZ2 + o * h, p.W2, rc, h, h, a.A1 + o * h, a.dZ1 + o * h);
  }
  k_dense_dw<<<grid2(in, h), blk, 0, m->stream>>>(a.dZ1, a.X, rows, in, h, g.W1, g.b1);
  QVDG_LAUNCH_CHECK();
  std::vector<float> part(static_cast<size_t>(nb));
  QVDG_CUDA(cudaMemcpyAsync(part.data(), a.partial, part.size() * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  QVDG_CUDA(cudaStreamSynchronize(m->stream));
  double s = 0.0;
  for (float x : part) s += x;
  return float(s / rows);
}

void upload(qvdg_mlp* m, const Acts& a, const float* x, const float* t, size_t rows) {
  QVDG_CUDA(cudaMemcpyAsync(a.X, x, rows * m->in * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  if (t) QVDG_CUDA(cudaMemcpyAsync(a.t, t, rows * sizeof(float), cudaMemcpyHostToDevice, m->stream));
}

}  // namespace

qvdg_mlp* mlp_create(uint32_t in, uint32_t hid, uint64_t seed) {
  auto* m = new qvdg_mlp();
  try {
    QVDG_CUDA(cudaGetDevice(&m->device));
    m->in = in;
    m->hid = hid;
    m->nparams = size_t(hid) * in + hid + size_t(hid) * hid + hid + hid + 1;
    QVDG_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    QVDG_CUDA(cudaMalloc(&m->params, 4 * m->nparams * sizeof(float)));
    m->grads = m->params + m->nparams;
    m->adam_m = m->grads + m->nparams;
    m->adam_v = m->adam_m + m->nparams;
    QVDG_CUDA(cudaMemset(m->grads, 0, 3 * m->nparams * sizeof(float)));
    // He-uniform weights, zero biases.
    std::vector<float> p(m->nparams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](float* w, size_t count, uint32_t fan_in) {
      std::uniform_real_distribution<float> u(-std::sqrt(6.f / float(fan_in)), std::sqrt(6.f / float(fan_in)));
      for (size_t i = 0; i < count; ++i) w[i] = u(rng);
    };
    const Views v = views(p.data(), in, hid);
    fill(v.W1, size_t(hid) * in, in);
    fill(v.W2, size_t(hid) * hid, hid);
    fill(v.W3, hid, hid);
    QVDG_CUDA(cudaMemcpy(m->params, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice));
    return m;
  } catch (...) {
    if (m->params) cudaFree(m->params);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    throw;
  }
}

void mlp_destroy(qvdg_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->buf) cudaFree(m->buf);
  if (m->params) cudaFree(m->params);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

size_t mlp_num_params(const qvdg_mlp* m) { return m->nparams; }

void mlp_get_params(const qvdg_mlp* m, float* out) {
  QVDG_CUDA(cudaMemcpy(out, m->params, m->nparams * sizeof(float), cudaMemcpyDeviceToHost));
}

void mlp_set_params(qvdg_mlp* m, const float* in) {
  QVDG_CUDA(cudaMemcpy(m->params, in, m->nparams * sizeof(float), cudaMemcpyHostToDevice));
  QVDG_CUDA(cudaMemset(m->adam_m, 0, 2 * m->nparams * sizeof(float)));
  m->adam_step = 0;
}

void mlp_forward(qvdg_mlp* m, const float* x, size_t rows, float* y) {
  QVDG_CUDA(cudaSetDevice(m->device));
  ensure(m, rows);
  const Acts a = acts(m->buf, m->cap, m->in, m->hid);
  upload(m, a, x, nullptr, rows);
  forward(m, a, int(rows));
  QVDG_CUDA(cudaMemcpyAsync(y, a.y, rows * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  QVDG_CUDA(cudaStreamSynchronize(m->stream));
}

float mlp_gradients(qvdg_mlp* m, const float* x, const float* t, size_t rows, float* grads) {
  QVDG_CUDA(cudaSetDevice(m->device));
  ensure(m, rows);
  const Acts a = acts(m->buf, m->cap, m->in, m->hid);
  upload(m, a, x, t, rows);
  forward(m, a, int(rows));
  const float loss = backward(m, a, int(rows));
  if (grads) QVDG_CUDA(cudaMemcpy(grads, m->grads, m->nparams * sizeof(float), cudaMemcpyDeviceToHost));
  return loss;
}

float mlp_train(qvdg_mlp* m, const float* x, const float* t, size_t rows, uint32_t epochs, uint32_t batch, float lr,
                uint64_t seed) {
  QVDG_CUDA(cudaSetDevice(m->device));
  batch = std::max<uint32_t>(1, std::min<uint32_t>(batch, uint32_t(rows)));
  // The whole data set stays on the device; batches are gathered rows.
  float *data = nullptr;
  uint32_t* idx = nullptr;
  QVDG_CUDA(cudaMalloc(&data, rows * (m->in + 1) * sizeof(float)));
  if (cudaMalloc(&idx, rows * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(data);
    throw Error(QVDG_ERR_OUT_OF_MEMORY, "cannot allocate the training index");
  }
  float* tdata = data + rows * m->in;
  float loss = 0.f;
  try {
    QVDG_CUDA(cudaMemcpy(data, x, rows * m->in * sizeof(float), cudaMemcpyHostToDevice));
    QVDG_CUDA(cudaMemcpy(tdata, t, rows * sizeof(float), cudaMemcpyHostToDevice));
    ensure(m, std::max<size_t>(rows, batch));
    const Acts a = acts(m->buf, batch, m->in, m->hid);
    std::vector<uint32_t> order(rows);
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (uint32_t e = 0; e < epochs; ++e) {
      std::iota(order.begin(), order.end(), 0u);
      std::shuffle(order.begin(), order.end(), rng);
      QVDG_CUDA(cudaMemcpyAsync(idx, order.data(), rows * sizeof(uint32_t), cudaMemcpyHostToDevice, m->stream));
      for (size_t s = 0; s + batch <= rows; s += batch) {
        k_gather_rows<<<batch, 128, 0, m->stream>>>(data, tdata, idx + s, int(batch), int(m->in), a.X, a.t);
        forward(m, a, int(batch));
        // backward without the loss read-back (no host sync per step)
        const Views p = views(m->params, m->in, m->hid);
        const Views g = views(m->grads, m->in, m->hid);
        const dim3 blk(kTile, kTile);
        const int h = int(m->hid), in = int(m->in), rb = int(batch);
        k_mse<<<(rb + 255) / 256, 256, 0, m->stream>>>(a.y, a.t, rb, a.dy, a.partial);
        k_dense_dw<<<grid2(h, 1), blk, 0, m->stream>>>(a.dy, a.A2, rb, h, 1, g.W3, g.b3);
        k_dense_dx<true><<<grid2(h, rb), blk, 0, m->stream>>>(a.dy, p.W3, rb, h, 1, a.A2, a.dZ2);
        k_dense_dw<<<grid2(h, h), blk, 0, m->stream>>>(a.dZ2, a.A1, rb, h, h, g.W2, g.b2);
        k_dense_dx<true><<<grid2(h, rb), blk, 0, m->stream>>>(a.dZ2, p.W2, rb, h, h, a.A1, a.dZ1);
        k_dense_dw<<<grid2(in, h), blk, 0, m->stream>>>(a.dZ1, a.X, rb, in, h, g.W1, g.b1);
        ++m->adam_step;
        const float c1 = 1.f - std::pow(b1, float(m->adam_step)), c2 = 1.f - std::pow(b2, float(m->adam_step));
        k_adam<<<unsigned((m->nparams + 255) / 256), 256, 0, m->stream>>>(m->params, m->grads, m->adam_m, m->adam_v,
                                                                         m->nparams, lr, b1, b2, eps, c1, c2);
        QVDG_LAUNCH_CHECK();
      }
    }
    // Final loss over all rows.
    const Acts full = acts(m->buf, m->cap, m->in, m->hid);
    QVDG_CUDA(cudaMemcpyAsync(full.X, data, rows * m->in * sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
    QVDG_CUDA(cudaMemcpyAsync(full.t, tdata, rows * sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
    forward(m, full, int(rows));
    loss = backward(m, full, int(rows));
  } catch (...) {
    cudaFree(data);
    cudaFree(idx);
    throw;
  }
  cudaFree(data);
  cudaFree(idx);
  return loss;
}

}  // namespace qvdg
