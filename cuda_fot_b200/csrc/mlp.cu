// The plan cost model: a 24 -> 64 -> 64 -> 1 multilayer perceptron (ReLU
// hidden layers, FP32) predicting log(seconds per iteration) of a candidate
// plan from mesh and plan features.  Forward, backward and Adam are
// hand-written kernels on CUDA cores (the matrices are tiny; there is no
// contraction worth tensor cores here).  The reference has no counterpart.
//
// Parameter layout (one contiguous float buffer):
//   W1[IN][H] | b1[H] | W2[H][H] | b2[H] | W3[H] | b3
// Loss: 0.5/N * sum_s (y_s - t_s)^2.  Inputs are standardised with the mean /
// std stored in the model.  The backward pass is deterministic: one kernel
// computes each sample's activations and deltas, a second reduces every
// parameter's gradient over the samples in a fixed order.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "devutil.cuh"
#include "engine.hpp"

namespace fot {
namespace {

constexpr int IN = FOT_MODEL_FEATURES;
constexpr int H = FOT_MODEL_HIDDEN;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + IN * H;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int NPARAM = OFF_B3 + 1;
constexpr int TPB = 128;

// Per-sample buffers of a batch (struct of arrays, sample-major rows).
struct Acts {
  float *xs;  // n x IN standardised inputs
  float *h1;  // n x H
  float *h2;  // n x H
  float *d1;  // n x H  dL/d(pre-activation 1)
  float *d2;  // n x H  dL/d(pre-activation 2)
  float *dy;  // n      dL/dy
  float *sq;  // n      squared residuals
};

// Forward (and, with targets, the deltas) of one sample per thread.
__global__ void __launch_bounds__(TPB) k_forward(const float *__restrict__ params,
                                                 const float *__restrict__ mean,
                                                 const float *__restrict__ inv_std,
                                                 const float *__restrict__ X,
                                                 const float *__restrict__ t, int n, float scale,
                                                 float *__restrict__ y, Acts a) {
  extern __shared__ float P[];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[IN], h1[H], h2[H];
#pragma unroll
  for (int i = 0; i < IN; ++i) x[i] = (X[(size_t)s * IN + i] - mean[i]) * inv_std[i];
  for (int j = 0; j < H; ++j) {
    float v = P[OFF_B1 + j];
#pragma unroll
    for (int i = 0; i < IN; ++i) v += x[i] * P[OFF_W1 + i * H + j];
    h1[j] = v > 0.f ? v : 0.f;
  }
  for (int j = 0; j < H; ++j) {
    float v = P[OFF_B2 + j];
    for (int i = 0; i < H; ++i) v += h1[i] * P[OFF_W2 + i * H + j];
    h2[j] = v > 0.f ? v : 0.f;
  }
  float out = P[OFF_B3];
  for (int i = 0; i < H; ++i) out += h2[i] * P[OFF_W3 + i];
  if (y) y[s] = out;
  if (!t) return;
  const float r = out - t[s];
  const float dy = r * scale;  // scale = 1/N of the loss
  a.dy[s] = dy;
  a.sq[s] = r * r;
  for (int i = 0; i < IN; ++i) a.xs[(size_t)s * IN + i] = x[i];
  float d2[H];
  for (int i = 0; i < H; ++i) {
    a.h1[(size_t)s * H + i] = h1[i];
    a.h2[(size_t)s * H + i] = h2[i];
    d2[i] = h2[i] > 0.f ? dy * P[OFF_W3 + i] : 0.f;
    a.d2[(size_t)s * H + i] = d2[i];
  }
  for (int i = 0; i < H; ++i) {
    float v = 0.f;
    if (h1[i] > 0.f)
      for (int j = 0; j < H; ++j) v += P[OFF_W2 + i * H + j] * d2[j];
    a.d1[(size_t)s * H + i] = v;
  }
}

// One thread per parameter: its gradient summed over the samples in order.
__global__ void k_param_grad(Acts a, int n, float *__restrict__ grad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NPARAM) return;
  float g = 0.f;
  if (q < OFF_B1) {  // W1[k][i] = sum x[k] d1[i]
    const int k = q / H, i = q % H;
    for (int s = 0; s < n; ++s) g += a.xs[(size_t)s * IN + k] * a.d1[(size_t)s * H + i];
  } else if (q < OFF_W2) {  // b1
    const int i = q - OFF_B1;
    for (int s = 0; s < n; ++s) g += a.d1[(size_t)s * H + i];
  } else if (q < OFF_B2) {  // W2[i][j] = sum h1[i] d2[j]
    const int i = (q - OFF_W2) / H, j = (q - OFF_W2) % H;
    for (int s = 0; s < n; ++s) g += a.h1[(size_t)s * H + i] * a.d2[(size_t)s * H + j];
  } else if (q < OFF_W3) {  // b2
    const int j = q - OFF_B2;
    for (int s = 0; s < n; ++s) g += a.d2[(size_t)s * H + j];
  } else if (q < OFF_B3) {  // W3[i] = sum h2[i] dy
    const int i = q - OFF_W3;
    for (int s = 0; s < n; ++s) g += a.h2[(size_t)s * H + i] * a.dy[s];
  } else {  // b3
    for (int s = 0; s < n; ++s) g += a.dy[s];
  }
  grad[q] = g;
}

__global__ void k_sum(const float *v, int n, float scale, float *out) {
  __shared__ float sh[256];
  float acc = 0.f;
  for (int i = threadIdx.x; i < n; i += 256) acc += v[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0] * scale;
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * p[i];
  m[i] = b1 * m[i] + (1.f - b1) * gi;
  v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
  p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

} // namespace
} // namespace fot

using namespace fot;

struct fot_model {
  DevBuf params, grad, m, v, mean, inv_std, loss;
  int step = 0;
};

namespace {

struct Batch {
  DevBuf X, t, xs, h1, h2, d1, d2, dy, sq;
  int n = 0;
  int alloc(int n_) {
    n = n_;
    FOT_TRY(X.alloc((size_t)n * IN * 4));
    FOT_TRY(t.alloc((size_t)n * 4));
    FOT_TRY(xs.alloc((size_t)n * IN * 4));
    FOT_TRY(h1.alloc((size_t)n * H * 4));
    FOT_TRY(h2.alloc((size_t)n * H * 4));
    FOT_TRY(d1.alloc((size_t)n * H * 4));
    FOT_TRY(d2.alloc((size_t)n * H * 4));
    FOT_TRY(dy.alloc((size_t)n * 4));
    FOT_TRY(sq.alloc((size_t)n * 4));
    return FOT_OK;
  }
  Acts acts(size_t off) {
    return Acts{xs.as<float>() + off * IN, h1.as<float>() + off * H, h2.as<float>() + off * H,
                d1.as<float>() + off * H,  d2.as<float>() + off * H, dy.as<float>() + off,
                sq.as<float>() + off};
  }
};

// Forward + deltas + parameter gradients of samples [off, off+n) of B.
int grad_pass(fot_model *M, Batch &B, size_t off, int n, float *y) {
  const size_t smem = NPARAM * sizeof(float);
  FOT_CUDA(cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_forward<<<(n + TPB - 1) / TPB, TPB, smem>>>(M->params.as<float>(), M->mean.as<float>(),
                                                M->inv_std.as<float>(), B.X.as<float>() + off * IN,
                                                B.t.as<float>() + off, n, 1.f / n, y, B.acts(off));
  k_param_grad<<<(NPARAM + 127) / 128, 128>>>(B.acts(off), n, M->grad.as<float>());
  k_sum<<<1, 256>>>(B.sq.as<float>() + off, n, 0.5f / n, M->loss.as<float>());
  FOT_CUDA(cudaGetLastError());
  return FOT_OK;
}

int adam_step(fot_model *M, float lr, float wd) {
  M->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)M->step), c2 = 1.f - std::pow(b2, (float)M->step);
  k_adam<<<(NPARAM + 255) / 256, 256>>>(M->params.as<float>(), M->grad.as<float>(), M->m.as<float>(),
                                       M->v.as<float>(), NPARAM, lr, b1, b2, 1e-8f, c1, c2, wd);
  FOT_CUDA(cudaGetLastError());
  return FOT_OK;
}

} // namespace

extern "C" {

int fot_model_num_params(void) { return NPARAM; }

int fot_model_create(uint64_t seed, fot_model **out) {
  if (!out) return fail(FOT_ERR_ARG, "null argument");
  *out = nullptr;
  auto *M = new fot_model();
  std::vector<float> p(NPARAM, 0.f);
  std::mt19937_64 g(seed);
  auto init = [&](int off, int fan_in, int count) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / fan_in));
    for (int i = 0; i < count; ++i) p[off + i] = nd(g);
  };
  init(OFF_W1, IN, IN * H);
  init(OFF_W2, H, H * H);
  init(OFF_W3, H, H);
  std::vector<float> zero(NPARAM, 0.f), mean(IN, 0.f), one(IN, 1.f);
  int rc = upload(M->params, p);
  if (rc == FOT_OK) rc = upload(M->grad, zero);
  if (rc == FOT_OK) rc = upload(M->m, zero);
  if (rc == FOT_OK) rc = upload(M->v, zero);
  if (rc == FOT_OK) rc = upload(M->mean, mean);
  if (rc == FOT_OK) rc = upload(M->inv_std, one);
  if (rc == FOT_OK) rc = M->loss.alloc(4);
  if (rc != FOT_OK) {
    delete M;
    return rc;
  }
  *out = M;
  return FOT_OK;
}

int fot_model_destroy(fot_model *M) {
  delete M;
  return FOT_OK;
}

int fot_model_set_params(fot_model *M, const float *params) {
  if (!M || !params) return fail(FOT_ERR_ARG, "null argument");
  FOT_CUDA(cudaMemcpy(M->params.ptr, params, NPARAM * 4, cudaMemcpyHostToDevice));
  return FOT_OK;
}

int fot_model_get_params(const fot_model *M, float *params) {
  if (!M || !params) return fail(FOT_ERR_ARG, "null argument");
  FOT_CUDA(cudaMemcpy(params, M->params.ptr, NPARAM * 4, cudaMemcpyDeviceToHost));
  return FOT_OK;
}

int fot_model_set_normalisation(fot_model *M, const float *mean, const float *stddev) {
  if (!M || !mean || !stddev) return fail(FOT_ERR_ARG, "null argument");
  std::vector<float> inv(IN);
  for (int i = 0; i < IN; ++i) inv[i] = stddev[i] > 0.f ? 1.f / stddev[i] : 1.f;
  FOT_CUDA(cudaMemcpy(M->mean.ptr, mean, IN * 4, cudaMemcpyHostToDevice));
  FOT_CUDA(cudaMemcpy(M->inv_std.ptr, inv.data(), IN * 4, cudaMemcpyHostToDevice));
  return FOT_OK;
}

int fot_model_predict(fot_model *M, const float *X, int n, float *y) {
  if (!M || !X || !y || n <= 0) return fail(FOT_ERR_ARG, "bad argument");
  DevBuf dX, dy;
  FOT_TRY(dX.alloc((size_t)n * IN * 4));
  FOT_TRY(dy.alloc((size_t)n * 4));
  FOT_CUDA(cudaMemcpy(dX.ptr, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice));
  const size_t smem = NPARAM * sizeof(float);
  FOT_CUDA(cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_forward<<<(n + TPB - 1) / TPB, TPB, smem>>>(M->params.as<float>(), M->mean.as<float>(),
                                                M->inv_std.as<float>(), dX.as<float>(), nullptr, n,
                                                0.f, dy.as<float>(), Acts{});
  FOT_CUDA(cudaGetLastError());
  FOT_CUDA(cudaMemcpy(y, dy.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return FOT_OK;
}

} // extern "C"

namespace {
// Device scratch of fot_model_predict_noalloc: rows x IN inputs, then rows
// outputs.  Nothing in it has to start at zero: a call copies its inputs in
// and the forward kernel writes every output row it copies back.
constexpr int kNoAllocRows = FOT_MODEL_NOALLOC_MAX_ROWS;
static __device__ __align__(256) float g_noalloc_scratch[(size_t)kNoAllocRows * (IN + 1)];
constexpr int kMaxDevices = 64;
float *g_noalloc_ptr[kMaxDevices] = {};  // per device, set by its first call
} // namespace

extern "C" {

int fot_model_predict_noalloc(fot_model *M, const float *X, int n, float *y) {
  if (!M || !X || !y || n <= 0) return fail(FOT_ERR_ARG, "bad argument");
  if (n > kNoAllocRows)
    return fail(FOT_ERR_LIMIT,
                "fot_model_predict_noalloc takes at most %d rows per call (got %d): split the "
                "rows over several calls or use fot_model_predict",
                kNoAllocRows, n);
  int dev = 0;
  FOT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(FOT_ERR_LIMIT, "device %d out of range", dev);
  if (!g_noalloc_ptr[dev]) {  // setup, once per device
    void *p = nullptr;
    FOT_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    FOT_CUDA(cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(NPARAM * sizeof(float))));
    g_noalloc_ptr[dev] = static_cast<float *>(p);
  }
  float *dX = g_noalloc_ptr[dev];
  float *dy = dX + (size_t)kNoAllocRows * IN;
  FOT_CUDA(cudaMemcpy(dX, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice));
  k_forward<<<(n + TPB - 1) / TPB, TPB, NPARAM * sizeof(float)>>>(
      M->params.as<float>(), M->mean.as<float>(), M->inv_std.as<float>(), dX, nullptr, n, 0.f, dy,
      Acts{});
  FOT_CUDA(cudaGetLastError());
  FOT_CUDA(cudaMemcpy(y, dy, (size_t)n * 4, cudaMemcpyDeviceToHost));
  return FOT_OK;
}

int fot_model_grad(fot_model *M, const float *X, const float *t, int n, float *grad, float *loss) {
  if (!M || !X || !t || n <= 0) return fail(FOT_ERR_ARG, "bad argument");
  Batch B;
  FOT_TRY(B.alloc(n));
  FOT_CUDA(cudaMemcpy(B.X.ptr, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice));
  FOT_CUDA(cudaMemcpy(B.t.ptr, t, (size_t)n * 4, cudaMemcpyHostToDevice));
  FOT_TRY(grad_pass(M, B, 0, n, nullptr));
  if (grad) FOT_CUDA(cudaMemcpy(grad, M->grad.ptr, NPARAM * 4, cudaMemcpyDeviceToHost));
  if (loss) FOT_CUDA(cudaMemcpy(loss, M->loss.ptr, 4, cudaMemcpyDeviceToHost));
  return FOT_OK;
}

int fot_model_train(fot_model *M, const float *X, const float *t, int n, int epochs, int batch,
                    float lr, float weight_decay, float *epoch_loss) {
  if (!M || !X || !t || n <= 0 || epochs <= 0 || batch <= 0) return fail(FOT_ERR_ARG, "bad argument");
  Batch B;
  FOT_TRY(B.alloc(n));
  FOT_CUDA(cudaMemcpy(B.X.ptr, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice));
  FOT_CUDA(cudaMemcpy(B.t.ptr, t, (size_t)n * 4, cudaMemcpyHostToDevice));
  for (int e = 0; e < epochs; ++e) {
    for (int off = 0; off < n; off += batch) {
      const int m = std::min(batch, n - off);
      FOT_TRY(grad_pass(M, B, (size_t)off, m, nullptr));
      FOT_TRY(adam_step(M, lr, weight_decay));
    }
    if (epoch_loss) {
      // loss of the whole set after the epoch
      FOT_TRY(grad_pass(M, B, 0, n, nullptr));
      FOT_CUDA(cudaMemcpy(&epoch_loss[e], M->loss.ptr, 4, cudaMemcpyDeviceToHost));
    }
  }
  FOT_CUDA(cudaDeviceSynchronize());
  return FOT_OK;
}

} // extern "C"
