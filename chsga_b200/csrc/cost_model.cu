// FP32 MLP cost model (8 -> 64 -> 64 -> 2, ReLU) with hand-written training
// and inference kernels. No reference counterpart.
//
// It predicts, from a request's features (read length, graph size,
// hierarchy profile, slots, traceback mode and checkpoint interval), the
// per-read device time in ms and the peak device bytes. The serving loop's
// admission control and the autotuner use it; it never touches a score.
// Targets are learned in log space, standardised; features are
// standardised with statistics of the training set.
//
// Parameters, one float array:
//   W1[8][64]  b1[64]  W2[64][64]  b2[64]  W3[64][2]  b3[2]   (4866 floats)
// with W[i][j] the weight from input i to unit j.
//
// Loss: L = 1/(2B) * sum_b sum_j (o_bj - t_bj)^2 over a batch of B, t the
// standardised log targets. Kernels (one thread per sample unless noted):
//   k_cm_forward   standardise, three layers; keeps x^, h1, h2, dL/do
//   k_cm_backward  dz2 = (W3 dL/do) * [h2 > 0], dz1 = (W2 dz2) * [h1 > 0]
//   k_cm_wgrad     one thread per parameter: sums activation x delta over
//                  the batch in sample order (deterministic, no atomics)
//   k_cm_adam      Adam update, one thread per parameter
//   k_cm_loss      one block: the batch loss in a fixed reduction order
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "common.hpp"

namespace chsga {
extern thread_local std::string g_last_error;

namespace cm {

constexpr int F = CHSGA_CM_FEATURES;
constexpr int H = CHSGA_CM_HIDDEN;
constexpr int O = CHSGA_CM_OUTPUTS;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + F * H, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H * O, NPARAM = OFF_B3 + O;
constexpr int NNORM = 2 * F + 2 * O;  // x mean, x std, y mean, y std
static_assert(NPARAM == CHSGA_CM_NUM_PARAMS, "parameter count");

#define CKM(x)                                                                              \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess)                                                                  \
      fail(e_ == cudaErrorMemoryAllocation ? CHSGA_ERR_OOM : CHSGA_ERR_CUDA,                \
           std::string(#x) + ": " + cudaGetErrorString(e_));                                \
  } while (0)

// Forward for samples idx[0..n) (idx == nullptr: 0..n-1). X raw features
// [*, F]; Y raw targets [*, O] or nullptr (inference). Outputs per batch
// position b: xn[b][F], h1[b][H], h2[b][H] (when non-null), o[b][O] in
// standardised log units, and d[b][O] = (o - t) / n when Y is given.
__global__ void __launch_bounds__(128) k_cm_forward(const float* __restrict__ P,
                                                    const float* __restrict__ norm,
                                                    const float* __restrict__ X,
                                                    const float* __restrict__ Y,
                                                    const uint32_t* __restrict__ idx, uint32_t n,
                                                    float* __restrict__ xn, float* __restrict__ h1,
                                                    float* __restrict__ h2, float* __restrict__ o,
                                                    float* __restrict__ d) {
  __shared__ float sP[NPARAM];
  __shared__ float sN[NNORM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sP[i] = P[i];
  for (int i = threadIdx.x; i < NNORM; i += blockDim.x) sN[i] = norm[i];
  __syncthreads();
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const uint32_t s = idx ? idx[b] : b;
  float x[F];
#pragma unroll
  for (int i = 0; i < F; ++i) {
    x[i] = (X[(size_t)s * F + i] - sN[i]) / sN[F + i];
    if (xn) xn[(size_t)b * F + i] = x[i];
  }
  float a1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) a1[j] = sP[OFF_B1 + j];
#pragma unroll
  for (int i = 0; i < F; ++i)
#pragma unroll
    for (int j = 0; j < H; ++j) a1[j] = fmaf(x[i], sP[OFF_W1 + i * H + j], a1[j]);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    a1[j] = fmaxf(a1[j], 0.f);
    if (h1) h1[(size_t)b * H + j] = a1[j];
  }
  float out[O];
#pragma unroll
  for (int k = 0; k < O; ++k) out[k] = sP[OFF_B3 + k];
  // layer 2 one unit at a time, folded straight into layer 3
  for (int j = 0; j < H; ++j) {
    float z = sP[OFF_B2 + j];
#pragma unroll
    for (int i = 0; i < H; ++i) z = fmaf(a1[i], sP[OFF_W2 + i * H + j], z);
    z = fmaxf(z, 0.f);
    if (h2) h2[(size_t)b * H + j] = z;
#pragma unroll
    for (int k = 0; k < O; ++k) out[k] = fmaf(z, sP[OFF_W3 + j * O + k], out[k]);
  }
#pragma unroll
  for (int k = 0; k < O; ++k) {
    o[(size_t)b * O + k] = out[k];
    if (Y && d) {
      const float t = (logf(Y[(size_t)s * O + k]) - sN[2 * F + k]) / sN[2 * F + O + k];
      d[(size_t)b * O + k] = (out[k] - t) / (float)n;
    }
  }
}

__global__ void __launch_bounds__(128) k_cm_backward(const float* __restrict__ P,
                                                     const float* __restrict__ h1,
                                                     const float* __restrict__ h2,
                                                     const float* __restrict__ d, uint32_t n,
                                                     float* __restrict__ dz1,
                                                     float* __restrict__ dz2) {
  __shared__ float sW2[H * H];
  __shared__ float sW3[H * O];
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) sW2[i] = P[OFF_W2 + i];
  for (int i = threadIdx.x; i < H * O; i += blockDim.x) sW3[i] = P[OFF_W3 + i];
  __syncthreads();
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  float g[O];
#pragma unroll
  for (int k = 0; k < O; ++k) g[k] = d[(size_t)b * O + k];
  float e2[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float v = 0.f;
#pragma unroll
    for (int k = 0; k < O; ++k) v = fmaf(sW3[j * O + k], g[k], v);
    e2[j] = h2[(size_t)b * H + j] > 0.f ? v : 0.f;
    dz2[(size_t)b * H + j] = e2[j];
  }
  for (int i = 0; i < H; ++i) {
    float v = 0.f;
#pragma unroll
    for (int j = 0; j < H; ++j) v = fmaf(sW2[i * H + j], e2[j], v);
    dz1[(size_t)b * H + i] = h1[(size_t)b * H + i] > 0.f ? v : 0.f;
  }
}

// One thread per parameter: dW[i][j] = sum_b a[b][i] * delta[b][j] and
// db[j] = sum_b delta[b][j], summed in sample order.
__global__ void k_cm_wgrad(const float* __restrict__ xn, const float* __restrict__ h1,
                           const float* __restrict__ h2, const float* __restrict__ dz1,
                           const float* __restrict__ dz2, const float* __restrict__ d, uint32_t n,
                           float* __restrict__ G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  const float* a = nullptr;  // activation column (nullptr: bias)
  const float* e = nullptr;  // delta column
  int as = 0, es = 0, i = 0, j = 0;
  if (p < OFF_B1) {
    i = (p - OFF_W1) / H, j = (p - OFF_W1) % H, a = xn, as = F, e = dz1, es = H;
  } else if (p < OFF_W2) {
    j = p - OFF_B1, e = dz1, es = H;
  } else if (p < OFF_B2) {
    i = (p - OFF_W2) / H, j = (p - OFF_W2) % H, a = h1, as = H, e = dz2, es = H;
  } else if (p < OFF_W3) {
    j = p - OFF_B2, e = dz2, es = H;
  } else if (p < OFF_B3) {
    i = (p - OFF_W3) / O, j = (p - OFF_W3) % O, a = h2, as = H, e = d, es = O;
  } else {
    j = p - OFF_B3, e = d, es = O;
  }
  float s = 0.f;
  if (a) {
    for (uint32_t b = 0; b < n; ++b) s = fmaf(a[(size_t)b * as + i], e[(size_t)b * es + j], s);
  } else {
    for (uint32_t b = 0; b < n; ++b) s += e[(size_t)b * es + j];
  }
  G[p] = s;
}

__global__ void k_cm_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                          float* __restrict__ V, float lr, float b1, float b2, float eps, float c1,
                          float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  const float g = G[p];
  const float m = b1 * M[p] + (1.f - b1) * g;
  const float v = b2 * V[p] + (1.f - b2) * g * g;
  M[p] = m;
  V[p] = v;
  P[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// One block of 256: L = 1/(2n) sum (o - t)^2 from d = (o - t)/n, i.e.
// L = n/2 * sum d^2, in a fixed order.
__global__ void __launch_bounds__(256) k_cm_loss(const float* __restrict__ d, uint32_t n,
                                                 float* __restrict__ out) {
  __shared__ float s[256];
  float v = 0.f;
  for (uint32_t i = threadIdx.x; i < n * O; i += 256) v = fmaf(d[i], d[i], v);
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = 0.5f * (float)n * s[0];
}

template <typename T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p) cudaFree(p);
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    CKM(cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T)));
    n = count;
  }
};

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double uniform01(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace cm
}  // namespace chsga

using namespace chsga;
using namespace chsga::cm;

struct chsga_cost_model {
  int device = 0;
  cudaStream_t st = nullptr;
  std::vector<float> params = std::vector<float>(NPARAM, 0.f);
  std::vector<float> norm = std::vector<float>(NNORM, 0.f);
  bool trained = false;
  std::string err;
  Buf<float> P, N, G, M, V, X, Y, xn, h1, h2, o, d, dz1, dz2, loss;
  Buf<uint32_t> idx;

  void upload() {
    CKM(cudaMemcpyAsync(P.p, params.data(), NPARAM * 4, cudaMemcpyHostToDevice, st));
    CKM(cudaMemcpyAsync(N.p, norm.data(), NNORM * 4, cudaMemcpyHostToDevice, st));
  }
  void download() {
    CKM(cudaMemcpyAsync(params.data(), P.p, NPARAM * 4, cudaMemcpyDeviceToHost, st));
    CKM(cudaStreamSynchronize(st));
  }
  void stage(const float* x, const float* y, uint32_t n) {
    X.alloc((size_t)n * F);
    CKM(cudaMemcpyAsync(X.p, x, (size_t)n * F * 4, cudaMemcpyHostToDevice, st));
    if (y) {
      Y.alloc((size_t)n * O);
      CKM(cudaMemcpyAsync(Y.p, y, (size_t)n * O * 4, cudaMemcpyHostToDevice, st));
    }
  }
  void batch_bufs(uint32_t n) {
    xn.alloc((size_t)n * F);
    h1.alloc((size_t)n * H);
    h2.alloc((size_t)n * H);
    o.alloc((size_t)n * O);
    d.alloc((size_t)n * O);
    dz1.alloc((size_t)n * H);
    dz2.alloc((size_t)n * H);
  }
  // forward + backward of the batch idx (or all n) into G
  void grad(const uint32_t* didx, uint32_t n) {
    const unsigned g = (n + 127) / 128;
    k_cm_forward<<<g, 128, 0, st>>>(P.p, N.p, X.p, Y.p, didx, n, xn.p, h1.p, h2.p, o.p, d.p);
    k_cm_backward<<<g, 128, 0, st>>>(P.p, h1.p, h2.p, d.p, n, dz1.p, dz2.p);
    k_cm_wgrad<<<(NPARAM + 127) / 128, 128, 0, st>>>(xn.p, h1.p, h2.p, dz1.p, dz2.p, d.p, n, G.p);
    CKM(cudaGetLastError());
  }
};

namespace {

template <typename F_>
chsga_status guarded_cm(chsga_cost_model* m, F_&& f) {
  try {
    if (m) CKM(cudaSetDevice(m->device));
    f();
    return CHSGA_OK;
  } catch (const ChsgaError& e) {
    if (m) m->err = e.what();
    g_last_error = e.what();
    return e.status;
  } catch (const std::exception& e) {
    if (m) m->err = e.what();
    g_last_error = e.what();
    return CHSGA_ERR_INTERNAL;
  }
}

void check_data(const float* x, const float* y, uint32_t n) {
  for (size_t i = 0; i < (size_t)n * F; ++i)
    require(std::isfinite(x[i]), CHSGA_ERR_INVALID_ARG, "non-finite feature");
  if (y)
    for (size_t i = 0; i < (size_t)n * O; ++i)
      require(std::isfinite(y[i]) && y[i] > 0.f, CHSGA_ERR_INVALID_ARG,
              "targets must be positive and finite (time ms, bytes)");
}

// Feature and log-target statistics of the training set.
void fit_norm(chsga_cost_model& m, const float* x, const float* y, uint32_t n) {
  for (int i = 0; i < F; ++i) {
    double s = 0, q = 0;
    for (uint32_t b = 0; b < n; ++b) s += x[(size_t)b * F + i];
    const double mu = s / n;
    for (uint32_t b = 0; b < n; ++b) q += (x[(size_t)b * F + i] - mu) * (x[(size_t)b * F + i] - mu);
    m.norm[i] = (float)mu;
    m.norm[F + i] = (float)std::max(1e-3, std::sqrt(q / n));
  }
  for (int k = 0; k < O; ++k) {
    double s = 0, q = 0;
    for (uint32_t b = 0; b < n; ++b) s += std::log((double)y[(size_t)b * O + k]);
    const double mu = s / n;
    for (uint32_t b = 0; b < n; ++b) {
      const double t = std::log((double)y[(size_t)b * O + k]) - mu;
      q += t * t;
    }
    m.norm[2 * F + k] = (float)mu;
    m.norm[2 * F + O + k] = (float)std::max(1e-3, std::sqrt(q / n));
  }
}

}  // namespace

extern "C" {

uint32_t chsga_cm_num_params(void) { return NPARAM; }

chsga_status chsga_cm_create(int device, uint64_t seed, chsga_cost_model** out) {
  return guarded_cm(nullptr, [&] {
    require(out != nullptr, CHSGA_ERR_INVALID_ARG, "null output");
    auto m = std::make_unique<chsga_cost_model>();
    m->device = device;
    CKM(cudaSetDevice(device));
    CKM(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    // He-uniform weights, zero biases; identity normalisation until trained
    uint64_t s = seed ^ 0x5EEDC057ull;
    auto fill = [&](int off, int fan_in, int count) {
      const double lim = std::sqrt(6.0 / fan_in);
      for (int i = 0; i < count; ++i) m->params[off + i] = (float)((2 * uniform01(s) - 1) * lim);
    };
    fill(OFF_W1, F, F * H);
    fill(OFF_W2, H, H * H);
    fill(OFF_W3, H, H * O);
    for (int i = 0; i < F; ++i) m->norm[F + i] = 1.f;
    for (int k = 0; k < O; ++k) m->norm[2 * F + O + k] = 1.f;
    m->P.alloc(NPARAM);
    m->N.alloc(NNORM);
    m->G.alloc(NPARAM);
    m->M.alloc(NPARAM);
    m->V.alloc(NPARAM);
    m->loss.alloc(1);
    m->upload();
    CKM(cudaStreamSynchronize(m->st));
    *out = m.release();
  });
}

void chsga_cm_free(chsga_cost_model* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->st) {
    cudaStreamSynchronize(m->st);
    cudaStreamDestroy(m->st);
  }
  delete m;
}

const char* chsga_cm_last_error(chsga_cost_model* m) { return m ? m->err.c_str() : g_last_error.c_str(); }

chsga_status chsga_cm_get_params(chsga_cost_model* m, float* params, float* norm) {
  return guarded_cm(m, [&] {
    require(m != nullptr, CHSGA_ERR_INVALID_ARG, "null model");
    if (params) std::memcpy(params, m->params.data(), NPARAM * 4);
    if (norm) std::memcpy(norm, m->norm.data(), NNORM * 4);
  });
}

chsga_status chsga_cm_set_params(chsga_cost_model* m, const float* params, const float* norm) {
  return guarded_cm(m, [&] {
    require(m != nullptr, CHSGA_ERR_INVALID_ARG, "null model");
    if (params) std::memcpy(m->params.data(), params, NPARAM * 4);
    if (norm) {
      for (int i = 0; i < F; ++i) require(norm[F + i] > 0, CHSGA_ERR_INVALID_ARG, "feature std <= 0");
      for (int k = 0; k < O; ++k) require(norm[2 * F + O + k] > 0, CHSGA_ERR_INVALID_ARG, "target std <= 0");
      std::memcpy(m->norm.data(), norm, NNORM * 4);
    }
    m->upload();
    CKM(cudaStreamSynchronize(m->st));
    m->trained = true;
  });
}

chsga_status chsga_cm_loss_grad(chsga_cost_model* m, const float* x, const float* y, uint32_t n,
                                float* loss, float* grad) {
  return guarded_cm(m, [&] {
    require(m && x && y && n > 0, CHSGA_ERR_INVALID_ARG, "bad argument");
    check_data(x, y, n);
    m->stage(x, y, n);
    m->batch_bufs(n);
    m->grad(nullptr, n);
    k_cm_loss<<<1, 256, 0, m->st>>>(m->d.p, n, m->loss.p);
    CKM(cudaGetLastError());
    float l = 0;
    CKM(cudaMemcpyAsync(&l, m->loss.p, 4, cudaMemcpyDeviceToHost, m->st));
    if (grad) CKM(cudaMemcpyAsync(grad, m->G.p, NPARAM * 4, cudaMemcpyDeviceToHost, m->st));
    CKM(cudaStreamSynchronize(m->st));
    if (loss) *loss = l;
  });
}

chsga_status chsga_cm_train(chsga_cost_model* m, const float* x, const float* y, uint32_t n,
                            const chsga_cm_train_opts* opts, float* final_loss) {
  return guarded_cm(m, [&] {
    require(m && x && y && n > 0, CHSGA_ERR_INVALID_ARG, "bad argument");
    check_data(x, y, n);
    chsga_cm_train_opts o = opts ? *opts : chsga_cm_train_opts{};
    if (!o.epochs) o.epochs = 200;
    if (!o.batch) o.batch = 256;
    if (!(o.lr > 0)) o.lr = 3e-3f;
    const uint32_t B = std::min(o.batch, n);
    if (!o.keep_norm) fit_norm(*m, x, y, n);
    m->upload();
    m->stage(x, y, n);
    m->batch_bufs(B);
    m->idx.alloc(n);
    CKM(cudaMemsetAsync(m->M.p, 0, NPARAM * 4, m->st));
    CKM(cudaMemsetAsync(m->V.p, 0, NPARAM * 4, m->st));
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    uint64_t s = o.seed ^ 0x7EA1Bull;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    uint64_t t = 0;
    for (uint32_t ep = 0; ep < o.epochs; ++ep) {
      for (uint32_t i = n; i > 1; --i) std::swap(perm[i - 1], perm[splitmix(s) % i]);
      CKM(cudaMemcpyAsync(m->idx.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->st));
      for (uint32_t off = 0; off + B <= n; off += B) {  // full batches only
        m->grad(m->idx.p + off, B);
        ++t;
        const float c1 = 1.f - std::pow(b1, (float)t), c2 = 1.f - std::pow(b2, (float)t);
        k_cm_adam<<<(NPARAM + 127) / 128, 128, 0, m->st>>>(m->P.p, m->G.p, m->M.p, m->V.p, o.lr, b1,
                                                           b2, eps, c1, c2);
        CKM(cudaGetLastError());
      }
      // the permutation buffer is rewritten next epoch: wait for its readers
      CKM(cudaStreamSynchronize(m->st));
    }
    m->download();
    m->trained = true;
    if (final_loss) {
      m->batch_bufs(n);
      m->grad(nullptr, n);
      k_cm_loss<<<1, 256, 0, m->st>>>(m->d.p, n, m->loss.p);
      CKM(cudaGetLastError());
      CKM(cudaMemcpyAsync(final_loss, m->loss.p, 4, cudaMemcpyDeviceToHost, m->st));
      CKM(cudaStreamSynchronize(m->st));
    }
  });
}

chsga_status chsga_cm_predict(chsga_cost_model* m, const float* x, uint32_t n, float* y_out) {
  return guarded_cm(m, [&] {
    require(m && x && y_out, CHSGA_ERR_INVALID_ARG, "bad argument");
    if (n == 0) return;
    check_data(x, nullptr, n);
    m->stage(x, nullptr, n);
    m->o.alloc((size_t)n * O);
    k_cm_forward<<<(n + 127) / 128, 128, 0, m->st>>>(m->P.p, m->N.p, m->X.p, nullptr, nullptr, n,
                                                     nullptr, nullptr, nullptr, m->o.p, nullptr);
    CKM(cudaGetLastError());
    std::vector<float> z((size_t)n * O);
    CKM(cudaMemcpyAsync(z.data(), m->o.p, z.size() * 4, cudaMemcpyDeviceToHost, m->st));
    CKM(cudaStreamSynchronize(m->st));
    for (uint32_t b = 0; b < n; ++b)
      for (int k = 0; k < O; ++k)
        y_out[(size_t)b * O + k] =
            std::exp(z[(size_t)b * O + k] * m->norm[2 * F + O + k] + m->norm[2 * F + k]);
  });
}

chsga_status chsga_cm_save(chsga_cost_model* m, const char* path) {
  return guarded_cm(m, [&] {
    require(m && path, CHSGA_ERR_INVALID_ARG, "bad argument");
    std::ofstream f(path, std::ios::binary);
    require((bool)f, CHSGA_ERR_IO, std::string("cannot write ") + path);
    const char magic[8] = {'C', 'H', 'S', 'G', 'A', 'C', 'M', '1'};
    f.write(magic, 8);
    f.write(reinterpret_cast<const char*>(m->params.data()), NPARAM * 4);
    f.write(reinterpret_cast<const char*>(m->norm.data()), NNORM * 4);
    require((bool)f, CHSGA_ERR_IO, std::string("short write to ") + path);
  });
}

chsga_status chsga_cm_load(chsga_cost_model* m, const char* path) {
  return guarded_cm(m, [&] {
    require(m && path, CHSGA_ERR_INVALID_ARG, "bad argument");
    std::ifstream f(path, std::ios::binary);
    require((bool)f, CHSGA_ERR_IO, std::string("cannot read ") + path);
    char magic[8];
    std::vector<float> p(NPARAM), nm(NNORM);
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(p.data()), NPARAM * 4);
    f.read(reinterpret_cast<char*>(nm.data()), NNORM * 4);
    require((bool)f && std::memcmp(magic, "CHSGACM1", 8) == 0, CHSGA_ERR_FORMAT,
            std::string("not a cost model file: ") + path);
    require(chsga_cm_set_params(m, p.data(), nm.data()) == CHSGA_OK, CHSGA_ERR_FORMAT, m->err);
  });
}

}  // extern "C"
