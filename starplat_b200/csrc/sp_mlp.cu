// The learned scheduler's network: a small MLP, with hand-written CUDA kernels
// for batched inference, the loss gradient, and fully fused training (one launch
// runs every Adam step, parameters and moments held in shared memory).
//
// Architecture (fixed): x[SP_MLP_IN] -> tanh(W1 x + b1)[H] -> tanh(W2 h1 + b2)[H]
// -> y = w3 . h2 + b3, H = SP_MLP_HIDDEN. Loss: mean squared error over the batch.
// Parameter vector layout: W1 (H x IN, row-major), b1 (H), W2 (H x H), b2 (H),
// w3 (H), b3 (1). FP32 throughout.
//
// It never affects results: it only scores candidate schedules (see sp_sssp), and
// the scheduler falls back to the fixed heuristic when no model is loaded.
#include <cmath>
#include <mutex>
#include <vector>

#include "sp_internal.cuh"

namespace sp {
namespace mlp {

constexpr int IN = SP_MLP_IN;
constexpr int H = SP_MLP_HIDDEN;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * IN;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int P = OFF_B3 + 1;
static_assert(P == SP_MLP_PARAMS, "parameter count");

// forward for one sample; keeps the activations for the backward pass
__device__ __forceinline__ float forward(const float* __restrict__ p, const float* x, float* h1, float* h2) {
#pragma unroll 4
  for (int j = 0; j < H; ++j) {
    float z = p[OFF_B1 + j];
#pragma unroll
    for (int i = 0; i < IN; ++i) z = fmaf(p[OFF_W1 + j * IN + i], x[i], z);
    h1[j] = tanhf(z);
  }
#pragma unroll 4
  for (int j = 0; j < H; ++j) {
    float z = p[OFF_B2 + j];
#pragma unroll 8
    for (int i = 0; i < H; ++i) z = fmaf(p[OFF_W2 + j * H + i], h1[i], z);
    h2[j] = tanhf(z);
  }
  float y = p[OFF_B3];
#pragma unroll 8
  for (int j = 0; j < H; ++j) y = fmaf(p[OFF_W3 + j], h2[j], y);
  return y;
}

// Add one sample's gradient (scaled by gy = dL/dy) into g, summed over the warp
// first (shuffles), then one shared/global atomic per parameter per warp.
__device__ __forceinline__ void warp_add(float* g, int idx, float v, bool lane0) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane0 && v != 0.0f) atomicAdd(&g[idx], v);
}

__device__ void backward(const float* __restrict__ p, const float* x, const float* h1, const float* h2, float gy,
                         float* g, bool lane0) {
  float dz2[H];
#pragma unroll 4
  for (int j = 0; j < H; ++j) {
    warp_add(g, OFF_W3 + j, gy * h2[j], lane0);
    dz2[j] = gy * p[OFF_W3 + j] * (1.0f - h2[j] * h2[j]);
    warp_add(g, OFF_B2 + j, dz2[j], lane0);
  }
  warp_add(g, OFF_B3, gy, lane0);
#pragma unroll 2
  for (int j = 0; j < H; ++j)
#pragma unroll 8
    for (int i = 0; i < H; ++i) warp_add(g, OFF_W2 + j * H + i, dz2[j] * h1[i], lane0);
#pragma unroll 2
  for (int i = 0; i < H; ++i) {
    float dh1 = 0.0f;
#pragma unroll 8
    for (int j = 0; j < H; ++j) dh1 = fmaf(p[OFF_W2 + j * H + i], dz2[j], dh1);
    const float dz1 = dh1 * (1.0f - h1[i] * h1[i]);
    warp_add(g, OFF_B1 + i, dz1, lane0);
#pragma unroll
    for (int k = 0; k < IN; ++k) warp_add(g, OFF_W1 + i * IN + k, dz1 * x[k], lane0);
  }
}

__global__ void k_forward(const float* __restrict__ params, const float* __restrict__ X, int N, float* __restrict__ y) {
  __shared__ float sp_[P];
  for (int i = threadIdx.x; i < P; i += blockDim.x) sp_[i] = params[i];
  __syncthreads();
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    float x[IN], h1[H], h2[H];
#pragma unroll
    for (int i = 0; i < IN; ++i) x[i] = X[(size_t)n * IN + i];
    y[n] = forward(sp_, x, h1, h2);
  }
}

// dL/dparams of L = mean (y - t)^2 into grad (zeroed by the caller) and L into loss.
__global__ void k_grad(const float* __restrict__ params, const float* __restrict__ X, const float* __restrict__ T,
                       int N, float* grad, float* loss) {
  __shared__ float sp_[P];
  __shared__ float sg[P];
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    sp_[i] = params[i];
    sg[i] = 0.0f;
  }
  __syncthreads();
  float lsum = 0.0f;
  const int lane = threadIdx.x & 31;
  // whole warps step through the samples together (shuffles need every lane)
  const int base0 = (blockIdx.x * blockDim.x + (threadIdx.x & ~31));
  for (int b = base0; b < N; b += gridDim.x * blockDim.x) {
    const int n = b + lane;
    const bool valid = n < N;
    float x[IN], h1[H], h2[H];
#pragma unroll
    for (int i = 0; i < IN; ++i) x[i] = valid ? X[(size_t)n * IN + i] : 0.0f;
    const float y = forward(sp_, x, h1, h2);
    const float r = valid ? (y - T[n]) : 0.0f;
    lsum += r * r;
    backward(sp_, x, h1, h2, 2.0f * r / (float)N, sg, lane == 0);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < P; i += blockDim.x)
    if (sg[i] != 0.0f) atomicAdd(&grad[i], sg[i]);
  lsum = warp_sum(lsum);
  if (lane == 0 && lsum != 0.0f) atomicAdd(loss, lsum / (float)N);
}

// Fused training: ONE CTA runs `steps` full-batch Adam steps; parameters,
// gradients and both moments live in shared memory for the whole run.
__global__ void __launch_bounds__(256) k_train(float* params, const float* __restrict__ X,
                                                const float* __restrict__ T, int N, int steps, float lr,
                                                float* loss_out) {
  __shared__ float sp_[P];
  __shared__ float sg[P];
  __shared__ float sm[P];
  __shared__ float sv[P];
  __shared__ float s_loss;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    sp_[i] = params[i];
    sm[i] = 0.0f;
    sv[i] = 0.0f;
  }
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int lane = threadIdx.x & 31;
  float b1t = 1.0f, b2t = 1.0f;
  for (int t = 0; t < steps; ++t) {
    for (int i = threadIdx.x; i < P; i += blockDim.x) sg[i] = 0.0f;
    if (threadIdx.x == 0) s_loss = 0.0f;
    __syncthreads();
    float lsum = 0.0f;
    for (int b = (threadIdx.x & ~31); b < N; b += blockDim.x) {
      const int n = b + lane;
      const bool valid = n < N;
      float x[IN], h1[H], h2[H];
#pragma unroll
      for (int i = 0; i < IN; ++i) x[i] = valid ? X[(size_t)n * IN + i] : 0.0f;
      const float y = forward(sp_, x, h1, h2);
      const float r = valid ? (y - T[n]) : 0.0f;
      lsum += r * r;
      backward(sp_, x, h1, h2, 2.0f * r / (float)N, sg, lane == 0);
    }
    lsum = warp_sum(lsum);
    if (lane == 0) atomicAdd(&s_loss, lsum / (float)N);
    __syncthreads();
    b1t *= b1;
    b2t *= b2;
    const float a = lr * sqrtf(1.0f - b2t) / (1.0f - b1t);
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
      const float g = sg[i];
      sm[i] = b1 * sm[i] + (1.0f - b1) * g;
      sv[i] = b2 * sv[i] + (1.0f - b2) * g * g;
      sp_[i] -= a * sm[i] / (sqrtf(sv[i]) + eps);
    }
    if (threadIdx.x == 0 && t == steps - 1) *loss_out = s_loss;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < P; i += blockDim.x) params[i] = sp_[i];
}

// ---- the loaded scheduling model (process-wide)
std::mutex g_mu;
std::vector<float> g_params;   // empty = no model: fixed heuristic
unsigned g_generation = 0;     // bumped by every sp_sched_load
std::vector<float> g_mean, g_scale;
// the per-epoch bucket-width model of SSSP (same network shape, its own inputs)
std::vector<float> g_eparams;  // params, mean, scale packed; empty = no model
unsigned g_egeneration = 0;
// the per-level direction model of BC's forward sweep
std::vector<float> g_bparams;
unsigned g_bgeneration = 0;
// the kernel-variant models, one per algorithm (params, mean, scale packed)
std::vector<float> g_vparams[VAR_ALGOS];
unsigned g_vgeneration[VAR_ALGOS] = {};
unsigned g_vcounter = 0;  // generations are unique across algorithms and loads

// Degree statistics: per-block partials in shared memory, then one atomic per counter
// per block. out[0] = max row, out[1] = sum of squares, out[2 + 2i] / out[3 + 2i] = rows
// longer than thr[i] / entries in them.
struct Thr {
  int t[DEG_THR_MAX];
  int n;
};
__global__ void __launch_bounds__(256) k_deg_stats(const int32_t* __restrict__ off, int n, Thr thr,
                                                   unsigned long long* out) {
  __shared__ unsigned long long s_acc[2 + 2 * DEG_THR_MAX];
  for (int i = threadIdx.x; i < 2 + 2 * DEG_THR_MAX; i += blockDim.x) s_acc[i] = 0;
  __syncthreads();
  unsigned long long mx = 0, sq = 0, ra[DEG_THR_MAX] = {}, ea[DEG_THR_MAX] = {};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const unsigned long long d = (unsigned long long)(off[v + 1] - off[v]);
    mx = d > mx ? d : mx;
    sq += d * d;
#pragma unroll
    for (int i = 0; i < DEG_THR_MAX; ++i)
      if (i < thr.n && d > (unsigned long long)thr.t[i]) {
        ra[i] += 1;
        ea[i] += d;
      }
  }
  atomicMax(&s_acc[0], mx);
  atomicAdd(&s_acc[1], sq);
#pragma unroll
  for (int i = 0; i < DEG_THR_MAX; ++i)
    if (i < thr.n) {
      if (ra[i]) atomicAdd(&s_acc[2 + 2 * i], ra[i]);
      if (ea[i]) atomicAdd(&s_acc[3 + 2 * i], ea[i]);
    }
  __syncthreads();
  if (threadIdx.x == 0) atomicMax(&out[0], s_acc[0]);
  if (threadIdx.x >= 1 && threadIdx.x < 2 + 2 * thr.n && s_acc[threadIdx.x])
    atomicAdd(&out[threadIdx.x], s_acc[threadIdx.x]);
}

}  // namespace mlp

int degree_stats(const int32_t* off, int n, const int* thr, int nthr, cudaStream_t s, DegStats* st) {
  if (nthr < 0 || nthr > DEG_THR_MAX) {
    set_error("degree_stats: %d thresholds (at most %d)", nthr, DEG_THR_MAX);
    return SP_ERR_INVALID;
  }
  *st = DegStats();
  if (n <= 0) return SP_OK;
  mlp::Thr t;
  t.n = nthr;
  for (int i = 0; i < DEG_THR_MAX; ++i) t.t[i] = i < nthr ? thr[i] : 0;
  dbuf<unsigned long long> acc;
  SP_TRY(acc.alloc(2 + 2 * DEG_THR_MAX));
  SP_CHECK_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(unsigned long long) * (2 + 2 * DEG_THR_MAX), s));
  const int grid = std::max(1, std::min(num_sms() * 4, (n + 255) / 256));
  mlp::k_deg_stats<<<grid, 256, 0, s>>>(off, n, t, acc.p);
  SP_CHECK_LAUNCH();
  unsigned long long h[2 + 2 * DEG_THR_MAX];
  SP_TRY(copy_out(h, acc.p, sizeof(h), s));
  st->max_deg = (int64_t)h[0];
  st->sum_sq = (int64_t)h[1];
  for (int i = 0; i < nthr; ++i) {
    st->rows_above[i] = (int64_t)h[2 + 2 * i];
    st->edges_above[i] = (int64_t)h[3 + 2 * i];
  }
  return SP_OK;
}

int degree_stats_launch(const int32_t* off, int n, const int* thr, int nthr, unsigned long long* acc,
                        cudaStream_t s) {
  if (nthr < 0 || nthr > DEG_THR_MAX) {
    set_error("degree_stats: %d thresholds (at most %d)", nthr, DEG_THR_MAX);
    return SP_ERR_INVALID;
  }
  mlp::Thr t;
  t.n = nthr;
  for (int i = 0; i < DEG_THR_MAX; ++i) t.t[i] = i < nthr ? thr[i] : 0;
  SP_CHECK_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * (2 + 2 * DEG_THR_MAX), s));
  if (n <= 0) return SP_OK;
  const int grid = std::max(1, std::min(num_sms() * 4, (n + 255) / 256));
  mlp::k_deg_stats<<<grid, 256, 0, s>>>(off, n, t, acc);
  SP_CHECK_LAUNCH();
  return SP_OK;
}

unsigned variant_model(int algo, std::vector<float>& packed) {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  if (algo < 0 || algo >= VAR_ALGOS || mlp::g_vparams[algo].empty()) {
    packed.clear();
    return 0u;
  }
  packed = mlp::g_vparams[algo];
  return mlp::g_vgeneration[algo];
}

unsigned variant_generation(int algo) {
  if (algo < 0 || algo >= VAR_ALGOS) return 0;
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  return mlp::g_vparams[algo].empty() ? 0u : mlp::g_vgeneration[algo];
}

int variant_choose(int algo, const std::vector<float>& X, const std::vector<int>& ok, int dflt, cudaStream_t s,
                   int* best) {
  std::vector<float> packed;
  {
    std::lock_guard<std::mutex> lock(mlp::g_mu);
    if (algo < 0 || algo >= VAR_ALGOS || mlp::g_vparams[algo].empty()) return SP_ERR_UNSUPPORTED;
    packed = mlp::g_vparams[algo];
  }
  const int N = (int)(X.size() / mlp::IN);
  const float* mean = packed.data() + mlp::P;
  const float* scale = mean + mlp::IN;
  const float margin = scale[mlp::IN];
  std::vector<float> Xn(X.size());
  for (int k = 0; k < N; ++k)
    for (int i = 0; i < mlp::IN; ++i) Xn[(size_t)k * mlp::IN + i] = (X[(size_t)k * mlp::IN + i] - mean[i]) * scale[i];
  dbuf<float> dp, dx, dy;
  SP_TRY(dp.alloc(mlp::P));
  SP_TRY(dx.alloc(Xn.size()));
  SP_TRY(dy.alloc(N));
  SP_CHECK_CUDA(cudaMemcpyAsync(dp.p, packed.data(), sizeof(float) * mlp::P, cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(dx.p, Xn.data(), sizeof(float) * Xn.size(), cudaMemcpyHostToDevice, s));
  mlp::k_forward<<<std::max(1, (N + 127) / 128), 128, 0, s>>>(dp.p, dx.p, N, dy.p);
  SP_CHECK_LAUNCH();
  std::vector<float> y(N);
  SP_TRY(copy_out(y.data(), dy.p, sizeof(float) * N, s));
  int b = -1;
  for (int k = 0; k < N; ++k)
    if (ok[k] && (b < 0 || y[k] < y[b])) b = k;
  if (b < 0) return SP_ERR_UNSUPPORTED;
  // leave the default only for a predicted gain above the model's margin (log units)
  if (dflt >= 0 && dflt < N && ok[dflt] && !(y[dflt] - y[b] > margin)) b = dflt;
  *best = b;
  return SP_OK;
}

// The BC level model packed for the device and its generation (0 = none loaded).
unsigned mlp_level_model(std::vector<float>& packed) {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  packed = mlp::g_bparams;
  return mlp::g_bparams.empty() ? 0u : mlp::g_bgeneration;
}

// The epoch model packed for the device (params, feature mean, feature scale) and its
// generation (0 = none loaded).
unsigned mlp_epoch_model(std::vector<float>& packed) {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  packed = mlp::g_eparams;
  return mlp::g_eparams.empty() ? 0u : mlp::g_egeneration;
}

// Score candidate rows X[n][IN] with the loaded model (host in, host out).
// Returns SP_ERR_UNSUPPORTED when no model is loaded.
unsigned mlp_generation() {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  return mlp::g_params.empty() ? 0u : mlp::g_generation;
}

int mlp_score(const std::vector<float>& X, std::vector<float>& y, cudaStream_t s) {
  std::vector<float> params, mean, scale;
  {
    std::lock_guard<std::mutex> lock(mlp::g_mu);
    if (mlp::g_params.empty()) return SP_ERR_UNSUPPORTED;
    params = mlp::g_params;
    mean = mlp::g_mean;
    scale = mlp::g_scale;
  }
  const int N = (int)(X.size() / mlp::IN);
  std::vector<float> Xn(X.size());
  for (int n = 0; n < N; ++n)
    for (int i = 0; i < mlp::IN; ++i) Xn[(size_t)n * mlp::IN + i] = (X[(size_t)n * mlp::IN + i] - mean[i]) * scale[i];
  dbuf<float> dp, dx, dy;
  SP_TRY(dp.alloc(mlp::P));
  SP_TRY(dx.alloc(Xn.size()));
  SP_TRY(dy.alloc(N));
  SP_CHECK_CUDA(cudaMemcpyAsync(dp.p, params.data(), sizeof(float) * mlp::P, cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(dx.p, Xn.data(), sizeof(float) * Xn.size(), cudaMemcpyHostToDevice, s));
  mlp::k_forward<<<std::max(1, (N + 127) / 128), 128, 0, s>>>(dp.p, dx.p, N, dy.p);
  SP_CHECK_LAUNCH();
  y.resize(N);
  return copy_out(y.data(), dy.p, sizeof(float) * N, s);
}

}  // namespace sp

using namespace sp;

namespace {
int stage(const float* src, size_t n, dbuf<float>& buf, cudaStream_t s) {
  SP_TRY(buf.alloc(n));
  if (n) SP_CHECK_CUDA(cudaMemcpyAsync(buf.p, src, sizeof(float) * n, cudaMemcpyDefault, s));
  return SP_OK;
}
}  // namespace

extern "C" int sp_mlp_forward(const float* params, const float* X, int32_t N, float* y) {
  if (!params || !X || !y || N <= 0) {
    set_error("sp_mlp_forward: invalid argument");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = 0;
  dbuf<float> dp, dx, dy;
  SP_TRY(stage(params, mlp::P, dp, s));
  SP_TRY(stage(X, (size_t)N * mlp::IN, dx, s));
  SP_TRY(dy.alloc(N));
  mlp::k_forward<<<std::max(1, (N + 127) / 128), 128, 0, s>>>(dp.p, dx.p, N, dy.p);
  SP_CHECK_LAUNCH();
  return copy_out(y, dy.p, sizeof(float) * N, s);
}

extern "C" int sp_mlp_grad(const float* params, const float* X, const float* T, int32_t N, float* grad, float* loss) {
  if (!params || !X || !T || !grad || !loss || N <= 0) {
    set_error("sp_mlp_grad: invalid argument");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = 0;
  dbuf<float> dp, dx, dt, dg;
  SP_TRY(stage(params, mlp::P, dp, s));
  SP_TRY(stage(X, (size_t)N * mlp::IN, dx, s));
  SP_TRY(stage(T, N, dt, s));
  SP_TRY(dg.alloc(mlp::P + 1));
  SP_CHECK_CUDA(cudaMemsetAsync(dg.p, 0, sizeof(float) * (mlp::P + 1), s));
  mlp::k_grad<<<std::max(1, std::min(64, (N + 255) / 256)), 256, 0, s>>>(dp.p, dx.p, dt.p, N, dg.p, dg.p + mlp::P);
  SP_CHECK_LAUNCH();
  SP_TRY(copy_out(grad, dg.p, sizeof(float) * mlp::P, s));
  return copy_out(loss, dg.p + mlp::P, sizeof(float), s);
}

extern "C" int sp_mlp_train(float* params, const float* X, const float* T, int32_t N, int32_t steps, float lr,
                            float* final_loss) {
  if (!params || !X || !T || N <= 0 || steps <= 0 || !(lr > 0)) {
    set_error("sp_mlp_train: invalid argument");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = 0;
  dbuf<float> dp, dx, dt, dl;
  SP_TRY(stage(params, mlp::P, dp, s));
  SP_TRY(stage(X, (size_t)N * mlp::IN, dx, s));
  SP_TRY(stage(T, N, dt, s));
  SP_TRY(dl.alloc(1));
  mlp::k_train<<<1, 256, 0, s>>>(dp.p, dx.p, dt.p, N, steps, lr, dl.p);
  SP_CHECK_LAUNCH();
  SP_TRY(copy_out(params, dp.p, sizeof(float) * mlp::P, s));
  if (final_loss) SP_TRY(copy_out(final_loss, dl.p, sizeof(float), s));
  return SP_OK;
}

extern "C" int sp_sched_load(const float* params, const float* feat_mean, const float* feat_scale) {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  ++mlp::g_generation;
  if (!params) {
    mlp::g_params.clear();
    return SP_OK;
  }
  if (!feat_mean || !feat_scale) {
    set_error("sp_sched_load: feature normalisation required");
    return SP_ERR_INVALID;
  }
  mlp::g_params.assign(params, params + mlp::P);
  mlp::g_mean.assign(feat_mean, feat_mean + mlp::IN);
  mlp::g_scale.assign(feat_scale, feat_scale + mlp::IN);
  return SP_OK;
}

extern "C" int sp_sched_epoch_load(const float* params, const float* feat_mean, const float* feat_scale) {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  ++mlp::g_egeneration;
  if (!params) {
    mlp::g_eparams.clear();
    return SP_OK;
  }
  if (!feat_mean || !feat_scale) {
    set_error("sp_sched_epoch_load: feature normalisation required");
    return SP_ERR_INVALID;
  }
  mlp::g_eparams.assign(params, params + mlp::P);
  mlp::g_eparams.insert(mlp::g_eparams.end(), feat_mean, feat_mean + mlp::IN);
  mlp::g_eparams.insert(mlp::g_eparams.end(), feat_scale, feat_scale + mlp::IN);
  return SP_OK;
}

extern "C" int sp_sched_level_load(const float* params, const float* feat_mean, const float* feat_scale) {
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  ++mlp::g_bgeneration;
  if (!params) {
    mlp::g_bparams.clear();
    return SP_OK;
  }
  if (!feat_mean || !feat_scale) {
    set_error("sp_sched_level_load: feature normalisation required");
    return SP_ERR_INVALID;
  }
  mlp::g_bparams.assign(params, params + mlp::P);
  mlp::g_bparams.insert(mlp::g_bparams.end(), feat_mean, feat_mean + mlp::IN);
  mlp::g_bparams.insert(mlp::g_bparams.end(), feat_scale, feat_scale + mlp::IN);
  return SP_OK;
}

extern "C" int sp_sched_variant_load(int32_t algo, const float* params, const float* feat_mean,
                                     const float* feat_scale, float margin) {
  if (algo < 0 || algo >= VAR_ALGOS) {
    set_error("sp_sched_variant_load: unknown algorithm %d", algo);
    return SP_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(mlp::g_mu);
  mlp::g_vgeneration[algo] = ++mlp::g_vcounter;
  if (!params) {
    mlp::g_vparams[algo].clear();
    return SP_OK;
  }
  if (!feat_mean || !feat_scale || !(margin >= 0.0f)) {
    set_error("sp_sched_variant_load: feature normalisation and a margin >= 0 required");
    return SP_ERR_INVALID;
  }
  std::vector<float>& v = mlp::g_vparams[algo];
  v.assign(params, params + mlp::P);
  v.insert(v.end(), feat_mean, feat_mean + mlp::IN);
  v.insert(v.end(), feat_scale, feat_scale + mlp::IN);
  v.push_back(margin);
  return SP_OK;
}

extern "C" int sp_variant_count(int32_t algo, int32_t* n) {
  if (!n || algo < 0 || algo >= VAR_ALGOS) {
    set_error("sp_variant_count: invalid argument");
    return SP_ERR_INVALID;
  }
  *n = algo == VAR_PR ? pr_variant_count()
       : algo == VAR_TC ? tc_variant_count()
       : algo == VAR_BC ? bc_variant_count()
                        : lv_variant_count();
  return SP_OK;
}

extern "C" int sp_variant_features(sp_graph_h g, int32_t algo, int32_t cand, int32_t nsrc, float* x,
                                   int32_t* applicable) {
  int32_t n = 0;
  if (!g || !x || !applicable || sp_variant_count(algo, &n) != SP_OK || cand < 0 || cand >= n) {
    set_error("sp_variant_features: invalid argument");
    return SP_ERR_INVALID;
  }
  int ok = 0;
  int st = algo == VAR_PR ? pr_variant_features(g, cand, x, &ok)
           : algo == VAR_TC ? tc_variant_features(g, cand, x, &ok)
           : algo == VAR_BC ? bc_variant_features(g, cand, std::max(1, (int)nsrc), x, &ok)
                            : lv_variant_features(g, cand, x, &ok);
  *applicable = ok;
  return st;
}
