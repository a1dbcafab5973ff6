// dmf_sched.cu -- the learned schedule picker: an MLP 12 -> 64 -> 64 -> 4 with
// bf16 weights and fp32 accumulation, trained and evaluated by the kernels
// below.  It only picks how a batch is solved (incremental repair with one of
// three settings, or a recompute from scratch); every choice yields the same
// exact flow.  No counterpart in the reference, whose schedule is fixed.
//
// The network is tiny (5,252 parameters, batch <= 64): one block holds all of
// it in shared memory, and the whole training run -- sampling, forward,
// backward, Adam -- is one launch.  Tensor cores would not help at this size:
// a step is a few hundred thousand multiply-adds and is latency-bound.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "dmf_internal.h"
#include "dmf_sched_internal.h"

using namespace dmfs;
using dmf::fail;
using dmf::ok;
using dmf::guarded;

namespace {

constexpr int kNumP = kNumW + kNumB;  // all parameters, weights first
constexpr int kMaxBatch = 64;
constexpr int kTrainThreads = 256;

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// The network in shared memory: the bf16 weights and fp32 biases are copied in
// with coalesced 16-byte loads (all of a thread's loads issued before any
// store), one DRAM round trip for the 10.8 KB, instead of each thread walking
// its own weight row with 2-byte loads -- a few dependent misses per row when
// the weights are not in L2, which is the normal case for a decision taken once
// per batch between solves that stream far more than L2 holds.
struct NetSmem {
  alignas(16) __nv_bfloat16 w[kNumW];
  float b[kNumB];
};
constexpr int kStageVec = 8;                                // bf16 per 16-byte load
constexpr int kStageRounds = kNumW / (kStageVec * kHidden);  // loads per thread
static_assert(kNumW % (kStageVec * kHidden) == 0, "weights split evenly over the block");

// Called by all kHidden threads of the block; W must be 16-byte aligned
// (cudaMalloc).  Ends with a block barrier.
__device__ __forceinline__ void stage_net(const __nv_bfloat16 *__restrict__ W, const float *__restrict__ b,
                                          NetSmem &S) {
  const uint4 *src = reinterpret_cast<const uint4 *>(W);
  uint4 *dst = reinterpret_cast<uint4 *>(S.w);
  uint4 v[kStageRounds];
#pragma unroll
  for (int r = 0; r < kStageRounds; r++) v[r] = __ldg(src + r * kHidden + threadIdx.x);
  for (int i = threadIdx.x; i < kNumB; i += kHidden) S.b[i] = __ldg(b + i);
#pragma unroll
  for (int r = 0; r < kStageRounds; r++) dst[r * kHidden + threadIdx.x] = v[r];
  __syncthreads();
}

// Forward pass of one sample by 64 threads (thread j owns hidden unit j), from
// the staged network.  In the 64 x 64 layer thread j starts its row at column
// j, so the threads of a warp read different shared-memory banks (rows are 128
// bytes apart: read in step they would all hit one bank).
__device__ void forward64(const NetSmem &S, const float *x, float *h1, float *h2, float *out) {
  const int j = threadIdx.x;
  float acc = S.b[kB1 + j];
#pragma unroll
  for (int f = 0; f < kFeatures; f++) acc += __bfloat162float(S.w[kW1 + j * kFeatures + f]) * x[f];
  h1[j] = fmaxf(acc, 0.f);
  __syncthreads();
  acc = S.b[kB2 + j];
  for (int c = 0; c < kHidden; c++) {
    const int i = (c + j) & (kHidden - 1);
    acc += __bfloat162float(S.w[kW2 + j * kHidden + i]) * h1[i];
  }
  h2[j] = fmaxf(acc, 0.f);
  __syncthreads();
  if (j < kActions) {
    acc = S.b[kB3 + j];
    for (int i = 0; i < kHidden; i++) acc += __bfloat162float(S.w[kW3 + j * kHidden + i]) * h2[i];
    out[j] = acc;
  }
  __syncthreads();
}

// One sample per block of 64 threads.
__global__ void __launch_bounds__(kHidden) k_predict(const __nv_bfloat16 *W, const float *b, const float *X, int n,
                                                     float *Y) {
  __shared__ NetSmem net;
  __shared__ float x[kFeatures], h1[kHidden], h2[kHidden], out[kActions];
  stage_net(W, b, net);
  for (int s = blockIdx.x; s < n; s += gridDim.x) {
    if (threadIdx.x < kFeatures) x[threadIdx.x] = X[(size_t)s * kFeatures + threadIdx.x];
    __syncthreads();
    forward64(net, x, h1, h2, out);
    if (threadIdx.x < kActions) Y[(size_t)s * kActions + threadIdx.x] = out[threadIdx.x];
    __syncthreads();
  }
}

// The 12 features of one batch (names in dyn_maxflow_b200/sched.py).
__device__ void make_features(const FeatAcc &a, const FeatScalars &sc, float *x) {
  const float valid = fmaxf(1.f, (float)a.valid);
  x[0] = sc.k / fmaxf(1.f, sc.m);
  x[1] = log2f(1.f + sc.k) / 24.f;
  x[2] = (float)a.dec / valid;
  x[3] = (float)a.satdec / valid;
  x[4] = fminf(1.f, (float)a.excess_created / fmaxf(1.f, sc.last_flow));
  x[5] = (float)a.incsat / valid;
  x[6] = (float)a.ins / valid;
  x[7] = (float)a.del / valid;
  x[8] = log2f(1.f + (float)a.sum_deg / valid) / 16.f;
  x[9] = log2f(1.f + (float)a.max_deg) / 24.f;
  x[10] = log2f(1.f + sc.last_levels / fmaxf(1.f, sc.last_outer)) / 16.f;
  x[11] = log2f(1.f + sc.n) / 32.f;
}

// Features, then (use_model) the forward pass and the argmin action.
// Outputs are log2 of each action's time relative to the plain schedule; a
// non-plain action is taken only when it is predicted to beat the plain one by
// more than `margin` (log2 units), so that prediction noise falls back to plain.
__global__ void __launch_bounds__(kHidden) k_decide(const __nv_bfloat16 *W, const float *b, const FeatAcc *acc,
                                                    FeatScalars sc, int use_model, float margin, float *feat,
                                                    float *pred, int *action) {
  __shared__ NetSmem net;
  __shared__ float x[kFeatures], h1[kHidden], h2[kHidden], out[kActions];
  if (use_model) stage_net(W, b, net);  // uniform over the block: every thread reaches its barrier
  if (threadIdx.x == 0) make_features(*acc, sc, x);
  __syncthreads();
  if (threadIdx.x < kFeatures) feat[threadIdx.x] = x[threadIdx.x];
  if (!use_model) {
    if (threadIdx.x < kActions) pred[threadIdx.x] = 0.f;
    if (threadIdx.x == 0) *action = 0;
    return;
  }
  forward64(net, x, h1, h2, out);
  if (threadIdx.x < kActions) pred[threadIdx.x] = out[threadIdx.x];
  if (threadIdx.x == 0) {
    int best = 0;
    float bestv = out[0] - margin;
    for (int a = 1; a < kActions; a++)
      if (out[a] < bestv) {
        best = a;
        bestv = out[a];
      }
    *action = best;
  }
}

// Shared-memory layout of the training kernel (floats).
struct TrainSmem {
  float wf[kNumP];  // forward weights: bf16-rounded masters, then fp32 biases
  float g[kNumP];   // gradients of the current minibatch
  float xs[kMaxBatch][kFeatures];
  float ys[kMaxBatch][kActions];
  float h1[kMaxBatch][kHidden];
  float h2[kMaxBatch][kHidden];
  float d2[kMaxBatch][kHidden];
  float d1[kMaxBatch][kHidden];
  float dout[kMaxBatch][kActions];
  float loss;
};

// Minibatch Adam with fp32 master weights; the forward and backward passes use
// the bf16-rounded weights (what inference uses), accumulating in fp32.  One
// block, `steps` minibatches of B samples drawn uniformly from the n samples.
__global__ void __launch_bounds__(kTrainThreads) k_train(__nv_bfloat16 *W, float *b, float *master, float *mom,
                                                         float *vel, const float *X, const float *Y, int n, int steps,
                                                         int B, float lr, unsigned long long seed, long long t0,
                                                         float *loss_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
  const int tid = threadIdx.x, nt = blockDim.x;
  const float b1m = 0.9f, b2m = 0.999f, eps = 1e-8f;
  for (int p = tid; p < kNumP; p += nt)
    S.wf[p] = p < kNumW ? __bfloat162float(__float2bfloat16_rn(master[p])) : master[p];
  __syncthreads();
  for (int step = 0; step < steps; step++) {
    // sample and load the minibatch; clear gradients and loss
    if (tid < B) {
      const int idx = (int)(mix64(seed ^ mix64(((unsigned long long)step << 8) | (unsigned)tid)) % (unsigned)n);
      for (int f = 0; f < kFeatures; f++) S.xs[tid][f] = X[(size_t)idx * kFeatures + f];
      for (int a = 0; a < kActions; a++) S.ys[tid][a] = Y[(size_t)idx * kActions + a];
    }
    for (int p = tid; p < kNumP; p += nt) S.g[p] = 0.f;
    if (tid == 0) S.loss = 0.f;
    __syncthreads();
    // forward
    for (int o = tid; o < B * kHidden; o += nt) {
      const int s = o / kHidden, j = o % kHidden;
      float acc = S.wf[kNumW + kB1 + j];
      for (int f = 0; f < kFeatures; f++) acc += S.wf[kW1 + j * kFeatures + f] * S.xs[s][f];
      S.h1[s][j] = fmaxf(acc, 0.f);
    }
    __syncthreads();
    for (int o = tid; o < B * kHidden; o += nt) {
      const int s = o / kHidden, j = o % kHidden;
      float acc = S.wf[kNumW + kB2 + j];
      for (int i = 0; i < kHidden; i++) acc += S.wf[kW2 + j * kHidden + i] * S.h1[s][i];
      S.h2[s][j] = fmaxf(acc, 0.f);
    }
    __syncthreads();
    float lsum = 0.f;
    for (int o = tid; o < B * kActions; o += nt) {
      const int s = o / kActions, a = o % kActions;
      float acc = S.wf[kNumW + kB3 + a];
      for (int i = 0; i < kHidden; i++) acc += S.wf[kW3 + a * kHidden + i] * S.h2[s][i];
      const float e = acc - S.ys[s][a];
      lsum += e * e;
      S.dout[s][a] = 2.f * e / (float)(B * kActions);
    }
    atomicAdd(&S.loss, lsum);
    __syncthreads();
    // backward: layer 3
    for (int o = tid; o < kActions * kHidden; o += nt) {
      const int a = o / kHidden, j = o % kHidden;
      float acc = 0.f;
      for (int s = 0; s < B; s++) acc += S.dout[s][a] * S.h2[s][j];
      S.g[kW3 + o] = acc;
    }
    if (tid < kActions) {
      float acc = 0.f;
      for (int s = 0; s < B; s++) acc += S.dout[s][tid];
      S.g[kNumW + kB3 + tid] = acc;
    }
    for (int o = tid; o < B * kHidden; o += nt) {
      const int s = o / kHidden, j = o % kHidden;
      float acc = 0.f;
      for (int a = 0; a < kActions; a++) acc += S.wf[kW3 + a * kHidden + j] * S.dout[s][a];
      S.d2[s][j] = S.h2[s][j] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    // layer 2
    for (int o = tid; o < kHidden * kHidden; o += nt) {
      const int j = o / kHidden, i = o % kHidden;
      float acc = 0.f;
      for (int s = 0; s < B; s++) acc += S.d2[s][j] * S.h1[s][i];
      S.g[kW2 + o] = acc;
    }
    if (tid < kHidden) {
      float acc = 0.f;
      for (int s = 0; s < B; s++) acc += S.d2[s][tid];
      S.g[kNumW + kB2 + tid] = acc;
    }
    for (int o = tid; o < B * kHidden; o += nt) {
      const int s = o / kHidden, i = o % kHidden;
      float acc = 0.f;
      for (int j = 0; j < kHidden; j++) acc += S.wf[kW2 + j * kHidden + i] * S.d2[s][j];
      S.d1[s][i] = S.h1[s][i] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    // layer 1
    for (int o = tid; o < kHidden * kFeatures; o += nt) {
      const int i = o / kFeatures, f = o % kFeatures;
      float acc = 0.f;
      for (int s = 0; s < B; s++) acc += S.d1[s][i] * S.xs[s][f];
      S.g[kW1 + o] = acc;
    }
    if (tid < kHidden) {
      float acc = 0.f;
      for (int s = 0; s < B; s++) acc += S.d1[s][tid];
      S.g[kNumW + kB1 + tid] = acc;
    }
    __syncthreads();
    // Adam on the masters; refresh the forward weights
    const long long t = t0 + step + 1;
    const float c1 = 1.f - powf(b1m, (float)t), c2 = 1.f - powf(b2m, (float)t);
    for (int p = tid; p < kNumP; p += nt) {
      const float g = S.g[p];
      const float m1 = b1m * mom[p] + (1.f - b1m) * g;
      const float v1 = b2m * vel[p] + (1.f - b2m) * g * g;
      mom[p] = m1;
      vel[p] = v1;
      const float w = master[p] - lr * (m1 / c1) / (sqrtf(v1 / c2) + eps);
      master[p] = w;
      S.wf[p] = p < kNumW ? __bfloat162float(__float2bfloat16_rn(w)) : w;
    }
    if (tid == 0 && loss_out) loss_out[step] = S.loss / (float)(B * kActions);
    __syncthreads();
  }
  for (int p = tid; p < kNumP; p += nt) {
    if (p < kNumW) W[p] = __float2bfloat16_rn(master[p]);
    else b[p - kNumW] = master[p];
  }
}

// masters -> bf16 weights and fp32 biases
__global__ void k_publish(const float *master, __nv_bfloat16 *W, float *b) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kNumP; p += gridDim.x * blockDim.x) {
    if (p < kNumW) W[p] = __float2bfloat16_rn(master[p]);
    else b[p - kNumW] = master[p];
  }
}

}  // namespace

struct dmf_sched {
  int dev = 0;
  cudaStream_t stream = nullptr;
  __nv_bfloat16 *W = nullptr;
  float *b = nullptr;
  float *master = nullptr, *mom = nullptr, *vel = nullptr;
  float *io = nullptr;  // decision outputs: feat[12] | pred[4] | action (int)
  float *h_io = nullptr;  // pinned
  long long adam_t = 0;
  bool trained = false;
  float margin = 0.1f;  // log2 units a non-plain action must win by
  std::mutex mu;  // one call at a time per model (training, prediction, decisions)
};

namespace {

#define SCK(call, what)                                                                           \
  do {                                                                                            \
    cudaError_t _e = (call);                                                                      \
    if (_e != cudaSuccess)                                                                        \
      return fail(_e == cudaErrorMemoryAllocation ? DMF_ERR_OOM : DMF_ERR_CUDA, "%s: %s", what,    \
                  cudaGetErrorString(_e));                                                        \
  } while (0)

int init_masters(dmf_sched *s, uint64_t seed) {
  std::vector<float> h(kNumP, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int rows, int fan_in) {
    const float a = std::sqrt(6.f / (float)fan_in);
    std::uniform_real_distribution<float> u(-a, a);
    for (int i = 0; i < rows * fan_in; i++) h[off + i] = u(rng);
  };
  fill(kW1, kHidden, kFeatures);
  fill(kW2, kHidden, kHidden);
  fill(kW3, kActions, kHidden);
  SCK(cudaMemcpyAsync(s->master, h.data(), sizeof(float) * kNumP, cudaMemcpyHostToDevice, s->stream), "H2D init");
  SCK(cudaMemsetAsync(s->mom, 0, sizeof(float) * kNumP, s->stream), "memset");
  SCK(cudaMemsetAsync(s->vel, 0, sizeof(float) * kNumP, s->stream), "memset");
  k_publish<<<(kNumP + 255) / 256, 256, 0, s->stream>>>(s->master, s->W, s->b);
  SCK(cudaGetLastError(), "publish");
  SCK(cudaStreamSynchronize(s->stream), "init");
  s->adam_t = 0;
  s->trained = false;
  return DMF_OK;
}

}  // namespace

extern "C" {

int dmf_sched_create(int32_t device, uint64_t seed, dmf_sched **out) {
  return guarded([&]() -> int {
    if (!out) return fail(DMF_ERR_INVALID_ARG, "null output");
    *out = nullptr;
    int dev = device;
    if (dev < 0) SCK(cudaGetDevice(&dev), "cudaGetDevice");
    SCK(cudaSetDevice(dev), "cudaSetDevice");
    dmf_sched *s = new dmf_sched();
    s->dev = dev;
    auto bail = [&](int st) {  // the destroy clears the last error: keep the message across it
      char msg[1024];
      std::snprintf(msg, sizeof msg, "%s", dmf_last_error());
      dmf_sched_destroy(s);
      return fail(st, "%s", msg);
    };
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&s->W, sizeof(__nv_bfloat16) * kNumW) != cudaSuccess ||
        cudaMalloc(&s->b, sizeof(float) * kNumB) != cudaSuccess ||
        cudaMalloc(&s->master, sizeof(float) * kNumP) != cudaSuccess ||
        cudaMalloc(&s->mom, sizeof(float) * kNumP) != cudaSuccess ||
        cudaMalloc(&s->vel, sizeof(float) * kNumP) != cudaSuccess ||
        cudaMalloc(&s->io, sizeof(float) * 32) != cudaSuccess ||
        cudaMallocHost(&s->h_io, sizeof(float) * 32) != cudaSuccess)
      return bail(fail(DMF_ERR_OOM, "scheduler allocation: %s", cudaGetErrorString(cudaGetLastError())));
    int st;
    try {
      st = init_masters(s, seed);
    } catch (...) {
      dmf_sched_destroy(s);
      throw;
    }
    if (st) return bail(st);
    *out = s;
    return ok();
  });
}

int dmf_sched_destroy(dmf_sched *s) {
  if (!s) return ok();
  cudaSetDevice(s->dev);
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaFree(s->W);
  cudaFree(s->b);
  cudaFree(s->master);
  cudaFree(s->mom);
  cudaFree(s->vel);
  cudaFree(s->io);
  if (s->h_io) cudaFreeHost(s->h_io);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return ok();
}

int dmf_sched_set_weights(dmf_sched *s, const uint16_t *weights, const float *biases) {
  return guarded([&]() -> int {
    if (!s || !weights || !biases) return fail(DMF_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    SCK(cudaSetDevice(s->dev), "cudaSetDevice");
    std::vector<float> h(kNumP);
    for (int i = 0; i < kNumW; i++) {
      const uint32_t bits = (uint32_t)weights[i] << 16;
      std::memcpy(&h[i], &bits, 4);
      if (!std::isfinite(h[i])) return fail(DMF_ERR_INVALID_ARG, "weight %d is not finite", i);
    }
    for (int i = 0; i < kNumB; i++) {
      if (!std::isfinite(biases[i])) return fail(DMF_ERR_INVALID_ARG, "bias %d is not finite", i);
      h[kNumW + i] = biases[i];
    }
    SCK(cudaMemcpyAsync(s->master, h.data(), sizeof(float) * kNumP, cudaMemcpyHostToDevice, s->stream), "H2D weights");
    SCK(cudaMemsetAsync(s->mom, 0, sizeof(float) * kNumP, s->stream), "memset");
    SCK(cudaMemsetAsync(s->vel, 0, sizeof(float) * kNumP, s->stream), "memset");
    k_publish<<<(kNumP + 255) / 256, 256, 0, s->stream>>>(s->master, s->W, s->b);
    SCK(cudaGetLastError(), "publish");
    SCK(cudaStreamSynchronize(s->stream), "set weights");
    s->adam_t = 0;
    s->trained = true;
    return ok();
  });
}

int dmf_sched_set_margin(dmf_sched *s, float margin) {
  if (!s || !(margin >= 0.f) || !std::isfinite(margin)) return fail(DMF_ERR_INVALID_ARG, "margin must be >= 0");
  std::lock_guard<std::mutex> lock(s->mu);
  s->margin = margin;
  return ok();
}

int dmf_sched_get_weights(dmf_sched *s, uint16_t *weights, float *biases) {
  if (!s || !weights || !biases) return fail(DMF_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  SCK(cudaSetDevice(s->dev), "cudaSetDevice");
  SCK(cudaMemcpyAsync(weights, s->W, 2 * kNumW, cudaMemcpyDeviceToHost, s->stream), "D2H weights");
  SCK(cudaMemcpyAsync(biases, s->b, sizeof(float) * kNumB, cudaMemcpyDeviceToHost, s->stream), "D2H biases");
  SCK(cudaStreamSynchronize(s->stream), "get weights");
  return ok();
}

int dmf_sched_train(dmf_sched *s, int32_t n, const float *X, const float *Y, int32_t steps, int32_t batch, float lr,
                    uint64_t seed, float *loss) {
  return guarded([&]() -> int {
    if (!s || n <= 0 || !X || !Y || steps < 0 || batch < 1 || batch > kMaxBatch || !(lr > 0.f) || !std::isfinite(lr))
      return fail(DMF_ERR_INVALID_ARG, "bad training arguments (n > 0, 1 <= batch <= %d, lr > 0)", kMaxBatch);
    std::lock_guard<std::mutex> lock(s->mu);
    for (size_t i = 0; i < (size_t)n * kFeatures; i++)
      if (!std::isfinite(X[i])) return fail(DMF_ERR_INVALID_ARG, "feature value %zu is not finite", i);
    for (size_t i = 0; i < (size_t)n * kActions; i++)
      if (!std::isfinite(Y[i])) return fail(DMF_ERR_INVALID_ARG, "target value %zu is not finite", i);
    SCK(cudaSetDevice(s->dev), "cudaSetDevice");
    float *dX = nullptr, *dY = nullptr, *dL = nullptr;
    auto cleanup = [&]() {
      cudaFree(dX);
      cudaFree(dY);
      cudaFree(dL);
    };
    if (cudaMalloc(&dX, sizeof(float) * kFeatures * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dY, sizeof(float) * kActions * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dL, sizeof(float) * std::max(steps, 1)) != cudaSuccess) {
      cleanup();
      return fail(DMF_ERR_OOM, "training buffers");
    }
    cudaError_t e = cudaMemcpyAsync(dX, X, sizeof(float) * kFeatures * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dY, Y, sizeof(float) * kActions * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    const int smem = (int)sizeof(TrainSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess && steps > 0) {
      k_train<<<1, kTrainThreads, smem, s->stream>>>(s->W, s->b, s->master, s->mom, s->vel, dX, dY, n, steps, batch, lr,
                                                      seed, s->adam_t, dL);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && loss && steps > 0)
      e = cudaMemcpyAsync(loss, dL, sizeof(float) * steps, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cleanup();
    if (e != cudaSuccess) return fail(DMF_ERR_CUDA, "training: %s", cudaGetErrorString(e));
    s->adam_t += steps;
    s->trained = true;
    return ok();
  });
}

int dmf_sched_predict(dmf_sched *s, int32_t n, const float *X, float *Y) {
  return guarded([&]() -> int {
    if (!s || n < 0 || (n > 0 && (!X || !Y))) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
    std::lock_guard<std::mutex> lock(s->mu);
    if (n == 0) return ok();
    SCK(cudaSetDevice(s->dev), "cudaSetDevice");
    float *dX = nullptr, *dY = nullptr;
    if (cudaMalloc(&dX, sizeof(float) * kFeatures * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dY, sizeof(float) * kActions * (size_t)n) != cudaSuccess) {
      cudaFree(dX);
      cudaFree(dY);
      return fail(DMF_ERR_OOM, "prediction buffers");
    }
    cudaError_t e = cudaMemcpyAsync(dX, X, sizeof(float) * kFeatures * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
      k_predict<<<std::min(n, 4096), kHidden, 0, s->stream>>>(s->W, s->b, dX, n, dY);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(Y, dY, sizeof(float) * kActions * (size_t)n, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(dX);
    cudaFree(dY);
    if (e != cudaSuccess) return fail(DMF_ERR_CUDA, "prediction: %s", cudaGetErrorString(e));
    return ok();
  });
}

}  // extern "C"

int dmf_sched_decide(dmf_sched *s, const FeatAcc *d_acc, const FeatScalars &sc, cudaStream_t stream, int device,
                     float *h_feat, float *h_pred, int *h_action) {
  // without a model the decision buffers of a per-device scratch are used
  static float *scratch[64] = {nullptr};
  static float *h_scratch[64] = {nullptr};
  static std::mutex scratch_mu;
  std::unique_lock<std::mutex> lock = s ? std::unique_lock<std::mutex>(s->mu) : std::unique_lock<std::mutex>(scratch_mu);
  float *io = nullptr, *h_io = nullptr;
  const __nv_bfloat16 *W = nullptr;
  const float *b = nullptr;
  const bool use = s && s->trained;
  if (s) {
    if (s->dev != device) return fail(DMF_ERR_INVALID_ARG, "scheduler and solver are on different devices");
    io = s->io;
    h_io = s->h_io;
    W = s->W;
    b = s->b;
  } else {
    if (device < 0 || device >= 64) return fail(DMF_ERR_INVALID_ARG, "device id");
    if (!scratch[device]) {
      SCK(cudaMalloc(&scratch[device], sizeof(float) * 32), "decision scratch");
      SCK(cudaMallocHost(&h_scratch[device], sizeof(float) * 32), "decision scratch");
    }
    io = scratch[device];
    h_io = h_scratch[device];
  }
  k_decide<<<1, kHidden, 0, stream>>>(W, b, d_acc, sc, use ? 1 : 0, s ? s->margin : 0.f, io, io + kFeatures,
                                      (int *)(io + kFeatures + kActions));
  SCK(cudaGetLastError(), "decision launch");
  SCK(cudaMemcpyAsync(h_io, io, sizeof(float) * (kFeatures + kActions + 1), cudaMemcpyDeviceToHost, stream), "D2H decision");
  SCK(cudaStreamSynchronize(stream), "decision");
  if (h_feat) std::memcpy(h_feat, h_io, sizeof(float) * kFeatures);
  if (h_pred) std::memcpy(h_pred, h_io + kFeatures, sizeof(float) * kActions);
  int a = 0;
  std::memcpy(&a, h_io + kFeatures + kActions, sizeof(int));
  if (a < 0 || a >= kActions) a = 0;
  *h_action = a;
  return DMF_OK;
}
