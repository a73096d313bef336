// Learned router: a small MLP that predicts the neighbour-count bucket of a
// point that needs an exact count, and routes it into one of two queues.
//
//   early-exit queue  predicted inliers (and every point with a long candidate
//                     list): one warp per point, 128 candidates per step,
//                     stopping as soon as the count passes K;
//   full-sweep queue  predicted outliers with a short candidate list: one lane
//                     per point, 32 points per warp, each lane sweeps its own
//                     candidates (no warp-wide step per candidate).
//
// The exact count always decides the result; a misroute only costs time, and
// the result is identical with the router on or off. The network is trained
// online, on the GPU, on the capped counts k_count has just produced (one
// Adam step every few batches).
//
// Network: x (3) -> relu(W1 x + b1) (32) -> relu(W2 h1 + b2) (32) -> W3 h2 + b3 (4)
// Parameter packing (floats): W1[32][3], b1[32], W2[32][32], b2[32], W3[4][32], b3[4]
// Loss: mean softmax cross-entropy; optimiser: Adam (Kingma & Ba 2015).
// Features: f0 = log2(1 + points in the point's bin) / 8,
//           f1 = log2(1 + points in its stencil row) / 8 (the whole stencil
//                in 1-d, the centre row of cells along the last hashed
//                dimension otherwise),
//           f2 = its capped count in the previous window / (K + 1)
//                (-1 if none yet, 2 if it was a safe inlier).
// Inference: after every training step k_table evaluates the network at the
// centres of a 32 x 32 x 16 grid over (f0, f1, f2) and stores P(count > K)
// as a byte; k_scatter routes a point by one lookup of its grid cell.
// Buckets of the capped count c (self included): 0: c <= K/4, 1: c <= K/2,
// 2: c <= K, 3: c > K.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rtod {

constexpr int MLP_IN = 3, MLP_H = 32, MLP_B = 4;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + MLP_H * MLP_IN;   // 96
constexpr int OFF_W2 = OFF_B1 + MLP_H;            // 128
constexpr int OFF_B2 = OFF_W2 + MLP_H * MLP_H;    // 1152
constexpr int OFF_W3 = OFF_B2 + MLP_H;            // 1184
constexpr int OFF_B3 = OFF_W3 + MLP_B * MLP_H;    // 1312
constexpr int MLP_P = OFF_B3 + MLP_B;             // 1316 parameters
constexpr int TRAIN_CAP = 2048;                   // training samples buffered between steps
constexpr int TRAIN_CHUNK = 128;                  // samples per chunk of k_train
constexpr int TRAIN_MAX = 128;                    // samples used by one training step
constexpr int TRAIN_STEPS = 2;                    // training steps per k_train launch at most
constexpr uint32_t INLIER_THIN = 16;              // inlier samples kept: one in 16
constexpr int TQ0 = 32, TQ1 = 32, TQ2 = 16;       // routing table grid
constexpr float F0_MAX = 1.5f, F1_MAX = 2.5f, F2_MIN = -1.0f, F2_MAX = 2.0f;

// Router state (device), one per handle.
struct RouterState {
  float params[MLP_P];
  float m[MLP_P];    // Adam first moments
  float v[MLP_P];    // Adam second moments
  float b1t, b2t;    // beta1^t, beta2^t
  float lr, beta1, beta2, eps;
  float threshold;   // route to the early-exit queue when P(bucket 3) >= threshold
  uint32_t max_sweep;  // full-sweep queue only for stencils of at most this many points
  uint32_t steps;      // Adam steps taken
  uint32_t min_samples;  // train once at least this many samples are buffered
  float last_loss;
  uint32_t n_samples;  // samples buffered (atomic counter)
  float samples[TRAIN_CAP][4];  // f0, f1, f2, label
  // routing counters (since create)
  unsigned long long routed_early, routed_sweep, misrouted;
  uint8_t table[TQ0][TQ1][TQ2];  // P(count > K) * 255 at the grid-cell centres
};

__device__ __forceinline__ int quant(float v, float lo, float hi, int n) {
  const int q = (int)((v - lo) * (float)n / (hi - lo));
  return q < 0 ? 0 : (q >= n ? n - 1 : q);
}

// Routing decision of one point from its features: true = early-exit queue.
__device__ __forceinline__ bool route_early(const RouterState* rs, const float* f) {
  const int q0 = quant(f[0], 0.0f, F0_MAX, TQ0), q1 = quant(f[1], 0.0f, F1_MAX, TQ1),
            q2 = quant(f[2], F2_MIN, F2_MAX, TQ2);
  return (float)rs->table[q0][q1][q2] >= rs->threshold * 255.0f;
}

__device__ __forceinline__ int count_bucket(int c, int K) {
  return c > K ? 3 : (4 * c <= K ? 0 : (2 * c <= K ? 1 : 2));
}

__device__ __forceinline__ float prev_feature(uint8_t pv, int K) {
  return pv == 254 ? -1.0f : (pv == 255 ? 2.0f : (float)pv / (float)(K + 1));
}

// Forward pass of one sample (one thread) with the parameters in shared or
// global memory; writes the 4 logits.
__device__ __forceinline__ void mlp_forward(const float* P, const float* x, float* z) {
  float h1[MLP_H];
#pragma unroll
  for (int i = 0; i < MLP_H; ++i) {
    float a = P[OFF_B1 + i];
#pragma unroll
    for (int j = 0; j < MLP_IN; ++j) a = fmaf(P[OFF_W1 + i * MLP_IN + j], x[j], a);
    h1[i] = fmaxf(a, 0.0f);
  }
  float h2[MLP_H];
#pragma unroll 4
  for (int i = 0; i < MLP_H; ++i) {
    float a = P[OFF_B2 + i];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) a = fmaf(P[OFF_W2 + i * MLP_H + j], h1[j], a);
    h2[i] = fmaxf(a, 0.0f);
  }
#pragma unroll
  for (int k = 0; k < MLP_B; ++k) {
    float a = P[OFF_B3 + k];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) a = fmaf(P[OFF_W3 + k * MLP_H + j], h2[j], a);
    z[k] = a;
  }
}

// Probability of bucket 3 (count > K) from the logits.
__device__ __forceinline__ float p_inlier(const float* z) {
  float mx = fmaxf(fmaxf(z[0], z[1]), fmaxf(z[2], z[3]));
  float e[MLP_B], s = 0.0f;
#pragma unroll
  for (int k = 0; k < MLP_B; ++k) {
    e[k] = expf(z[k] - mx);
    s += e[k];
  }
  return e[3] / s;
}

// ---------------------------------------------------------------------------
// One training step on n samples (x: n x 3, y: n labels) by one block of 256
// threads, deterministic: forward/backward per sample (sample-parallel, in
// chunks of TRAIN_CHUNK kept in shared memory), then every gradient entry is
// summed over the samples in a fixed order by the thread that owns it.
// grad (may be null) receives the mean-loss gradient; if adam, the parameters
// take one Adam step. Returns the mean loss in *loss.
// Shared memory: TRAIN_CHUNK * (3 + 32 + 32 + 32 + 32 + 4) floats for the
// per-sample rows, then a copy of the parameters (read by every sample).
// ---------------------------------------------------------------------------
constexpr int TRAIN_ROW = MLP_IN + 4 * MLP_H + MLP_B;  // x, h1, h2, d1, d2, d3 = 135
constexpr size_t TRAIN_SMEM = sizeof(float) * (TRAIN_CHUNK * TRAIN_ROW + MLP_P);

static __device__ void mlp_train_block(float* P, float* m, float* v, float* b1t, float* b2t, float lr, float beta1,
                                float beta2, float eps, const float* x, int xstride, const float* yf,
                                int ystride, int n, float* grad, float* loss, bool adam, float* smem) {
  const int t = threadIdx.x;
  constexpr int PER = (MLP_P + 255) / 256;  // parameters owned per thread
  float* PS = smem + TRAIN_CHUNK * TRAIN_ROW;
  for (int i = t; i < MLP_P; i += blockDim.x) PS[i] = P[i];
  __syncthreads();
  float g[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) g[q] = 0.0f;
  float lsum = 0.0f;
  const float inv_n = 1.0f / (float)n;
  for (int c0 = 0; c0 < n; c0 += TRAIN_CHUNK) {
    const int cn = min(TRAIN_CHUNK, n - c0);
    if (t < cn) {
      const int s = c0 + t;
      float* row = smem + t * TRAIN_ROW;
      float* xs = row;
      float* h1 = xs + MLP_IN;
      float* h2 = h1 + MLP_H;
      float* d1 = h2 + MLP_H;
      float* d2 = d1 + MLP_H;
      float* d3 = d2 + MLP_H;
#pragma unroll
      for (int j = 0; j < MLP_IN; ++j) xs[j] = x[(int64_t)s * xstride + j];
      const int lab = (int)yf[(int64_t)s * ystride];
      // ReLU derivatives below use h > 0, which is the same test as a > 0.
#pragma unroll 4
      for (int i = 0; i < MLP_H; ++i) {
        float a = PS[OFF_B1 + i];
#pragma unroll
        for (int j = 0; j < MLP_IN; ++j) a = fmaf(PS[OFF_W1 + i * MLP_IN + j], xs[j], a);
        h1[i] = fmaxf(a, 0.0f);
      }
#pragma unroll 2
      for (int i = 0; i < MLP_H; ++i) {
        float a = PS[OFF_B2 + i];
#pragma unroll 8
        for (int j = 0; j < MLP_H; ++j) a = fmaf(PS[OFF_W2 + i * MLP_H + j], h1[j], a);
        h2[i] = fmaxf(a, 0.0f);
      }
      float z[MLP_B], mx = -INFINITY;
#pragma unroll
      for (int k = 0; k < MLP_B; ++k) {
        float a = PS[OFF_B3 + k];
#pragma unroll 8
        for (int j = 0; j < MLP_H; ++j) a = fmaf(PS[OFF_W3 + k * MLP_H + j], h2[j], a);
        z[k] = a;
        mx = fmaxf(mx, a);
      }
      float se = 0.0f;
#pragma unroll
      for (int k = 0; k < MLP_B; ++k) se += expf(z[k] - mx);
      lsum += -(z[lab] - mx - logf(se));
#pragma unroll
      for (int k = 0; k < MLP_B; ++k) d3[k] = (expf(z[k] - mx) / se - (k == lab ? 1.0f : 0.0f)) * inv_n;
#pragma unroll 4
      for (int j = 0; j < MLP_H; ++j) {
        float a = 0.0f;
#pragma unroll
        for (int k = 0; k < MLP_B; ++k) a = fmaf(PS[OFF_W3 + k * MLP_H + j], d3[k], a);
        d2[j] = h2[j] > 0.0f ? a : 0.0f;
      }
#pragma unroll 2
      for (int j = 0; j < MLP_H; ++j) {
        float a = 0.0f;
#pragma unroll 8
        for (int i = 0; i < MLP_H; ++i) a = fmaf(PS[OFF_W2 + i * MLP_H + j], d2[i], a);
        d1[j] = h1[j] > 0.0f ? a : 0.0f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int p = t + q * 256;
      if (p >= MLP_P) break;
      // gradient term of parameter p for one sample = row[a] * (b < 0 ? 1 : row[b])
      int a, bb;
      if (p < OFF_B1) { a = MLP_IN + 2 * MLP_H + p / MLP_IN; bb = p % MLP_IN; }
      else if (p < OFF_W2) { a = MLP_IN + 2 * MLP_H + (p - OFF_B1); bb = -1; }
      else if (p < OFF_B2) { a = MLP_IN + 3 * MLP_H + (p - OFF_W2) / MLP_H; bb = MLP_IN + (p - OFF_W2) % MLP_H; }
      else if (p < OFF_W3) { a = MLP_IN + 3 * MLP_H + (p - OFF_B2); bb = -1; }
      else if (p < OFF_B3) { a = MLP_IN + 4 * MLP_H + (p - OFF_W3) / MLP_H; bb = MLP_IN + MLP_H + (p - OFF_W3) % MLP_H; }
      else { a = MLP_IN + 4 * MLP_H + (p - OFF_B3); bb = -1; }
      float acc = 0.0f;
      if (bb >= 0) {
        for (int s = 0; s < cn; ++s) acc = fmaf(smem[s * TRAIN_ROW + a], smem[s * TRAIN_ROW + bb], acc);
      } else {
        for (int s = 0; s < cn; ++s) acc += smem[s * TRAIN_ROW + a];
      }
      g[q] += acc;
    }
    __syncthreads();
  }
  // mean loss: block reduction of the per-thread sums
  float* red = smem;
  red[t] = lsum;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) red[t] += red[t + o];
    __syncthreads();
  }
  if (t == 0) *loss = red[0] * inv_n;
  __syncthreads();
  if (adam) {
    const float c1 = 1.0f - *b1t * beta1, c2 = 1.0f - *b2t * beta2;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int p = t + q * 256;
      if (p >= MLP_P) break;
      const float gi = g[q];
      const float mi = beta1 * m[p] + (1.0f - beta1) * gi;
      const float vi = beta2 * v[p] + (1.0f - beta2) * gi * gi;
      m[p] = mi;
      v[p] = vi;
      P[p] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
    __syncthreads();
    if (t == 0) {
      *b1t *= beta1;
      *b2t *= beta2;
    }
  }
  if (grad) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int p = t + q * 256;
      if (p < MLP_P) grad[p] = g[q];
    }
  }
}

// Online training: once enough samples are buffered, up to TRAIN_STEPS Adam
// steps, each on the next TRAIN_MAX buffered samples; the buffer is then
// emptied.
static __global__ void __launch_bounds__(256) k_train(RouterState* rs) {
  extern __shared__ float smem[];
  pdl_trigger();
  pdl_wait();
  const uint32_t n = min(rs->n_samples, (uint32_t)TRAIN_CAP);
  if (n < rs->min_samples || n == 0) return;
  float loss = 0.0f;
  uint32_t steps = 0;
  for (uint32_t off = 0; off < n && steps < (uint32_t)TRAIN_STEPS; off += TRAIN_MAX, ++steps) {
    const int m = (int)min((uint32_t)TRAIN_MAX, n - off);
    if (m < (int)rs->min_samples && steps > 0) break;  // a short tail waits for the next launch
    mlp_train_block(rs->params, rs->m, rs->v, &rs->b1t, &rs->b2t, rs->lr, rs->beta1, rs->beta2, rs->eps,
                    &rs->samples[off][0], 4, &rs->samples[off][3], 4, m, nullptr, &loss, true, smem);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    rs->last_loss = loss;
    rs->steps += steps;
    rs->n_samples = 0;
  }
}

// Routing table from the current parameters: one thread per grid cell.
static __global__ void __launch_bounds__(256) k_table(RouterState* rs) {
  __shared__ float P[MLP_P];
  pdl_trigger();
  pdl_wait();
  for (int i = threadIdx.x; i < MLP_P; i += blockDim.x) P[i] = rs->params[i];
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= TQ0 * TQ1 * TQ2) return;
  const int q2 = t % TQ2, q1 = (t / TQ2) % TQ1, q0 = t / (TQ2 * TQ1);
  const float x[MLP_IN] = {(q0 + 0.5f) * F0_MAX / TQ0, (q1 + 0.5f) * F1_MAX / TQ1,
                           F2_MIN + (q2 + 0.5f) * (F2_MAX - F2_MIN) / TQ2};
  float z[MLP_B];
  mlp_forward(P, x, z);
  rs->table[q0][q1][q2] = (uint8_t)fminf(255.0f, p_inlier(z) * 255.0f + 0.5f);
}

// Test kernels behind the diagnostic C ABI: gradients of a given batch and
// forward logits, on the parameters passed in.
static __global__ void __launch_bounds__(256) k_mlp_grad(float* params, const float* x, const int32_t* y, int n,
                                                  float* grad, float* loss, float* yf) {
  extern __shared__ float smem[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) yf[i] = (float)y[i];
  __syncthreads();
  mlp_train_block(params, nullptr, nullptr, nullptr, nullptr, 0.f, 0.f, 0.f, 0.f, x, 3, yf, 1, n, grad, loss,
                  false, smem);
}

static __global__ void __launch_bounds__(256) k_mlp_adam(float* params, float* m, float* v, float* bt, const float* x,
                                                  const int32_t* y, int n, float lr, float beta1, float beta2,
                                                  float eps, float* loss, float* yf) {
  extern __shared__ float smem[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) yf[i] = (float)y[i];
  __syncthreads();
  mlp_train_block(params, m, v, &bt[0], &bt[1], lr, beta1, beta2, eps, x, 3, yf, 1, n, nullptr, loss, true, smem);
}

static __global__ void k_mlp_forward(const float* params, const float* x, int n, float* logits) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float xs[MLP_IN], z[MLP_B];
  for (int j = 0; j < MLP_IN; ++j) xs[j] = x[s * MLP_IN + j];
  mlp_forward(params, xs, z);
  for (int k = 0; k < MLP_B; ++k) logits[s * MLP_B + k] = z[k];
}

}  // namespace rtod
