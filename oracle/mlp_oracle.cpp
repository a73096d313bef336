// CPU oracle for the router network (TEST INFRASTRUCTURE ONLY; the product
// library never links it). RTOD has no learned component, so there is no
// reference file to follow: this restates, in double precision, the network
// the product trains on the GPU, so that the GPU forward pass, gradients and
// Adam step can be checked against it.
//
// Network: x (3) -> relu(W1 x + b1) (32) -> relu(W2 h1 + b2) (32) -> W3 h2 + b3 (B)
// Loss: mean over the batch of softmax cross-entropy against integer labels.
// Parameter packing (floats, in this order):
//   W1[32][3], b1[32], W2[32][32], b2[32], W3[B][32], b3[B]

#include <cmath>
#include <cstdint>
#include <vector>

namespace {
constexpr int IN = 3, H = 32;

struct View {
  const float *W1, *b1, *W2, *b2, *W3, *b3;
  explicit View(const float* p, int B) {
    W1 = p;
    b1 = W1 + H * IN;
    W2 = b1 + H;
    b2 = W2 + H * H;
    W3 = b2 + H;
    b3 = W3 + B * H;
    (void)B;
  }
};
}  // namespace

extern "C" {

int32_t oracle_mlp_param_count(int32_t B) { return H * IN + H + H * H + H + B * H + B; }

// logits[n][B] in double.
int32_t oracle_mlp_forward(const float* params, int32_t B, const float* X, int64_t n, double* logits) {
  if (B < 2 || B > 8) return -1;
  View v(params, B);
  for (int64_t s = 0; s < n; ++s) {
    const float* x = X + s * IN;
    double h1[H], h2[H];
    for (int i = 0; i < H; ++i) {
      double a = v.b1[i];
      for (int j = 0; j < IN; ++j) a += (double)v.W1[i * IN + j] * x[j];
      h1[i] = a > 0 ? a : 0;
    }
    for (int i = 0; i < H; ++i) {
      double a = v.b2[i];
      for (int j = 0; j < H; ++j) a += (double)v.W2[i * H + j] * h1[j];
      h2[i] = a > 0 ? a : 0;
    }
    for (int k = 0; k < B; ++k) {
      double a = v.b3[k];
      for (int j = 0; j < H; ++j) a += (double)v.W3[k * H + j] * h2[j];
      logits[s * B + k] = a;
    }
  }
  return 0;
}

// Mean cross-entropy loss and its gradient (double) w.r.t. the packed params.
int32_t oracle_mlp_loss_grad(const float* params, int32_t B, const float* X, const int32_t* y,
                             int64_t n, double* loss, double* grad) {
  if (B < 2 || B > 8 || n < 1) return -1;
  View v(params, B);
  int P = oracle_mlp_param_count(B);
  for (int i = 0; i < P; ++i) grad[i] = 0;
  double* gW1 = grad;
  double* gb1 = gW1 + H * IN;
  double* gW2 = gb1 + H;
  double* gb2 = gW2 + H * H;
  double* gW3 = gb2 + H;
  double* gb3 = gW3 + B * H;
  double L = 0;
  for (int64_t s = 0; s < n; ++s) {
    const float* x = X + s * IN;
    double a1[H], h1[H], a2[H], h2[H], z[8];
    for (int i = 0; i < H; ++i) {
      double a = v.b1[i];
      for (int j = 0; j < IN; ++j) a += (double)v.W1[i * IN + j] * x[j];
      a1[i] = a;
      h1[i] = a > 0 ? a : 0;
    }
    for (int i = 0; i < H; ++i) {
      double a = v.b2[i];
      for (int j = 0; j < H; ++j) a += (double)v.W2[i * H + j] * h1[j];
      a2[i] = a;
      h2[i] = a > 0 ? a : 0;
    }
    double zmax = -INFINITY;
    for (int k = 0; k < B; ++k) {
      double a = v.b3[k];
      for (int j = 0; j < H; ++j) a += (double)v.W3[k * H + j] * h2[j];
      z[k] = a;
      zmax = a > zmax ? a : zmax;
    }
    double se = 0;
    for (int k = 0; k < B; ++k) se += std::exp(z[k] - zmax);
    int lab = y[s];
    L += -(z[lab] - zmax - std::log(se));
    double d3[8], d2[H], d1[H];
    for (int k = 0; k < B; ++k) d3[k] = (std::exp(z[k] - zmax) / se - (k == lab ? 1.0 : 0.0)) / (double)n;
    for (int j = 0; j < H; ++j) {
      double a = 0;
      for (int k = 0; k < B; ++k) a += (double)v.W3[k * H + j] * d3[k];
      d2[j] = a2[j] > 0 ? a : 0;
    }
    for (int j = 0; j < H; ++j) {
      double a = 0;
      for (int i = 0; i < H; ++i) a += (double)v.W2[i * H + j] * d2[i];
      d1[j] = a1[j] > 0 ? a : 0;
    }
    for (int k = 0; k < B; ++k) {
      gb3[k] += d3[k];
      for (int j = 0; j < H; ++j) gW3[k * H + j] += d3[k] * h2[j];
    }
    for (int i = 0; i < H; ++i) {
      gb2[i] += d2[i];
      for (int j = 0; j < H; ++j) gW2[i * H + j] += d2[i] * h1[j];
    }
    for (int i = 0; i < H; ++i) {
      gb1[i] += d1[i];
      for (int j = 0; j < IN; ++j) gW1[i * IN + j] += d1[i] * x[j];
    }
  }
  *loss = L / (double)n;
  return 0;
}

// One Adam step (Kingma & Ba 2015, Algorithm 1) on float params in place;
// m and v are the float moment buffers, t the 1-based step number.
int32_t oracle_mlp_adam(float* params, float* m, float* vv, const float* grad, int32_t P, int32_t t,
                        double lr, double b1, double b2, double eps) {
  if (t < 1) return -1;
  double c1 = 1.0 - std::pow(b1, t), c2 = 1.0 - std::pow(b2, t);
  for (int i = 0; i < P; ++i) {
    double g = grad[i];
    double mi = b1 * m[i] + (1 - b1) * g;
    double vi = b2 * vv[i] + (1 - b2) * g * g;
    m[i] = (float)mi;
    vv[i] = (float)vi;
    params[i] = (float)((double)params[i] - lr * (mi / c1) / (std::sqrt(vi / c2) + eps));
  }
  return 0;
}

}  // extern "C"
