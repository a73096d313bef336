// Host engine and C ABI of the detector (include/rtod.h).
//
// One rtod_handle = one stream. It owns a CUDA stream, the device ring and
// the cell-ordered SoA, and (optionally) a captured CUDA graph of one slide.
// The slide pipeline reads all per-slide positions from a DevState block in
// device memory, so the same graph is replayed for every slide.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/rtod.h"
#include "kernels.cuh"

#define RTOD_API extern "C" __attribute__((visibility("default")))

using namespace rtod;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CU(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(RTOD_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                 \
  } while (0)

#define DISPATCH_D(D_, ...)                      \
  switch (D_) {                                  \
    case 1: { constexpr int D = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int D = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int D = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int D = 4; __VA_ARGS__; } break; \
    case 5: { constexpr int D = 5; __VA_ARGS__; } break; \
    case 6: { constexpr int D = 6; __VA_ARGS__; } break; \
    case 7: { constexpr int D = 7; __VA_ARGS__; } break; \
    case 8: { constexpr int D = 8; __VA_ARGS__; } break; \
    default: break;                              \
  }

#define DISPATCH_DP(D_, P_, ...)                                        \
  if ((P_) == 0) {                                                      \
    DISPATCH_D(D_, { constexpr int PRED = 0; __VA_ARGS__; });           \
  } else {                                                              \
    DISPATCH_D(D_, { constexpr int PRED = 1; __VA_ARGS__; });           \
  }

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
int dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  CU(cudaMalloc((void**)p, count * sizeof(T)));
  return RTOD_OK;
}

}  // namespace

struct rtod_handle {
  rtod_config cfg;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  KParams kp{};
  int32_t block_warps = 8;

  // device buffers owned by the handle
  float* ring = nullptr;
  uint64_t* ckey = nullptr;
  uint32_t* bin_count = nullptr;
  uint32_t* bin_start = nullptr;
  uint32_t* cursor = nullptr;
  uint64_t* owner = nullptr;
  uint8_t* mixed = nullptr;
  uint32_t* s_slot = nullptr;
  uint64_t* s_ckey = nullptr;
  float* s_x = nullptr;
  uint8_t* flags = nullptr;
  uint8_t* prev = nullptr;
  DevState* state = nullptr;
  float* staging = nullptr;   // W * D floats
  int64_t* ids = nullptr;     // result buffer
  int64_t ids_cap = 0;
  int32_t* slide_nout = nullptr;
  int32_t* slide_undet = nullptr;
  int64_t slide_rec_cap = 0;
  float* run_buf = nullptr;   // resident copy of a host stream (rtod_run)
  int64_t run_buf_cap = 0;    // floats

  // host mirror of the stream position
  int64_t n_pushed = 0;
  int64_t slides_done = 0;
  bool pending = false;
  bool poisoned = false;

  // slide graph (captured for a given src pointer and output buffers)
  cudaGraphExec_t graph = nullptr;
  KParams graph_kp{};  // kernel parameters baked into the graph

  cudaEvent_t ev[8] = {};
  int64_t launches = 0;       // kernels issued (graph replays count their kernels)
  int64_t graph_replays = 0;
  int64_t undet_total = 0;
  cudaEvent_t* kev = nullptr; // per-kernel events of a profiled run (7 per slide)
};

namespace {

int check_config(const rtod_config* c) {
  if (!c) return fail(RTOD_ERR_ARG, "config is null");
  if (c->window < 1 || c->slide < 1 || c->slide > c->window)
    return fail(RTOD_ERR_CONFIG, "need 1 <= slide <= window (got W=%lld S=%lld)",
                (long long)c->window, (long long)c->slide);
  if (c->window % c->slide != 0)
    return fail(RTOD_ERR_CONFIG, "window %% slide must be 0 (W=%lld S=%lld)", (long long)c->window,
                (long long)c->slide);
  if (c->window > (1ll << 31) - 64)
    return fail(RTOD_ERR_CONFIG, "window too large (max 2^31-64 points)");
  if (!(c->R >= 1e-18) || !(c->R <= 1e18) || !std::isfinite(c->R))
    return fail(RTOD_ERR_CONFIG, "R must be finite and in [1e-18, 1e18] (got %g)", c->R);
  if (c->K < 0) return fail(RTOD_ERR_CONFIG, "K must be >= 0");
  if (c->dim < 1 || c->dim > 8) return fail(RTOD_ERR_CONFIG, "dim must be in 1..8 (got %d)", c->dim);
  if (c->opt < 0 || c->opt > 2) return fail(RTOD_ERR_CONFIG, "opt must be 0, 1 or 2");
  if (c->pred != RTOD_PRED_FP32_LE && c->pred != RTOD_PRED_F64_LT)
    return fail(RTOD_ERR_CONFIG, "unknown predicate %d", c->pred);
  if (c->cells_per_r < 0 || c->cells_per_r > 3) return fail(RTOD_ERR_CONFIG, "cells_per_r must be 0..3");
  if (c->block_warps != 0 && c->block_warps != 1 && c->block_warps != 2 && c->block_warps != 4 &&
      c->block_warps != 8)
    return fail(RTOD_ERR_CONFIG, "block_warps must be 0 (auto), 1, 2, 4 or 8");
  return RTOD_OK;
}

// Derives the grid parameters from the configuration and the cells per R.
void set_grid(rtod_handle* h, int n) {
  KParams& k = h->kp;
  k.n = n;
  k.cell = h->cfg.R * (1.0 + std::ldexp(1.0, -12)) / (double)n;
  // A cell is provably all-inlier when it holds more than K points only if
  // its diagonal is below R: needs every dimension hashed and n >= 2.
  k.filter = (h->cfg.opt >= 1 && h->cfg.dim <= 3 && n >= 2) ? 1 : 0;
}

int launch_ingest(rtod_handle* h, int64_t n_new) {
  int64_t work = std::max<int64_t>(std::max<int64_t>(NB, h->kp.W), n_new);
  int blocks = (int)std::min<int64_t>((work + 255) / 256, (int64_t)h->sm_count * 8);
  DISPATCH_D(h->kp.D, (k_ingest<D><<<blocks, 256, 0, h->stream>>>(h->kp, n_new)));
  CU(cudaGetLastError());
  h->launches++;
  return RTOD_OK;
}

constexpr int kSlideKernels = 6;
const char* kKernelNames[kSlideKernels] = {"k_ingest", "k_hist", "k_scan", "k_scatter", "k_count",
                                           "k_compact"};

// Stages of one slide. ev (may be null) receives 3 timestamps: ev[1] after
// ingest+hist, ev[2] after scan+scatter, ev[3] after count+compact. kev (may
// be null) receives one timestamp after each of the six kernels.
int launch_slide(rtod_handle* h, cudaEvent_t* ev, cudaEvent_t* kev = nullptr) {
  const KParams& kp = h->kp;
  cudaStream_t st = h->stream;
  int r = launch_ingest(h, kp.S);
  if (r) return r;
  if (kev) CU(cudaEventRecord(kev[0], st));
  int wblocks = (int)std::min<int64_t>((kp.W + 255) / 256, (int64_t)h->sm_count * 16);
  DISPATCH_D(kp.D, (k_hist<Hashed<D>::value><<<wblocks, 256, 0, st>>>(kp)));
  if (kev) CU(cudaEventRecord(kev[1], st));
  if (ev) CU(cudaEventRecord(ev[1], st));
  k_scan<<<1, 1024, 0, st>>>(kp);
  if (kev) CU(cudaEventRecord(kev[2], st));
  DISPATCH_D(kp.D, (k_scatter<D><<<wblocks, 256, 0, st>>>(kp)));
  if (kev) CU(cudaEventRecord(kev[3], st));
  if (ev) CU(cudaEventRecord(ev[2], st));
  int64_t warps = (kp.W + 31) / 32;
  int wpb = h->block_warps;
  int cblocks = (int)((warps + wpb - 1) / wpb);
  DISPATCH_DP(kp.D, h->cfg.pred, (k_count<D, PRED><<<cblocks, wpb * 32, 0, st>>>(kp)));
  if (kev) CU(cudaEventRecord(kev[4], st));
  k_compact<<<1, 1024, 0, st>>>(kp);
  CU(cudaGetLastError());
  if (kev) CU(cudaEventRecord(kev[5], st));
  if (ev) CU(cudaEventRecord(ev[3], st));
  h->launches += kSlideKernels - 1;
  return RTOD_OK;
}

void drop_graph(rtod_handle* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
}

int ensure_graph(rtod_handle* h) {
  if (h->graph && std::memcmp(&h->graph_kp, &h->kp, sizeof(KParams)) == 0) return RTOD_OK;
  drop_graph(h);
  cudaGraph_t g;
  CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  const int64_t before = h->launches;
  int r = launch_slide(h, nullptr);
  h->launches = before;
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (r) return r;
  if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  h->graph_kp = h->kp;
  return RTOD_OK;
}

int run_slide(rtod_handle* h, cudaEvent_t* ev) {
  if (h->cfg.use_graph && !ev) {
    int r = ensure_graph(h);
    if (r) return r;
    CU(cudaGraphLaunch(h->graph, h->stream));
    h->launches += kSlideKernels;
    h->graph_replays++;
    return RTOD_OK;
  }
  return launch_slide(h, ev);
}

int check_device_error(rtod_handle* h, const DevState& s) {
  if (s.err == DERR_NONE) return RTOD_OK;
  h->poisoned = true;
  switch (s.err) {
    case DERR_NONFINITE: return fail(RTOD_ERR_INPUT, "non-finite coordinate in the stream");
    case DERR_RANGE:
      return fail(RTOD_ERR_INPUT, "coordinate too large for the grid (|x| / cell beyond the limit)");
    case DERR_CAPACITY: return fail(RTOD_ERR_CAPACITY, "outlier ID buffer too small");
    default: return fail(RTOD_ERR_CUDA, "device error %d", s.err);
  }
}

int reset_state(rtod_handle* h) {
  CU(cudaMemsetAsync(h->state, 0, sizeof(DevState), h->stream));
  h->n_pushed = 0;
  h->slides_done = 0;
  h->pending = false;
  h->poisoned = false;
  return RTOD_OK;
}

int ensure_ids(rtod_handle* h, int64_t cap) {
  if (cap <= h->ids_cap) return RTOD_OK;
  if (h->ids) cudaFree(h->ids);
  h->ids = nullptr;
  h->ids_cap = 0;
  if (dalloc(&h->ids, (size_t)cap)) return RTOD_ERR_CUDA;
  h->ids_cap = cap;
  h->kp.out_ids = h->ids;
  drop_graph(h);
  return RTOD_OK;
}

int ensure_slide_records(rtod_handle* h, int64_t n) {
  if (n <= h->slide_rec_cap) return RTOD_OK;
  if (h->slide_nout) cudaFree(h->slide_nout);
  if (h->slide_undet) cudaFree(h->slide_undet);
  h->slide_nout = h->slide_undet = nullptr;
  h->slide_rec_cap = 0;
  if (dalloc(&h->slide_nout, (size_t)n) || dalloc(&h->slide_undet, (size_t)n)) return RTOD_ERR_CUDA;
  h->slide_rec_cap = n;
  h->kp.slide_nout = h->slide_nout;
  h->kp.slide_undet = h->slide_undet;
  h->kp.slide_rec_cap = n;
  drop_graph(h);
  return RTOD_OK;
}

void free_all(rtod_handle* h) {
  drop_graph(h);
  void* bufs[] = {h->ring, h->ckey, h->bin_count, h->bin_start, h->cursor, h->owner, h->mixed,
                  h->s_slot, h->s_ckey, h->s_x, h->flags, h->prev, h->state, h->staging, h->ids,
                  h->slide_nout, h->slide_undet, h->run_buf};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

RTOD_API const char* rtod_version(void) { return "rtod-b200 0.1 (sm_100a)"; }

RTOD_API const char* rtod_last_error(void) { return g_last_error.c_str(); }

RTOD_API int rtod_config_init(rtod_config* c) {
  if (!c) return fail(RTOD_ERR_ARG, "config is null");
  std::memset(c, 0, sizeof *c);
  c->window = 100000;
  c->slide = 5000;
  c->R = 0.45;
  c->K = 50;
  c->dim = 1;
  c->opt = 2;
  c->pred = RTOD_PRED_FP32_LE;
  c->use_graph = 1;
  return RTOD_OK;
}

RTOD_API int rtod_create(const rtod_config* cfg, rtod_handle** out) {
  if (!out) return fail(RTOD_ERR_ARG, "out is null");
  *out = nullptr;
  int r = check_config(cfg);
  if (r) return r;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(RTOD_ERR_NODEV, "no CUDA device");
  }
  if (cfg->device < 0 || cfg->device >= ndev) return fail(RTOD_ERR_NODEV, "bad device ordinal %d", cfg->device);
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, cfg->device));
  if (prop.major != 10)
    return fail(RTOD_ERR_NODEV, "device %d is sm_%d%d; this library is built for sm_100a only",
                cfg->device, prop.major, prop.minor);
  CU(cudaSetDevice(cfg->device));

  rtod_handle* h = new (std::nothrow) rtod_handle();
  if (!h) return fail(RTOD_ERR_ARG, "out of host memory");
  h->cfg = *cfg;
  h->device = cfg->device;
  h->sm_count = prop.multiProcessorCount;
  h->block_warps = cfg->block_warps ? cfg->block_warps : 8;

  const int64_t W = cfg->window, S = cfg->slide;
  const int D = cfg->dim;
  KParams& k = h->kp;
  k.W = W;
  k.S = S;
  k.D = D;
  k.h = D < 3 ? D : 3;
  k.K = cfg->K;
  k.R = cfg->R;
  k.R2 = cfg->R * cfg->R;
  {
    volatile float rf = (float)cfg->R;
    volatile float r2f = rf * rf;
    k.R2f = r2f;
  }
  set_grid(h, cfg->cells_per_r ? cfg->cells_per_r : 2);

  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && !dalloc(&h->ring, (size_t)(W * D)) && !dalloc(&h->ckey, (size_t)W) &&
       !dalloc(&h->bin_count, NB) && !dalloc(&h->bin_start, NB + 1) && !dalloc(&h->cursor, NB) &&
       !dalloc(&h->owner, NB) && !dalloc(&h->mixed, NB) && !dalloc(&h->s_slot, (size_t)W) &&
       !dalloc(&h->s_ckey, (size_t)W) && !dalloc(&h->s_x, (size_t)(W * D)) &&
       !dalloc(&h->flags, (size_t)W) && !dalloc(&h->prev, (size_t)W) && !dalloc(&h->state, 1) &&
       !dalloc(&h->staging, (size_t)(W * D));
  for (auto& e : h->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
  if (!ok) {
    std::string msg = g_last_error.empty() ? "device allocation failed" : g_last_error;
    free_all(h);
    delete h;
    return fail(RTOD_ERR_CUDA, "%s", msg.c_str());
  }
  k.ring = h->ring;
  k.ckey = h->ckey;
  k.bin_count = h->bin_count;
  k.bin_start = h->bin_start;
  k.cursor = h->cursor;
  k.owner = h->owner;
  k.mixed = h->mixed;
  k.s_slot = h->s_slot;
  k.s_ckey = h->s_ckey;
  k.s_x = h->s_x;
  k.flags = h->flags;
  k.prev = h->prev;
  k.state = h->state;
  k.src = h->staging;
  k.src_staging = 1;
  r = ensure_ids(h, W);
  if (!r) r = reset_state(h);
  if (!r && cudaStreamSynchronize(h->stream) != cudaSuccess) r = fail(RTOD_ERR_CUDA, "init sync failed");
  if (r) {
    free_all(h);
    delete h;
    return r;
  }
  *out = h;
  return RTOD_OK;
}

RTOD_API void rtod_destroy(rtod_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
}

RTOD_API int rtod_reset(rtod_handle* h) {
  if (!h) return fail(RTOD_ERR_ARG, "handle is null");
  CU(cudaSetDevice(h->device));
  int r = reset_state(h);
  if (r) return r;
  CU(cudaStreamSynchronize(h->stream));
  return RTOD_OK;
}

RTOD_API int64_t rtod_slides_done(const rtod_handle* h) { return h ? h->slides_done : -1; }

RTOD_API int rtod_get_tuning(const rtod_handle* h, int32_t out[3]) {
  if (!h || !out) return fail(RTOD_ERR_ARG, "null argument");
  out[0] = h->kp.n;
  out[1] = h->block_warps;
  out[2] = h->kp.h;
  return RTOD_OK;
}

RTOD_API int rtod_push_slide(rtod_handle* h, const float* pts, int64_t n) {
  if (!h || !pts) return fail(RTOD_ERR_ARG, "null argument");
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  CU(cudaSetDevice(h->device));
  const int64_t W = h->kp.W, S = h->kp.S, D = h->kp.D;
  if (h->n_pushed == 0) {
    if (n != W) return fail(RTOD_ERR_STATE, "the first push must hold exactly W=%lld points", (long long)W);
  } else {
    if (h->pending) return fail(RTOD_ERR_STATE, "rtod_detect must follow each slide push");
    if (n != S) return fail(RTOD_ERR_STATE, "a slide push must hold exactly S=%lld points", (long long)S);
  }
  CU(cudaEventRecord(h->ev[4], h->stream));
  CU(cudaMemcpyAsync(h->staging, pts, (size_t)(n * D) * sizeof(float), cudaMemcpyDefault, h->stream));
  CU(cudaEventRecord(h->ev[5], h->stream));
  h->kp.src = h->staging;
  h->kp.src_staging = 1;
  if (h->n_pushed == 0) {
    int r = launch_ingest(h, W);
    if (r) return r;
    k_advance<<<1, 32, 0, h->stream>>>(h->state, W);
    CU(cudaGetLastError());
    h->launches++;
    DevState s;
    CU(cudaMemcpyAsync(&s, h->state, sizeof s, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    r = check_device_error(h, s);
    if (r) return r;
  } else {
    h->pending = true;
  }
  h->n_pushed += n;
  return RTOD_OK;
}

RTOD_API int rtod_detect(rtod_handle* h, int64_t* out_ids, int64_t cap, int64_t* n_out, rtod_times* times) {
  if (!h || !n_out || (cap > 0 && !out_ids)) return fail(RTOD_ERR_ARG, "null argument");
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  if (!h->pending) return fail(RTOD_ERR_STATE, "no pushed slide to detect");
  CU(cudaSetDevice(h->device));
  // Per-call output: results start at the beginning of the ID buffer.
  CU(cudaMemsetAsync(&h->state->out_total, 0, sizeof(int64_t), h->stream));
  h->kp.out_cap = h->ids_cap;
  cudaEvent_t* ev = times ? h->ev : nullptr;
  if (ev) CU(cudaEventRecord(ev[0], h->stream));
  int r = run_slide(h, ev);
  if (r) return r;
  DevState s;
  CU(cudaMemcpyAsync(&s, h->state, sizeof s, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->pending = false;
  r = check_device_error(h, s);
  if (r) return r;
  h->slides_done++;
  h->undet_total += s.n_undet;
  *n_out = s.n_out;
  if (s.n_out > cap) return fail(RTOD_ERR_CAPACITY, "%d outliers but room for %lld", s.n_out, (long long)cap);
  if (ev) CU(cudaEventRecord(ev[6], h->stream));
  if (s.n_out > 0)
    CU(cudaMemcpyAsync(out_ids, h->ids, (size_t)s.n_out * sizeof(int64_t), cudaMemcpyDefault, h->stream));
  if (ev) CU(cudaEventRecord(ev[7], h->stream));
  CU(cudaStreamSynchronize(h->stream));
  if (times) {
    std::memset(times, 0, sizeof *times);
    times->copy_new_points_h2d = elapsed(h->ev[4], h->ev[5]);
    times->prepare_cell = elapsed(h->ev[0], h->ev[1]);
    times->build_bvh = elapsed(h->ev[1], h->ev[2]);
    times->detect_outlier = elapsed(h->ev[2], h->ev[3]);
    times->copy_outlier_d2h = elapsed(h->ev[6], h->ev[7]);
    times->total = times->copy_new_points_h2d + elapsed(h->ev[0], h->ev[3]) + times->copy_outlier_d2h;
    times->undetermined_per_slide = s.n_undet;
    times->slides = 1;
  }
  return RTOD_OK;
}

RTOD_API int rtod_run(rtod_handle* h, const float* pts, int64_t n, int64_t max_slides, int64_t* out_offsets,
                      int64_t* out_ids, int64_t ids_cap, int64_t* slides_out, rtod_times* times) {
  if (!h || !pts || !out_offsets || !slides_out || (ids_cap > 0 && !out_ids))
    return fail(RTOD_ERR_ARG, "null argument");
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  if (h->n_pushed != 0) return fail(RTOD_ERR_STATE, "rtod_run needs a fresh handle (call rtod_reset)");
  if (n < 0 || ids_cap < 0) return fail(RTOD_ERR_ARG, "negative size");
  CU(cudaSetDevice(h->device));
  const int64_t W = h->kp.W, S = h->kp.S, D = h->kp.D;
  int64_t slides = n >= W ? (n - W) / S : 0;
  if (max_slides >= 0) slides = std::min(slides, max_slides);
  *slides_out = slides;
  out_offsets[0] = 0;
  if (slides == 0) return RTOD_OK;
  const int64_t used = W + slides * S;
  int r;
  // Device input.
  cudaEvent_t t0, t1, t2, t3;
  bool timing = times != nullptr;
  std::vector<cudaEvent_t> evs;
  auto mk = [&](cudaEvent_t* e) { cudaEventCreate(e); evs.push_back(*e); };
  mk(&t0); mk(&t1); mk(&t2); mk(&t3);
  struct Cleanup {
    std::vector<cudaEvent_t>& e;
    ~Cleanup() { for (auto x : e) cudaEventDestroy(x); }
  } cleanup{evs};
  CU(cudaEventRecord(t0, h->stream));
  const float* src = pts;
  if (!is_device_ptr(pts)) {
    if (h->run_buf_cap < used * D) {
      if (h->run_buf) cudaFree(h->run_buf);
      h->run_buf = nullptr;
      h->run_buf_cap = 0;
      if (dalloc(&h->run_buf, (size_t)(used * D))) return RTOD_ERR_CUDA;
      h->run_buf_cap = used * D;
    }
    CU(cudaMemcpyAsync(h->run_buf, pts, (size_t)(used * D) * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    src = h->run_buf;
  }
  CU(cudaEventRecord(t1, h->stream));
  if ((r = ensure_ids(h, std::max<int64_t>(1, std::min(ids_cap, slides * W))))) return r;
  if ((r = ensure_slide_records(h, slides))) return r;
  h->kp.out_cap = std::min(ids_cap, h->ids_cap);
  h->kp.src = src;
  h->kp.src_staging = 0;
  if ((r = reset_state(h))) return r;
  if ((r = launch_ingest(h, W))) return r;
  k_advance<<<1, 32, 0, h->stream>>>(h->state, W);
  CU(cudaGetLastError());
  h->launches++;
  h->n_pushed = W;
  // Per-stage events only when a breakdown is requested without graphs.
  const bool stage = timing && !h->cfg.use_graph;
  std::vector<cudaEvent_t> sev;
  if (stage) {
    sev.resize((size_t)slides * 4);
    for (auto& e : sev) mk(&e);
  }
  CU(cudaEventRecord(t2, h->stream));
  for (int64_t j = 0; j < slides; ++j) {
    if (stage) {
      CU(cudaEventRecord(sev[j * 4], h->stream));
      r = launch_slide(h, &sev[j * 4]);
    } else {
      r = run_slide(h, nullptr);
    }
    if (r) return r;
  }
  CU(cudaEventRecord(t3, h->stream));
  DevState s;
  std::vector<int32_t> nout((size_t)slides), nund((size_t)slides);
  CU(cudaMemcpyAsync(&s, h->state, sizeof s, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaMemcpyAsync(nout.data(), h->slide_nout, slides * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaMemcpyAsync(nund.data(), h->slide_undet, slides * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->n_pushed = used;
  h->slides_done = slides;
  if ((r = check_device_error(h, s))) return r;
  h->undet_total += s.undet_total;
  for (int64_t j = 0; j < slides; ++j) out_offsets[j + 1] = out_offsets[j] + nout[j];
  if (out_offsets[slides] != s.out_total) return fail(RTOD_ERR_CUDA, "inconsistent outlier totals");
  cudaEvent_t d0, d1;
  mk(&d0); mk(&d1);
  CU(cudaEventRecord(d0, h->stream));
  if (s.out_total > 0)
    CU(cudaMemcpyAsync(out_ids, h->ids, (size_t)s.out_total * sizeof(int64_t), cudaMemcpyDefault, h->stream));
  CU(cudaEventRecord(d1, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  if (times) {
    std::memset(times, 0, sizeof *times);
    const double inv = 1.0 / (double)slides;
    times->slides = slides;
    times->copy_new_points_h2d = elapsed(t0, t1) * inv;
    times->copy_outlier_d2h = elapsed(d0, d1) * inv;
    if (stage) {
      double pc = 0, bb = 0, de = 0;
      for (int64_t j = 0; j < slides; ++j) {
        pc += elapsed(sev[j * 4], sev[j * 4 + 1]);
        bb += elapsed(sev[j * 4 + 1], sev[j * 4 + 2]);
        de += elapsed(sev[j * 4 + 2], sev[j * 4 + 3]);
      }
      times->prepare_cell = pc * inv;
      times->build_bvh = bb * inv;
      times->detect_outlier = de * inv;
    }
    // Everything on the library stream: input copy, state reset, initial
    // fill, all slides and the outlier copy-out (the counts read-back and
    // its host wait are the only parts outside).
    times->total = (elapsed(t0, t3) + elapsed(d0, d1)) * inv;
    times->undetermined_per_slide = (double)s.undet_total * inv;
  }
  return RTOD_OK;
}

RTOD_API int rtod_get_stats(const rtod_handle* h, int64_t out[4]) {
  if (!h || !out) return fail(RTOD_ERR_ARG, "null argument");
  out[0] = h->launches;
  out[1] = h->graph_replays;
  out[2] = h->slides_done;
  out[3] = h->undet_total;
  return RTOD_OK;
}

RTOD_API const char* rtod_kernel_name(int32_t i) {
  return (i >= 0 && i < kSlideKernels) ? kKernelNames[i] : nullptr;
}

RTOD_API int rtod_profile_run(rtod_handle* h, const float* pts, int64_t n, int64_t max_slides,
                              double* kernel_ms, int32_t n_kernels) {
  if (!h || !pts || !kernel_ms || n_kernels < 1) return fail(RTOD_ERR_ARG, "null argument");
  if (h->n_pushed != 0) return fail(RTOD_ERR_STATE, "rtod_profile_run needs a fresh handle");
  CU(cudaSetDevice(h->device));
  const int64_t W = h->kp.W, S = h->kp.S, D = h->kp.D;
  int64_t slides = n >= W ? (n - W) / S : 0;
  if (max_slides >= 0) slides = std::min(slides, max_slides);
  if (slides == 0) return fail(RTOD_ERR_ARG, "stream shorter than one slide");
  const int64_t used = W + slides * S;
  const float* src = pts;
  int r;
  if (!is_device_ptr(pts)) {
    if (h->run_buf_cap < used * D) {
      if (h->run_buf) cudaFree(h->run_buf);
      h->run_buf = nullptr;
      h->run_buf_cap = 0;
      if (dalloc(&h->run_buf, (size_t)(used * D))) return RTOD_ERR_CUDA;
      h->run_buf_cap = used * D;
    }
    CU(cudaMemcpyAsync(h->run_buf, pts, (size_t)(used * D) * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    src = h->run_buf;
  }
  if ((r = ensure_ids(h, std::max<int64_t>(1, slides * W)))) return r;
  if ((r = ensure_slide_records(h, slides))) return r;
  h->kp.out_cap = h->ids_cap;
  h->kp.src = src;
  h->kp.src_staging = 0;
  if ((r = reset_state(h))) return r;
  if ((r = launch_ingest(h, W))) return r;
  k_advance<<<1, 32, 0, h->stream>>>(h->state, W);
  CU(cudaGetLastError());
  h->launches++;
  std::vector<cudaEvent_t> ev((size_t)slides * (kSlideKernels + 1));
  for (auto& e : ev) CU(cudaEventCreate(&e));
  struct Cleanup {
    std::vector<cudaEvent_t>& e;
    ~Cleanup() { for (auto x : e) cudaEventDestroy(x); }
  } cleanup{ev};
  for (int64_t j = 0; j < slides; ++j) {
    cudaEvent_t* e = &ev[(size_t)j * (kSlideKernels + 1)];
    CU(cudaEventRecord(e[0], h->stream));
    if ((r = launch_slide(h, nullptr, e + 1))) return r;
  }
  DevState s;
  CU(cudaMemcpyAsync(&s, h->state, sizeof s, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->n_pushed = used;
  h->slides_done = slides;
  if ((r = check_device_error(h, s))) return r;
  h->undet_total += s.undet_total;
  for (int i = 0; i < n_kernels; ++i) kernel_ms[i] = 0;
  for (int64_t j = 0; j < slides; ++j) {
    cudaEvent_t* e = &ev[(size_t)j * (kSlideKernels + 1)];
    for (int i = 0; i < kSlideKernels && i < n_kernels; ++i) kernel_ms[i] += elapsed(e[i], e[i + 1]);
  }
  for (int i = 0; i < n_kernels; ++i) kernel_ms[i] /= (double)slides;
  return RTOD_OK;
}
