// Host engine and C ABI of the detector (include/rtod.h).
//
// One rtod_handle = one stream. It owns a CUDA stream, a pool of per-window
// scratch buffers (one per job of a batch), the ring used by push/detect,
// the resident copy of a stream used by rtod_run, and captured CUDA graphs
// of a batch. All per-window positions live on the device (JobCtr), so a
// captured batch is replayed unchanged.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <cstddef>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/rtod.h"
#include "fused.cuh"
#include "grid.cuh"
#include "kernels.cuh"
#include "span.cuh"

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

#define CU(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(RTOD_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                   \
  } while (0)

#define DISPATCH_D(D_, ...)                              \
  switch (D_) {                                          \
    case 1: { constexpr int D = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int D = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int D = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int D = 4; __VA_ARGS__; } break; \
    case 5: { constexpr int D = 5; __VA_ARGS__; } break; \
    case 6: { constexpr int D = 6; __VA_ARGS__; } break; \
    case 7: { constexpr int D = 7; __VA_ARGS__; } break; \
    case 8: { constexpr int D = 8; __VA_ARGS__; } break; \
    default: break;                                      \
  }

#define DISPATCH_DP(D_, P_, ...)                              \
  if ((P_) == 0) {                                            \
    DISPATCH_D(D_, { constexpr int PRED = 0; __VA_ARGS__; }); \
  } else {                                                    \
    DISPATCH_D(D_, { constexpr int PRED = 1; __VA_ARGS__; }); \
  }

// Dimension x coordinate type (T = float, or double for a handle storing
// double coordinates).
#define DISPATCH_DT(F64_, D_, ...)                        \
  if (F64_) {                                             \
    DISPATCH_D(D_, { using T = double; __VA_ARGS__; });   \
  } else {                                                \
    DISPATCH_D(D_, { using T = float; __VA_ARGS__; });    \
  }

// Dimension x predicate x coordinate type: double coordinates always use
// RTOD's double predicate.
#define DISPATCH_DPT(F64_, D_, P_, ...)                                           \
  if (F64_) {                                                                     \
    DISPATCH_D(D_, { constexpr int PRED = 1; using T = double; __VA_ARGS__; });   \
  } else {                                                                        \
    DISPATCH_DP(D_, P_, { using T = float; __VA_ARGS__; });                       \
  }

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Whether kernels on `device` can read and write p directly: memory of that
// device, managed memory, or pinned (page-locked) host memory.
bool device_addressable(const void* p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged || a.type == cudaMemoryTypeHost) return true;
  return a.type == cudaMemoryTypeDevice && a.device == device;
}

// Pinned (page-locked) host memory.
bool pinned_host_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

template <typename T>
int dalloc(T** p, size_t count, int64_t* counter) {
  *p = nullptr;
  if (count == 0) count = 1;
  CU(cudaMalloc((void**)p, count * sizeof(T)));
  *counter += (int64_t)(count * sizeof(T));
  return RTOD_OK;
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// Launches a kernel with programmatic dependent launch allowed, so that its
// blocks can be scheduled while the previous kernel in the stream finishes;
// every kernel waits (griddepcontrol.wait) before reading its inputs.
template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, int block, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// Scratch of one job (one window in flight) of the window engine, allocated
// when that engine first runs the job (the span engine uses none of it).
struct Scratch {
  bool full = false;
  uint32_t* bin_count = nullptr;
  uint32_t* bin_start = nullptr;
  unsigned long long* kmin = nullptr;
  unsigned long long* kmax = nullptr;
  uint32_t* s_off = nullptr;
  uint64_t* s_ckey = nullptr;
  unsigned char* s_x = nullptr;  // coordinates, the handle's type
  uint32_t* queue = nullptr;
  float* feat = nullptr;
  uint32_t* flags = nullptr;
  unsigned long long* scan_status = nullptr;
  unsigned long long* cmp_status = nullptr;
};

// Scratch of the span engine (one per handle): sized for spans of up to
// nblk_cap slide blocks and pts_cap points.
struct SpanScratch {
  uint32_t* bin_count = nullptr;
  uint32_t* bin_start = nullptr;
  unsigned long long* kmin = nullptr;
  unsigned long long* kmax = nullptr;
  uint32_t* cnt = nullptr;  // [NB][ts]
  uint32_t* pre = nullptr;  // [NB][ts]
  int64_t ts = 0;           // nblk_cap + 1
  uint32_t* used = nullptr;
  uint32_t* s_off = nullptr;
  unsigned char* s_x = nullptr;  // coordinates, the handle's type
  unsigned long long* scan_status = nullptr;
  SpanCtr* sc = nullptr;
  uint4* groups = nullptr;    // [windows][min(W, NB)] listed groups of a batch
  uint32_t* bits = nullptr;   // [chunk][words] per-slide outlier bitsets
  int64_t nblk_cap = 0;
  int64_t pts_cap = 0;
  int64_t chunk_cap = 0;
  int64_t Wp = 0;
  int64_t gcap = 0;  // entries of groups
  int64_t bytes = 0;
};

constexpr int kMaxJobs = 256;  // windows per launch, either engine
static_assert(kMaxJobs <= BATCH_JOBS_MAX, "the batch-wide count list holds one prefix entry per job");

constexpr int kPipeKernels = 7;
const char* kKernelNames[kPipeKernels] = {"k_keys",  "k_hist",    "k_scan", "k_scatter",
                                          "k_count", "k_compact", "k_train"};

// Initial router parameters: uniform(-a, a) with a = sqrt(6 / (fan_in + fan_out))
// (Glorot & Bengio 2010) from a fixed-seed xorshift generator, zero biases
// except a prior towards bucket 3 (most counted points are inliers).
void init_router(RouterState* r) {
  std::memset(r, 0, sizeof(RouterState));
  uint64_t st = 0x9e3779b97f4a7c15ull;
  auto uni = [&](float a) {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return (float)((double)(st >> 11) / 9007199254740992.0 * 2.0 - 1.0) * a;
  };
  const float a1 = std::sqrt(6.0f / (MLP_IN + MLP_H)), a2 = std::sqrt(6.0f / (MLP_H + MLP_H)),
              a3 = std::sqrt(6.0f / (MLP_H + MLP_B));
  for (int i = 0; i < MLP_H * MLP_IN; ++i) r->params[OFF_W1 + i] = uni(a1);
  for (int i = 0; i < MLP_H * MLP_H; ++i) r->params[OFF_W2 + i] = uni(a2);
  for (int i = 0; i < MLP_B * MLP_H; ++i) r->params[OFF_W3 + i] = uni(a3);
  r->params[OFF_B3 + 3] = 2.0f;
  r->b1t = r->b2t = 1.0f;
  r->lr = 3e-3f;
  r->beta1 = 0.9f;
  r->beta2 = 0.999f;
  r->eps = 1e-8f;
  r->threshold = 0.5f;
  r->max_sweep = 64;
  r->min_samples = (uint32_t)TRAIN_MAX;
}

enum Mode { MODE_NONE = 0, MODE_RING = 1, MODE_RUN = 2 };

// Streaming grid engine of push/detect (grid.cuh): its device arrays and
// the kernel argument that points at them.
struct GridHost {
  bool on = false;     // push/detect run the grid engine
  bool built = false;  // the grid holds the ring's window
  Grid g{};
  int64_t bytes = 0;
  int64_t builds = 0;  // builds from the ring (first window and rebuilds)
  uint64_t pool_first = 0;  // pool slots of the first build (0: 16 W + 2^21)
};

struct EventSet {
  std::vector<cudaEvent_t> ev;
  cudaEvent_t make() {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    ev.push_back(e);
    return e;
  }
  ~EventSet() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

}  // namespace

struct rtod_handle {
  rtod_config cfg{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  int64_t W = 0, S = 0, Wp = 0;
  int D = 1;
  int n = 2;
  int filter = 1;
  double cell = 0;
  float R2f = 0;
  int block_warps = 8;
  int batch_max = 32;       // windows per launch of the window engine
  int span_batch_max = 256; // windows per launch of the span engine
  int64_t device_bytes = 0;

  std::vector<Scratch> pool;  // allocated lazily, one per job of a batch
  SpanScratch span;           // span engine scratch, allocated on first use
  int engine = RTOD_ENGINE_WINDOW;  // engine of rtod_run (resolved from the config / tuner)
  int group = 0;                    // window-engine count: 1 = group counts (resolved from the config / tuner)
  JobCtr* ctr = nullptr;      // [kMaxJobs]
  JobCtr* ctr_init = nullptr; // pinned host [kMaxJobs]
  Job* jobs_dev = nullptr;    // [kMaxJobs]
  std::vector<Job> tab_host;  // last uploaded job table
  BatchState* bs = nullptr;
  RouterState* router = nullptr;

  int f64 = 0;   // coordinates stored as double (RTOD_COORD_F64)
  int esz = 4;   // bytes per coordinate
  unsigned char* ring = nullptr;  // SoA [D][W] coordinates
  uint64_t* ring_keys = nullptr;
  uint8_t* ring_prev = nullptr;
  unsigned char* staging = nullptr;  // W * D coordinates

  unsigned char* run_buf = nullptr;
  int64_t run_buf_cap = 0;  // coordinates
  uint64_t* run_keys = nullptr;
  uint8_t* run_prev = nullptr;
  int64_t run_key_cap = 0;
  long long* run_blk_lo = nullptr;  // per slide block: cell coordinate range [blocks][3]
  long long* run_blk_hi = nullptr;
  int64_t run_blk_cap = 0;
  // Per-slide outlier and counted-point records of rtod_run, in mapped
  // page-locked memory (written by the kernels, read by the host after the
  // pass): device views rec_nout / rec_undet, host views *_h.
  void* rec_host = nullptr;
  int32_t* rec_nout = nullptr;
  int32_t* rec_undet = nullptr;
  int32_t* rec_nout_h = nullptr;
  int32_t* rec_undet_h = nullptr;
  int64_t* rec_base = nullptr;  // per-slide output offsets (span engine), device
  int64_t rec_cap = 0;
  BatchState* bs_mirror = nullptr;      // mapped page-locked copy of bs written by k_run_out
  BatchState* bs_mirror_dev = nullptr;  // its device view
  // Streaming (push/detect): a page-locked copy of the caller's slide, and
  // the mapped landing buffer of one window's IDs written by k_run_out.
  void* stage_host = nullptr;
  void* slide_host = nullptr;      // mapped page-locked slide of a streaming push from host memory
  void* slide_host_dev = nullptr;  // its device address, which the ingest kernels read in place
  int64_t* ids_host = nullptr;
  int64_t* ids_host_dev = nullptr;
  int64_t ids_host_cap = 0;
  int64_t* ids = nullptr;
  int64_t ids_cap = 0;

  int mode = MODE_NONE;
  int64_t n_pushed = 0;
  int64_t slides_done = 0;
  bool pending = false;
  bool poisoned = false;
  bool launched = false;   // the pending slide's detection is already on the stream (eager push)
  bool eager = false;      // slide pushes launch their detection (the last rtod_detect asked for no times)

  cudaGraphExec_t graphs[2] = {nullptr, nullptr};  // without / with the router's training step
  int64_t graph_kernels[2] = {0, 0};
  Batch graph_batch{};
  Span graph_span{};
  bool graph_is_span = false;
  // A whole rtod_run of a device-resident stream with the span engine, as one
  // graph (memsets, counter upload, keys, batches, compaction), replayed while
  // its key (stream, slides, batch and span parameters) stays the same.
  cudaGraphExec_t run_graph[2] = {nullptr, nullptr};  // without / with the router's training step
  std::vector<unsigned char> run_graph_key[2];
  int64_t run_graph_kernels[2] = {0, 0};
  int graph_ring = -1;
  int64_t batches = 0;

  GridHost grid;           // streaming grid engine (push/detect)
  GridBar* bar = nullptr;  // grid barrier of the fused pipeline
  int fused_grid = 0;      // its blocks (all resident), found on first use
  cudaEvent_t ev[16] = {};
  cudaStream_t copy_stream = nullptr;     // host-stream pieces, overlapped with detection
  cudaEvent_t fork_ev = nullptr;          // the copy stream's start on the library stream
  std::vector<cudaEvent_t> piece_ev;      // one per piece
  int64_t launches = 0;
  int64_t graph_replays = 0;
  int64_t undet_total = 0;
  bool tuned = false;
  double flush_ms = 0;  // device ms of the span engine's deferred compaction in the last profiled run
  float threshold = 0.5f;
  uint32_t max_sweep = 64;
  int span_route = 1;  // with the router on: the span engine routes its counts (the tuner may turn it off)
  bool tuning_pass = false;  // the tuner's timed passes train nothing (it trains between them)
};

namespace {

int check_config(const rtod_config* c) {
  if (!c) return fail(RTOD_ERR_ARG, "config is null");
  if (c->window < 1 || c->slide < 1 || c->slide > c->window)
    return fail(RTOD_ERR_CONFIG, "need 1 <= slide <= window (got W=%lld S=%lld)", (long long)c->window,
                (long long)c->slide);
  if (c->window % c->slide != 0)
    return fail(RTOD_ERR_CONFIG, "window %% slide must be 0 (W=%lld S=%lld)", (long long)c->window,
                (long long)c->slide);
  if (c->window > (1ll << 31) - 64) return fail(RTOD_ERR_CONFIG, "window too large (max 2^31-64 points)");
  if (!(c->R >= 1e-18) || !(c->R <= 1e18) || !std::isfinite(c->R))
    return fail(RTOD_ERR_CONFIG, "R must be finite and in [1e-18, 1e18] (got %g)", c->R);
  if (c->K < 0) return fail(RTOD_ERR_CONFIG, "K must be >= 0");
  if (c->dim < 1 || c->dim > 8) return fail(RTOD_ERR_CONFIG, "dim must be in 1..8 (got %d)", c->dim);
  if (c->opt < 0 || c->opt > 2) return fail(RTOD_ERR_CONFIG, "opt must be 0, 1 or 2");
  if (c->pred != RTOD_PRED_FP32_LE && c->pred != RTOD_PRED_F64_LT)
    return fail(RTOD_ERR_CONFIG, "unknown predicate %d", c->pred);
  if (c->cells_per_r < 0 || c->cells_per_r > (c->dim == 1 ? 8 : 3))
    return fail(RTOD_ERR_CONFIG, "cells_per_r must be 0..3 (0..8 in 1-d)");
  if (c->block_warps != 0 && c->block_warps != 1 && c->block_warps != 2 && c->block_warps != 4 &&
      c->block_warps != 8)
    return fail(RTOD_ERR_CONFIG, "block_warps must be 0 (auto), 1, 2, 4 or 8");
  if (c->batch < 0 || c->batch > 256) return fail(RTOD_ERR_CONFIG, "batch must be 0..256");
  if (c->engine < RTOD_ENGINE_AUTO || c->engine > RTOD_ENGINE_GRID)
    return fail(RTOD_ERR_CONFIG, "engine must be 0 (auto), 1 (window), 2 (span) or 3 (grid)");
  if (c->coord != RTOD_COORD_F32 && c->coord != RTOD_COORD_F64)
    return fail(RTOD_ERR_CONFIG, "coord must be RTOD_COORD_F32 or RTOD_COORD_F64");
  if (c->coord == RTOD_COORD_F64 && c->pred != RTOD_PRED_F64_LT)
    return fail(RTOD_ERR_CONFIG, "double coordinates need the double predicate (RTOD_PRED_F64_LT)");
  if (c->count < RTOD_COUNT_AUTO || c->count > RTOD_COUNT_GROUP)
    return fail(RTOD_ERR_CONFIG, "count must be 0 (auto), 1 (point) or 2 (group)");
  if (c->pipeline != RTOD_PIPELINE_FUSED && c->pipeline != RTOD_PIPELINE_STAGED)
    return fail(RTOD_ERR_CONFIG, "pipeline must be RTOD_PIPELINE_FUSED or RTOD_PIPELINE_STAGED");
  return RTOD_OK;
}

void set_grid(rtod_handle* h, int n) {
  h->n = n;
  h->cell = h->cfg.R * (1.0 + std::ldexp(1.0, -12)) / (double)n;
  // A cell is provably all-inlier when it holds more than K points only if
  // its diagonal is below R: needs every dimension hashed and n >= 2.
  h->filter = (h->cfg.opt >= 1 && h->cfg.dim <= 3 && n >= 2) ? 1 : 0;
}

void drop_graph(rtod_handle* h) {
  for (auto& g : h->graphs) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  h->graph_ring = -1;
  for (auto& rg : h->run_graph) {
    if (rg) cudaGraphExecDestroy(rg);
    rg = nullptr;
  }
}

// Pool entries for `jobs` jobs; with `full`, their window-engine scratch.
int ensure_pool(rtod_handle* h, int jobs, bool full = true) {
  const int64_t W = h->W, Wp = h->Wp, D = h->D;
  const int64_t cmp_tiles = (W + CMP_TILE - 1) / CMP_TILE;
  int64_t* c = &h->device_bytes;
  while ((int)h->pool.size() < jobs) h->pool.push_back(Scratch{});
  for (int j = 0; j < jobs && full; ++j) {
    Scratch& s = h->pool[j];
    if (s.full) continue;
    bool ok = !dalloc(&s.bin_count, NB, c) && !dalloc(&s.bin_start, NB + 1, c) && !dalloc(&s.kmin, NB, c) &&
              !dalloc(&s.kmax, NB, c) && !dalloc(&s.s_off, (size_t)W, c) && !dalloc(&s.s_ckey, (size_t)W, c) &&
              !dalloc(&s.s_x, (size_t)(Wp * D * h->esz), c) && !dalloc(&s.queue, (size_t)W, c) &&
              !dalloc(&s.feat, (size_t)(h->cfg.router ? W * MLP_IN : 1), c) &&
              !dalloc(&s.flags, (size_t)((W + 31) / 32), c) && !dalloc(&s.scan_status, SCAN_TILES, c) &&
              !dalloc(&s.cmp_status, (size_t)cmp_tiles, c);
    if (!ok) return RTOD_ERR_CUDA;
    s.full = true;
    drop_graph(h);
    CU(cudaMemset(s.bin_count, 0, NB * sizeof(uint32_t)));
    CU(cudaMemset(s.kmin, 0xff, NB * sizeof(unsigned long long)));
    CU(cudaMemset(s.kmax, 0, NB * sizeof(unsigned long long)));
    CU(cudaMemset(s.s_x, 0, (size_t)(Wp * D * h->esz)));
    CU(cudaMemset(s.flags, 0, (size_t)((W + 31) / 32) * sizeof(uint32_t)));
    CU(cudaMemset(s.scan_status, 0, SCAN_TILES * sizeof(unsigned long long)));
    CU(cudaMemset(s.cmp_status, 0, (size_t)cmp_tiles * sizeof(unsigned long long)));
  }
  return RTOD_OK;
}

// Clears all scratch and counters (after an error may have left a batch
// unfinished, and on reset).
int scrub(rtod_handle* h) {
  const int64_t W = h->W;
  const int64_t cmp_tiles = (W + CMP_TILE - 1) / CMP_TILE;
  for (Scratch& s : h->pool) {
    if (!s.full) continue;
    CU(cudaMemsetAsync(s.bin_count, 0, NB * sizeof(uint32_t), h->stream));
    CU(cudaMemsetAsync(s.kmin, 0xff, NB * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(s.kmax, 0, NB * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(s.flags, 0, (size_t)((W + 31) / 32) * sizeof(uint32_t), h->stream));
    CU(cudaMemsetAsync(s.scan_status, 0, SCAN_TILES * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(s.cmp_status, 0, (size_t)cmp_tiles * sizeof(unsigned long long), h->stream));
  }
  if (h->span.sc) {
    SpanScratch& sp = h->span;
    CU(cudaMemsetAsync(sp.bin_count, 0, NB * sizeof(uint32_t), h->stream));
    CU(cudaMemsetAsync(sp.kmin, 0xff, NB * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(sp.kmax, 0, NB * sizeof(unsigned long long), h->stream));
    CU(cudaMemsetAsync(sp.cnt, 0, (size_t)(sp.ts * NB) * sizeof(uint32_t), h->stream));
    CU(cudaMemsetAsync(sp.scan_status, 0, SPAN_SCAN_TILES * sizeof(unsigned long long), h->stream));
    SpanCtr c{};  // counters back to their starting values
    for (int d = 0; d < 3; ++d) {
      c.cmin[d] = LLONG_MAX;
      c.cmax[d] = LLONG_MIN;
    }
    CU(cudaStreamSynchronize(h->stream));
    CU(cudaMemcpy(sp.sc, &c, offsetof(SpanCtr, used), cudaMemcpyHostToDevice));
    CU(cudaMemsetAsync(sp.bits, 0, (size_t)(sp.chunk_cap * ((h->W + 31) / 32)) * sizeof(uint32_t), h->stream));
  }
  CU(cudaMemsetAsync(h->ctr, 0, sizeof(JobCtr) * kMaxJobs, h->stream));
  CU(cudaMemsetAsync(h->bs, 0, sizeof(BatchState), h->stream));
  if (h->bar) CU(cudaMemsetAsync(h->bar, 0, sizeof(GridBar), h->stream));
  return RTOD_OK;
}

void free_span(rtod_handle* h) {
  SpanScratch& sp = h->span;
  dfree(sp.bin_count); dfree(sp.bin_start); dfree(sp.kmin); dfree(sp.kmax); dfree(sp.cnt); dfree(sp.pre);
  dfree(sp.used); dfree(sp.s_off); dfree(sp.s_x); dfree(sp.scan_status); dfree(sp.sc);
  dfree(sp.bits); dfree(sp.groups);
  h->device_bytes -= sp.bytes;
  sp = SpanScratch{};
}

// Span scratch for spans of nblk slide blocks (nblk * S points) and bitsets
// of `chunk` slides.
int ensure_span(rtod_handle* h, int64_t nblk, int64_t chunk) {
  SpanScratch& sp = h->span;
  const int64_t pts = nblk * h->S;
  const int64_t words = (h->W + 31) / 32;
  if (sp.sc && nblk <= sp.nblk_cap && pts <= sp.pts_cap && chunk <= sp.chunk_cap) return RTOD_OK;
  CU(cudaStreamSynchronize(h->stream));
  free_span(h);
  drop_graph(h);
  const int64_t Wp = ((pts + 3) / 4) * 4 + 4;
  int64_t bytes = 0;
  bool ok = !dalloc(&sp.bin_count, NB, &bytes) && !dalloc(&sp.bin_start, NB + 1, &bytes) &&
            !dalloc(&sp.kmin, NB, &bytes) && !dalloc(&sp.kmax, NB, &bytes) &&
            !dalloc(&sp.cnt, (size_t)((nblk + 1) * NB), &bytes) && !dalloc(&sp.pre, (size_t)((nblk + 1) * NB), &bytes) &&
            !dalloc(&sp.used, NB, &bytes) && !dalloc(&sp.s_off, (size_t)pts, &bytes) &&
            !dalloc(&sp.s_x, (size_t)(Wp * h->D * h->esz), &bytes) && !dalloc(&sp.scan_status, SPAN_SCAN_TILES, &bytes) &&
            !dalloc(&sp.sc, 1, &bytes) && !dalloc(&sp.bits, (size_t)(chunk * words), &bytes) &&
            !dalloc(&sp.groups, (size_t)((nblk - h->W / h->S + 1) * std::min<int64_t>(h->W, NB)), &bytes);
  sp.bytes = bytes;
  h->device_bytes += bytes;
  if (!ok) {
    free_span(h);
    return RTOD_ERR_CUDA;
  }
  sp.nblk_cap = nblk;
  sp.ts = nblk + 1;
  sp.pts_cap = pts;
  sp.chunk_cap = chunk;
  sp.Wp = Wp;
  sp.gcap = (nblk - h->W / h->S + 1) * std::min<int64_t>(h->W, NB);
  CU(cudaMemset(sp.bits, 0, (size_t)(chunk * words) * sizeof(uint32_t)));
  CU(cudaMemset(sp.bin_count, 0, NB * sizeof(uint32_t)));
  CU(cudaMemset(sp.kmin, 0xff, NB * sizeof(unsigned long long)));
  CU(cudaMemset(sp.kmax, 0, NB * sizeof(unsigned long long)));
  CU(cudaMemset(sp.cnt, 0, (size_t)(sp.ts * NB) * sizeof(uint32_t)));
  CU(cudaMemset(sp.s_x, 0, (size_t)(Wp * h->D * h->esz)));
  CU(cudaMemset(sp.scan_status, 0, SPAN_SCAN_TILES * sizeof(unsigned long long)));
  SpanCtr c{};
  for (int d = 0; d < 3; ++d) {
    c.cmin[d] = LLONG_MAX;
    c.cmax[d] = LLONG_MIN;
  }
  c.used = sp.used;
  c.bin_count = sp.bin_count;
  c.kmin = sp.kmin;
  c.kmax = sp.kmax;
  CU(cudaMemcpy(sp.sc, &c, sizeof(SpanCtr), cudaMemcpyHostToDevice));
  return RTOD_OK;
}

// Span parameters of a batch of B windows over the resident stream, with
// bitsets of `chunk` slides.
Span make_span(const rtod_handle* h, int B, const void* stream_pts, int64_t chunk) {
  const SpanScratch& ss = h->span;
  Span sp{};
  sp.S = h->S;
  sp.Wp = ss.Wp;
  sp.wblk = (int32_t)(h->W / h->S);
  sp.nblk = sp.wblk + B - 1;
  sp.K = h->cfg.K;
  sp.n = h->n;
  sp.filter = h->filter;
  sp.h = h->D < 3 ? h->D : 3;
  // cells within R of every point of the centre cell: sum (|d_i| + 1)^2 < n^2
  sp.n_sure = 0;
  if (h->D <= 3) {
    const int n = h->n, H = sp.h;
    for (int d0 = -n; d0 <= n; ++d0)
      for (int d1 = (H >= 2 ? -n : 0); d1 <= (H >= 2 ? n : 0); ++d1)
        for (int d2 = (H >= 3 ? -n : 0); d2 <= (H >= 3 ? n : 0); ++d2) {
          const int q = (std::abs(d0) + 1) * (std::abs(d0) + 1) + (H >= 2 ? (std::abs(d1) + 1) * (std::abs(d1) + 1) : 0) +
                        (H >= 3 ? (std::abs(d2) + 1) * (std::abs(d2) + 1) : 0);
          if (q >= n * n || sp.n_sure >= 16) continue;
          const int delta = H == 1 ? d0 : (H == 2 ? d1 + 256 * d0 : d2 + 64 * d1 + 4096 * d0);
          sp.sure_delta[sp.n_sure++] = delta;
        }
  }
  sp.R = h->cfg.R;
  sp.R2 = h->cfg.R * h->cfg.R;
  sp.R2f = h->R2f;
  sp.pts = stream_pts;
  sp.keys = h->run_keys;
  sp.inv_cell = 1.0 / h->cell;
  sp.bin_count = ss.bin_count;
  sp.bin_start = ss.bin_start;
  sp.kmin = ss.kmin;
  sp.kmax = ss.kmax;
  sp.cnt = ss.cnt;
  sp.pre = ss.pre;
  sp.ts = ss.ts;
  sp.used = ss.used;
  sp.s_off = ss.s_off;
  sp.s_x = ss.s_x;
  sp.scan_status = ss.scan_status;
  sp.sc = ss.sc;
  sp.groups = ss.groups;
  sp.bits = ss.bits;
  sp.words = (h->W + 31) / 32;
  sp.chunk = chunk;
  sp.gcap = (uint32_t)ss.gcap;
  // delta segments (learned router): stencils of at most 32 slots, a cell
  // filter, and up to 3 dimensions
  {
    const int w = 2 * h->n + 1;
    const int slots = sp.h == 1 ? w : (sp.h == 2 ? w * w : w * w * w);
    sp.route = (h->cfg.router && h->span_route && h->D <= 3 && slots <= 32) ? 1 : 0;
  }
  return sp;
}

// Slides per bitset chunk of the span engine: a multiple of the batch B,
// within about 256 MiB of bitsets, and no more than the run needs.
int64_t span_chunk(const rtod_handle* h, int B, int64_t slides) {
  const int64_t row = ((h->W + 31) / 32) * 4;
  const int64_t per_batch = std::max<int64_t>(1, (256ll << 20) / (row * B));
  const int64_t batches = (slides + B - 1) / B;
  return (int64_t)B * std::max<int64_t>(1, std::min(per_batch, batches));
}

// Points per listed part of a bin in group mode, for a launch counting
// `points` points: parts short enough that there are about 16 per SM (a
// part is one warp's work), and long enough (up to 1024) that a warp's
// lanes are refilled from the part's other points while it walks the
// candidates.
int32_t group_part(int64_t points, int sm_count) {
  const int64_t fill = points / ((int64_t)sm_count * 16);
  int32_t p = 32;
  while (p < 1024 && 2 * (int64_t)p <= fill) p *= 2;
  return p;
}

// Points per listed part of a bin in group mode. Parts are taken from the
// batch-wide count list (k_count), so short parts keep the launch's tail
// short; measured on the 8-d streams of the 64-stream workload (B200, median
// step): parts of up to 512 points 5.00 ms, 256 4.69 ms, 128 4.38 ms.
constexpr int32_t kGroupPartMax = 128;
int32_t group_part_size(int64_t points, int sm_count) { return std::min(kGroupPartMax, group_part(points, sm_count)); }

// Whether RTOD_COUNT_AUTO picks group counts for a launch of `points`
// points: in more than 3 dimensions (no cell is ever all-inlier, so every
// point is counted and a bin's points are many) when the parts hold at
// least 256 points. Measured on 8-d Gaussian blobs: shorter parts (a single
// window of 162k points, 64-point parts) are slower than point counts, while
// 64 streams of 1.6M points in all (512-point parts) gain a quarter.
bool auto_group(int D, int64_t points, int sm_count) { return D > 3 && group_part(points, sm_count) >= 256; }

Job make_job(rtod_handle* h, int j, bool ring, const void* stream_pts) {
  Job jb{};
  jb.W = h->W;
  jb.S = h->S;
  jb.Wp = h->Wp;
  jb.inv_cell = 1.0 / h->cell;
  jb.R = h->cfg.R;
  jb.R2 = h->cfg.R * h->cfg.R;
  jb.R2f = h->R2f;
  jb.K = h->cfg.K;
  jb.n = h->n;
  jb.filter = h->filter;
  jb.ring = ring ? 1 : 0;
  jb.gpts = 32;
  jb.pts = ring ? h->ring : stream_pts;
  jb.keys = ring ? h->ring_keys : h->run_keys;
  jb.stage = h->staging;
  jb.blk_lo = ring ? nullptr : h->run_blk_lo;
  jb.blk_hi = ring ? nullptr : h->run_blk_hi;
  jb.prev = ring ? h->ring_prev : h->run_prev;
  const Scratch& s = h->pool[j];
  jb.bin_count = s.bin_count;
  jb.bin_start = s.bin_start;
  jb.kmin = s.kmin;
  jb.kmax = s.kmax;
  jb.s_off = s.s_off;
  jb.s_ckey = s.s_ckey;
  jb.s_x = s.s_x;
  jb.queue = s.queue;
  jb.feat = s.feat;
  jb.flags = s.flags;
  jb.scan_status = s.scan_status;
  jb.cmp_status = s.cmp_status;
  jb.ctr = h->ctr + j;
  jb.rec_nout = ring ? nullptr : h->rec_nout;
  jb.rec_undet = ring ? nullptr : h->rec_undet;
  jb.rec_base = ring ? nullptr : h->rec_base;
  jb.rec_cap = ring ? 0 : h->rec_cap;
  return jb;
}

// Uploads the job table for a mode (only when it changed, so that captured
// graphs stay valid) and initialises the job counters: job j starts at
// window lo = first_lo + j*S and advances by jobs*S per batch.
int configure(rtod_handle* h, int mode, int jobs, int64_t first_lo, const void* stream_pts, bool full = true,
              bool copy_ctr = true) {
  int r = ensure_pool(h, jobs, full);
  if (r) return r;
  std::vector<Job> tab((size_t)jobs);
  for (int j = 0; j < jobs; ++j) {
    tab[j] = make_job(h, j, mode == MODE_RING, stream_pts);
    tab[j].gpts = group_part_size(h->W * jobs, h->sm_count);
  }
  if (tab.size() != h->tab_host.size() ||
      std::memcmp(tab.data(), h->tab_host.data(), sizeof(Job) * tab.size()) != 0) {
    CU(cudaMemcpy(h->jobs_dev, tab.data(), sizeof(Job) * jobs, cudaMemcpyHostToDevice));
    h->tab_host = tab;
    drop_graph(h);
  }
  for (int j = 0; j < jobs; ++j) {
    h->ctr_init[j] = JobCtr{};
    h->ctr_init[j].lo = first_lo + (int64_t)j * h->S;
    h->ctr_init[j].lo_step = (int64_t)jobs * h->S;
  }
  // Pinned source; every public call ends with a stream sync, so the buffer
  // is never rewritten while a copy from it is pending (without copy_ctr the
  // caller enqueues the copy).
  if (copy_ctr) CU(cudaMemcpyAsync(h->ctr, h->ctr_init, sizeof(JobCtr) * jobs, cudaMemcpyHostToDevice, h->stream));
  h->mode = mode;
  return RTOD_OK;
}

Batch make_batch(rtod_handle* h, int njobs, int64_t out_cap, int64_t* out_ids = nullptr) {
  Batch b{};
  b.jobs = h->jobs_dev;
  b.njobs = njobs;
  b.bs = h->bs;
  b.router = h->router;
  b.out_ids = out_ids ? out_ids : h->ids;
  b.out_cap = out_cap;
  b.cmp_tiles = (int64_t)njobs * ((h->W + CMP_TILE - 1) / CMP_TILE);
  return b;
}

// Launch geometry of a group of jobs that share a dimension and predicate.
struct Geom {
  int64_t Wmax, Smax;
  int D, pred, route, sm_count, block_warps;
  RouterState* router;
  int f64 = 0;    // double coordinates
  int group = 0;  // group counts (route is then 0)
};

// Online training of the router on the buffered counts (one block; it
// returns at once until enough samples are buffered), then the routing table.
int launch_train(const Geom& g, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = TRAIN_SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CU(cudaLaunchKernelEx(&cfg, k_train, g.router));
  CU(launch_k(k_table, dim3((TQ0 * TQ1 * TQ2 + 255) / 256), 256, st, g.router));
  return RTOD_OK;
}

// Launches one batch: hist (with the ring jobs' ingest folded in) scan
// scatter count compact [train]. kev (may be null) receives an event at the
// start (kev[0]) and after each kernel (kev[6] after training or compact).
// ids_host / mirror (streaming): the mapped landing buffers that the
// compaction's last block fills with the IDs and the batch state.
// Returns the number of kernels launched in *nk.
int launch_group(const Geom& g, const Batch& b, bool ingest, bool train, cudaStream_t st, cudaEvent_t* kev,
                 int64_t* nk, int64_t* ids_host = nullptr, int64_t ids_host_cap = 0, BatchState* mirror = nullptr) {
  const int64_t W = g.Wmax, nj = b.njobs;
  const unsigned gy = (unsigned)nj;
  int64_t launched = 0;
  if (kev) CU(cudaEventRecord(kev[0], st));
  const int64_t per_block = 256 * (g.D <= 3 ? 2 : 1);  // points per block per loop iteration (Unroll)
  const int64_t wx = std::max<int64_t>(
      1, std::min<int64_t>((W + per_block - 1) / per_block, std::max<int64_t>(2, (g.sm_count * 16 + nj - 1) / nj)));
  if (ingest) {  // ring jobs: the slide's ingest folded into the histogram, the output restarted
    DISPATCH_DT(g.f64, g.D, CU(launch_k(k_hist_ingest<D, T>, dim3((unsigned)wx, gy), 256, st, b, 1)));
  } else {
    DISPATCH_D(g.D, CU(launch_k(k_hist<D>, dim3((unsigned)wx, gy), 256, st, b)));
  }
  if (kev) CU(cudaEventRecord(kev[1], st));
  CU(launch_k(k_scan, dim3(SCAN_TILES, gy), 256, st, b));
  if (kev) CU(cudaEventRecord(kev[2], st));
  if (g.route) {
    DISPATCH_DT(g.f64, g.D, CU(launch_k(k_scatter<D, true, T>, dim3((unsigned)wx, gy), 256, st, b)));
  } else if (g.group) {
    DISPATCH_DT(g.f64, g.D, CU(launch_k(k_scatter<D, false, T, true>, dim3((unsigned)wx, gy), 256, st, b)));
  } else {
    DISPATCH_DT(g.f64, g.D, CU(launch_k(k_scatter<D, false, T>, dim3((unsigned)wx, gy), 256, st, b)));
  }
  if (kev) CU(cudaEventRecord(kev[3], st));
  const int wpb = g.block_warps;
  const int64_t cx = std::max<int64_t>(1, (int64_t)g.sm_count * (64 / wpb) / nj);
  if (g.route) {
    DISPATCH_DPT(g.f64, g.D, g.pred,
                 CU(launch_k(k_count<D, PRED, true, T>, dim3((unsigned)cx, gy), wpb * 32, st, b)));
  } else if (g.group) {
    DISPATCH_DPT(g.f64, g.D, g.pred,
                 CU(launch_k(k_count<D, PRED, false, T, true>, dim3((unsigned)cx, gy), wpb * 32, st, b)));
  } else {
    DISPATCH_DPT(g.f64, g.D, g.pred,
                 CU(launch_k(k_count<D, PRED, false, T>, dim3((unsigned)cx, gy), wpb * 32, st, b)));
  }
  if (kev) CU(cudaEventRecord(kev[4], st));
  if (ingest && W <= COMPACT1_MAX) {  // ring jobs: one block per window, delivering a detection's IDs itself
    CU(launch_k(k_compact_one, dim3(gy), 1024, st, b, ids_host, ids_host_cap, mirror));
  } else {
    CU(launch_k(k_compact, dim3((unsigned)((W + CMP_TILE - 1) / CMP_TILE), gy), 256, st, b));
    if (ids_host || mirror) {
      const unsigned ox = (unsigned)std::max<int64_t>(1, std::min<int64_t>((W + 255) / 256, g.sm_count));
      CU(launch_k(k_run_out, dim3(ox), 256, st, (const int64_t*)b.out_ids, ids_host, ids_host_cap, b.bs, mirror));
      launched++;
    }
  }
  if (kev) CU(cudaEventRecord(kev[5], st));
  launched += 5;
  if (g.route && train) {
    if (int r = launch_train(g, st)) return r;
    launched += 2;
  }
  if (kev) CU(cudaEventRecord(kev[6], st));
  if (nk) *nk = launched;
  return RTOD_OK;
}

// One batch of ring jobs (push/detect, the multi-stream API) as a single
// cooperative launch of the fused pipeline (fused.cuh), then the router's
// training step when due. *grid caches the launch's block count: as many
// blocks as can be resident (up to 2 per SM), found on first use.
int launch_fused(const Geom& g, const Batch& b, GridBar* bar, bool reset_out, int64_t* ids_host,
                 int64_t ids_host_cap, BatchState* mirror, bool train, cudaStream_t st, int* grid, int64_t* nk) {
  const FusedKind kind{g.D, g.f64 ? RTOD_PRED_F64_LT : g.pred, g.route, g.group};
  Fused f{};
  f.bar = bar;
  auto dispatch = [&](int gsize, int* per_sm) {
    return g.f64 ? fused_dispatch<double>(kind, b, f, gsize, st, per_sm)
                 : fused_dispatch<float>(kind, b, f, gsize, st, per_sm);
  };
  if (*grid <= 0) {
    int per_sm = 0;
    CU(dispatch(0, &per_sm));
    if (per_sm < 1) return fail(RTOD_ERR_CUDA, "the fused pipeline kernel cannot be resident");
    *grid = std::min(per_sm, 2) * g.sm_count;
  }
  const int64_t per_block = 256 * (g.D <= 3 ? 2 : 1);  // points per block and step (Unroll)
  f.hx = (uint32_t)std::max<int64_t>(1, (g.Wmax + per_block - 1) / per_block);
  f.cx = (uint32_t)*grid;  // every job's queue is shared by all warps of the grid
  f.tx = (uint32_t)((g.Wmax + CMP_TILE - 1) / CMP_TILE);
  f.reset_out = reset_out ? 1 : 0;
  f.ids_host = ids_host;
  f.ids_host_cap = ids_host_cap;
  f.mirror = mirror;
  CU(dispatch(*grid, nullptr));
  int64_t launched = 1;
  if (g.route && train) {
    if (int r = launch_train(g, st)) return r;
    launched += 2;
  }
  if (nk) *nk = launched;
  return RTOD_OK;
}

// Launches one batch of the span engine: hist scan prefix scatter classify
// count. kev as for launch_group, with kev[1] after hist, kev[2] after scan +
// prefix, kev[4] after classify and kev[5] after count (the stage slots of
// count, compact and train hold classify, count and the chunk compaction
// timed by run_stream).
int launch_span(const Geom& g, const Batch& b, const Span& sp, cudaStream_t st, cudaEvent_t* kev, int64_t* nk) {
  const int64_t npts = sp.nblk * sp.S;
  // histogram and scatter: 512 points per block and step, up to 16 blocks per SM
  const int64_t hx = std::max<int64_t>(1, std::min<int64_t>((npts + 511) / 512, (int64_t)g.sm_count * 16));
  if (kev) CU(cudaEventRecord(kev[0], st));
  DISPATCH_DT(g.f64, g.D, CU(launch_k(k_span_hist<D, T>, dim3((unsigned)hx), 256, st, b, sp)));
  if (kev) CU(cudaEventRecord(kev[1], st));
  CU(launch_k(k_span_scan, dim3(SPAN_SCAN_TILES), 256, st, b, sp));
  CU(launch_k(k_span_prefix, dim3((unsigned)(g.sm_count * 4)), 256, st, b, sp));
  if (kev) CU(cudaEventRecord(kev[2], st));
  DISPATCH_DT(g.f64, g.D, CU(launch_k(k_span_scatter<D, T>, dim3((unsigned)hx), 256, st, b, sp)));
  if (kev) CU(cudaEventRecord(kev[3], st));
  if (sp.route) {
    CU(launch_k(k_span_classify<true>, dim3((unsigned)(g.sm_count * 4)), 256, st, b, sp));
  } else {
    CU(launch_k(k_span_classify<false>, dim3((unsigned)(g.sm_count * 4)), 256, st, b, sp));
  }
  if (kev) CU(cudaEventRecord(kev[4], st));
  const int wpb = g.block_warps;
  const int64_t cx = (int64_t)g.sm_count * (64 / wpb);
  DISPATCH_DPT(g.f64, g.D, g.pred, {
    if constexpr (D <= 3) {
      if (sp.route) {
        CU(launch_k(k_span_count<D, PRED, T, true>, dim3((unsigned)cx), wpb * 32, st, b, sp));
      } else {
        CU(launch_k(k_span_count<D, PRED, T>, dim3((unsigned)cx), wpb * 32, st, b, sp));
      }
    } else {
      CU(launch_k(k_span_count<D, PRED, T>, dim3((unsigned)cx), wpb * 32, st, b, sp));
    }
  });
  if (kev) CU(cudaEventRecord(kev[5], st));
  if (kev) CU(cudaEventRecord(kev[6], st));  // no per-batch compaction: see span_flush
  if (nk) *nk = 6;
  return RTOD_OK;
}

// Deferred compaction of span-engine slides [s0, s0 + n) (one bitset chunk).
int span_flush(rtod_handle* h, const Span& sp, int64_t s0, int64_t n, int64_t out_cap, int64_t* out_ids) {
  SpanOut o{};
  o.bits = sp.bits;
  o.words = sp.words;
  o.chunk = sp.chunk;
  o.W = h->W;
  o.S = h->S;
  o.rec_base = h->rec_base;
  o.out_ids = out_ids;
  o.out_cap = out_cap;
  o.bs = h->bs;
  CU(launch_k(k_span_compact, dim3((unsigned)n), 1024, h->stream, o, s0));
  h->launches += 1;
  return RTOD_OK;
}

Geom geom_of(const rtod_handle* h) {
  return Geom{h->W, h->S, h->D, h->cfg.pred, h->cfg.router && !h->group, h->sm_count, h->block_warps,
              h->router, h->f64, h->group};
}

constexpr int kTrainEvery = 16;  // batches between two router training launches (after the first)
constexpr int kTrainWarm = 32;   // the first batches train after every batch

bool train_now(rtod_handle* h) {
  if (!h->cfg.router || h->tuning_pass) return false;
  const int64_t n = h->batches++;
  return n < kTrainWarm || n % kTrainEvery == 0;
}

// End of a streaming detection (ring jobs): the window's IDs and the batch
// state into the mapped landing buffers (ensure_detect_out).
// A streaming detection of the staged pipeline: its launch sequence, ending
// with the window's IDs and the batch state in the mapped landing buffers.
int launch_ring(rtod_handle* h, const Batch& b, bool train, cudaEvent_t* kev, int64_t* nk) {
  return launch_group(geom_of(h), b, true, train, h->stream, kev, nk, h->ids_host_dev,
                      std::min(h->ids_host_cap, h->ids_cap), h->bs_mirror_dev);
}

// Whether a streaming detection runs the fused pipeline (one launch): when
// configured, except when per-stage times are asked for.
bool fused_ring(const rtod_handle* h, const cudaEvent_t* kev) {
  return h->cfg.pipeline == RTOD_PIPELINE_FUSED && !kev;
}

// ---------------------------------------------------------------------------
// Streaming grid engine (push/detect; grid.cuh)
// ---------------------------------------------------------------------------
constexpr int64_t kGridMaxW = COMPACT1_MAX;  // one compaction block per detection
constexpr int64_t kGridMaxBlocks = 4096;    // slide blocks per window (per-block cell ranges)
constexpr uint64_t kGridMaxPool = 1ull << 31;  // pool slots (slot numbers are 32-bit)

int check_device_error(rtod_handle* h, const BatchState& s);

bool grid_wanted(const rtod_handle* h) {
  const rtod_config& c = h->cfg;
  // only on request: the window engine's per-slide sort was measured as fast
  // or faster on every benchmark stream
  if (c.engine != RTOD_ENGINE_GRID) return false;
  return h->D <= 3 && h->W <= kGridMaxW && h->W / h->S <= kGridMaxBlocks;
}

int64_t grid_pool_bytes(const rtod_handle* h, uint64_t pool) { return (int64_t)pool * (h->D * h->esz + 4); }

void free_grid_pool(rtod_handle* h) {
  Grid& g = h->grid.g;
  if (g.px) {
    h->grid.bytes -= grid_pool_bytes(h, g.pool);
    h->device_bytes -= grid_pool_bytes(h, g.pool);
  }
  dfree(g.px);
  dfree(g.pslot);
  g.pool = 0;
  h->grid.built = false;
}

void free_grid(rtod_handle* h) {
  Grid& g = h->grid.g;
  free_grid_pool(h);
  dfree(g.ctl); dfree(g.head); dfree(g.tail); dfree(g.base); dfree(g.cap); dfree(g.ref); dfree(g.mixed);
  dfree(g.growflag); dfree(g.grow); dfree(g.grow_to); dfree(g.ovf_bin); dfree(g.ovf_pos); dfree(g.ovf_slot); dfree(g.ovf_x);
  dfree(g.brange); dfree(g.qpos); dfree(g.qbin);
  h->device_bytes -= h->grid.bytes;
  h->grid.bytes = 0;
}

// Device arrays of the grid; a pool of at least `pool` slots (replaced when
// it is smaller).
int ensure_grid(rtod_handle* h, uint64_t pool) {
  GridHost& G = h->grid;
  Grid& g = G.g;
  if (!g.ctl) {
    int64_t n = 0;
    const size_t S = (size_t)h->S;
    g.ovf_cap = (uint32_t)S;
    g.nslots = (int32_t)(h->W / h->S + 1);
    bool ok = !dalloc(&g.ctl, 1, &n) && !dalloc(&g.head, NB, &n) && !dalloc(&g.tail, NB, &n) &&
              !dalloc(&g.base, NB, &n) && !dalloc(&g.cap, NB, &n) && !dalloc(&g.ref, NB, &n) &&
              !dalloc(&g.mixed, NB, &n) && !dalloc(&g.growflag, NB, &n) && !dalloc(&g.grow, S, &n) && !dalloc(&g.grow_to, 2 * S, &n) &&
              !dalloc(&g.ovf_bin, S, &n) && !dalloc(&g.ovf_pos, S, &n) && !dalloc(&g.ovf_slot, S, &n) &&
              !dalloc((unsigned char**)&g.ovf_x, S * (size_t)(h->D * h->esz), &n) &&
              !dalloc(&g.brange, (size_t)g.nslots * 6, &n) && !dalloc(&g.qpos, (size_t)h->W, &n) &&
              !dalloc(&g.qbin, (size_t)h->W, &n);
    G.bytes += n;
    h->device_bytes += n;
    if (!ok) return RTOD_ERR_CUDA;
  }
  if (g.pool < pool) {
    drop_graph(h);
    free_grid_pool(h);
    int64_t n = 0;
    if (dalloc((unsigned char**)&g.px, (size_t)pool * (size_t)(h->D * h->esz), &n) ||
        dalloc(&g.pslot, (size_t)pool, &n)) {
      dfree(g.px);
      dfree(g.pslot);
      return RTOD_ERR_CUDA;
    }
    g.pool = (uint32_t)pool;
    G.bytes += grid_pool_bytes(h, pool);
    h->device_bytes += grid_pool_bytes(h, pool);
  }
  return RTOD_OK;
}

GridKind grid_kind(const rtod_handle* h) { return GridKind{h->D, h->cfg.pred, h->f64}; }

// Builds the grid of the ring's window [lo, lo + W), doubling the pool
// while the regions do not fit. Returns RTOD_OK with h->grid.on cleared when
// no pool within kGridMaxPool holds them (push/detect then run the window
// engine).
int grid_build(rtod_handle* h, int64_t lo) {
  GridHost& G = h->grid;
  // default: the bins' starting regions (2 * GRID_FRESH_CAP slots each) and
  // eight times the window for grown regions and their garbage
  const uint64_t first = G.pool_first ? G.pool_first : 16ull * (uint64_t)h->W + 4ull * GRID_FRESH_CAP * NB;
  uint64_t pool = std::max<uint64_t>(G.g.pool, std::min<uint64_t>(kGridMaxPool, first));
  const Batch b = make_batch(h, 1, h->ids_cap);
  for (int attempt = 0; attempt < 8; ++attempt) {
    if (int r = ensure_grid(h, pool)) return r;
    CU(cudaMemsetAsync(&h->bs->err, 0, sizeof(int32_t), h->stream));
    CU(grid_launch_build(grid_kind(h), b, G.g, lo, h->W, h->S, h->sm_count, h->stream));
    h->launches += h->W / h->S + 4;
    int32_t err = 0;
    unsigned long long wanted = 0;  // slots the regions asked for (k_grid_alloc counts every bin)
    CU(cudaMemcpyAsync(&err, &h->bs->err, sizeof err, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(&wanted, &G.g.ctl->pool_top, sizeof wanted, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    G.builds++;
    if (err == DERR_NONE) {
      G.built = true;
      return RTOD_OK;
    }
    if (err != DERR_GRID) {
      BatchState s{};
      s.err = err;
      return check_device_error(h, s);
    }
    if (pool >= kGridMaxPool) break;
    // room for the regions and as much again for their growth
    pool = std::min<uint64_t>(kGridMaxPool, std::max<uint64_t>(2 * pool, 2 * (uint64_t)wanted));
  }
  // no pool holds the window's regions: the window engine takes over
  CU(cudaMemsetAsync(&h->bs->err, 0, sizeof(int32_t), h->stream));
  CU(cudaStreamSynchronize(h->stream));
  free_grid(h);
  G.on = false;
  drop_graph(h);
  return RTOD_OK;
}

// After a detection that reported DERR_GRID (nothing counted, the window
// not advanced): rebuilds the grid from the ring, which holds the window
// with the new slide, and counts it again; or, when no pool holds the
// grid, lets the window engine take the slide (its histogram re-ingests
// the staged slide) and the rest of the stream.
int launch_ring(rtod_handle* h, const Batch& b, bool train, cudaEvent_t* kev, int64_t* nk);
int launch_grid(rtod_handle* h, const Batch& b, bool ingest, cudaEvent_t* kev, int64_t* nk);

int grid_recount(rtod_handle* h, const Batch& b) {
  if (int r = grid_build(h, h->S * (h->slides_done + 1))) return r;
  int64_t nk = 0;
  int r = h->grid.on ? launch_grid(h, b, false, nullptr, &nk) : launch_ring(h, b, false, nullptr, &nk);
  if (r) return r;
  h->launches += nk;
  CU(cudaStreamSynchronize(h->stream));
  return RTOD_OK;
}

// One streaming detection of the grid engine: ingest, classify, count, compaction
// (into the mapped landing buffers). kev as for launch_group.
int launch_grid(rtod_handle* h, const Batch& b, bool ingest, cudaEvent_t* kev, int64_t* nk) {
  const GridKind k = grid_kind(h);
  if (kev) CU(cudaEventRecord(kev[0], h->stream));
  if (ingest) CU(grid_launch_ingest(k, b, h->grid.g, h->S, h->sm_count, h->stream));
  if (kev) {
    CU(cudaEventRecord(kev[1], h->stream));
    CU(cudaEventRecord(kev[2], h->stream));
    CU(cudaEventRecord(kev[3], h->stream));
  }
  CU(grid_launch_count(k, b, h->grid.g, h->sm_count, h->stream));
  if (kev) CU(cudaEventRecord(kev[4], h->stream));
  CU(launch_k(k_compact_one, dim3(1), 1024, h->stream, b, h->ids_host_dev, std::min(h->ids_host_cap, h->ids_cap),
              h->bs_mirror_dev));
  if (kev) {
    CU(cudaEventRecord(kev[5], h->stream));
    CU(cudaEventRecord(kev[6], h->stream));
  }
  if (nk) *nk = ingest ? 4 : 3;
  return RTOD_OK;
}

int launch_batch(rtod_handle* h, const Batch& b, bool ingest, cudaEvent_t* kev, const Span* sp = nullptr) {
  int64_t nk = 0;
  if (ingest && !sp && h->grid.on) {
    int r = launch_grid(h, b, true, kev, &nk);
    h->launches += nk;
    return r;
  }
  if (ingest && !sp && fused_ring(h, kev)) {
    int r = launch_fused(geom_of(h), b, h->bar, true, h->ids_host_dev, std::min(h->ids_host_cap, h->ids_cap),
                         h->bs_mirror_dev, train_now(h), h->stream, &h->fused_grid, &nk);
    h->launches += nk;
    return r;
  }
  int r = sp ? launch_span(geom_of(h), b, *sp, h->stream, kev, &nk)
             : (ingest ? launch_ring(h, b, train_now(h), kev, &nk)
                       : launch_group(geom_of(h), b, false, train_now(h), h->stream, kev, &nk));
  h->launches += nk;
  return r;
}

// Runs one batch, replaying a captured graph when graphs are on (two graphs
// with the router: with and without the training step).
int run_batch(rtod_handle* h, const Batch& b, bool ingest, const Span* sp = nullptr) {
  if (!h->cfg.use_graph) return launch_batch(h, b, ingest, nullptr, sp);
  const bool train = sp ? false : train_now(h);
  cudaGraphExec_t& gx = h->graphs[train ? 1 : 0];
  const bool same = h->graph_ring == (int)ingest && std::memcmp(&h->graph_batch, &b, sizeof(Batch)) == 0 &&
                    h->graph_is_span == (sp != nullptr) &&
                    (!sp || std::memcmp(&h->graph_span, sp, sizeof(Span)) == 0);
  if (!gx || !same) {
    if (!same) drop_graph(h);
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int64_t nk = 0;
    int r;
    if (ingest && !sp && h->grid.on) {
      r = launch_grid(h, b, true, nullptr, &nk);
    } else if (ingest && !sp && fused_ring(h, nullptr)) {
      r = launch_fused(geom_of(h), b, h->bar, true, h->ids_host_dev, std::min(h->ids_host_cap, h->ids_cap),
                       h->bs_mirror_dev, train, h->stream, &h->fused_grid, &nk);
    } else {
      r = sp ? launch_span(geom_of(h), b, *sp, h->stream, nullptr, &nk)
             : (ingest ? launch_ring(h, b, train, nullptr, &nk)
                       : launch_group(geom_of(h), b, false, train, h->stream, nullptr, &nk));
    }
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (r) return r;
    if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&gx, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    h->graph_batch = b;
    h->graph_ring = (int)ingest;
    h->graph_is_span = sp != nullptr;
    if (sp) h->graph_span = *sp;
    h->graph_kernels[train ? 1 : 0] = nk;
  }
  CU(cudaGraphLaunch(gx, h->stream));
  h->launches += h->graph_kernels[train ? 1 : 0];
  h->graph_replays++;
  return RTOD_OK;
}

int check_device_error(rtod_handle* h, const BatchState& s) {
  if (s.err == DERR_NONE) return RTOD_OK;
  h->poisoned = true;
  switch (s.err) {
    case DERR_NONFINITE: return fail(RTOD_ERR_INPUT, "non-finite coordinate in the stream");
    case DERR_RANGE: return fail(RTOD_ERR_INPUT, "coordinate too large for the grid (|x| / cell beyond the limit)");
    case DERR_CAPACITY: return fail(RTOD_ERR_CAPACITY, "outlier ID buffer too small");
    case DERR_TIMEOUT: return fail(RTOD_ERR_TIMEOUT, "a bounded device-side wait ran out");
    default: return fail(RTOD_ERR_CUDA, "device error %d", s.err);
  }
}

// Scratch cleans up after every completed batch, so a reset only clears the
// counters, unless an error may have left a batch half done.
int reset_state(rtod_handle* h) {
  int r;
  if (h->poisoned) {
    r = scrub(h);
  } else {
    CU(cudaMemsetAsync(h->ctr, 0, sizeof(JobCtr) * kMaxJobs, h->stream));
    CU(cudaMemsetAsync(h->bs, 0, sizeof(BatchState), h->stream));
    r = RTOD_OK;
  }
  if (r) return r;
  h->n_pushed = 0;
  h->slides_done = 0;
  h->pending = false;
  h->launched = false;
  h->poisoned = false;
  h->mode = MODE_NONE;
  // the next first push builds the grid again (or retries it, when no pool held it)
  const bool want = grid_wanted(h);
  if (want != h->grid.on) drop_graph(h);
  h->grid.on = want;
  h->grid.built = false;
  return RTOD_OK;
}

int ensure_ids(rtod_handle* h, int64_t cap) {
  if (cap <= h->ids_cap) return RTOD_OK;
  if (h->ids) h->device_bytes -= h->ids_cap * 8;
  dfree(h->ids);
  h->ids_cap = 0;
  if (dalloc(&h->ids, (size_t)cap, &h->device_bytes)) return RTOD_ERR_CUDA;
  h->ids_cap = cap;
  drop_graph(h);
  return RTOD_OK;
}

int ensure_records(rtod_handle* h, int64_t n) {
  if (!h->bs_mirror) {
    void* dp = nullptr;
    CU(cudaHostAlloc((void**)&h->bs_mirror, sizeof(BatchState), cudaHostAllocMapped));
    CU(cudaHostGetDevicePointer(&dp, h->bs_mirror, 0));
    h->bs_mirror_dev = (BatchState*)dp;
  }
  if (n <= h->rec_cap) return RTOD_OK;
  drop_graph(h);
  if (h->rec_base) h->device_bytes -= h->rec_cap * 8;
  dfree(h->rec_base);
  if (h->rec_host) cudaFreeHost(h->rec_host);
  h->rec_host = nullptr;
  h->rec_nout = h->rec_undet = h->rec_nout_h = h->rec_undet_h = nullptr;
  h->rec_cap = 0;
  if (dalloc(&h->rec_base, (size_t)n, &h->device_bytes)) return RTOD_ERR_CUDA;
  void* dp = nullptr;
  CU(cudaHostAlloc(&h->rec_host, 2 * (size_t)n * sizeof(int32_t), cudaHostAllocMapped));
  CU(cudaHostGetDevicePointer(&dp, h->rec_host, 0));
  h->rec_nout_h = (int32_t*)h->rec_host;
  h->rec_undet_h = h->rec_nout_h + n;
  h->rec_nout = (int32_t*)dp;
  h->rec_undet = h->rec_nout + n;
  h->rec_cap = n;
  return RTOD_OK;
}

// Landing buffers of streaming detection: the batch state mirror and one
// window's IDs in mapped page-locked memory (k_run_out writes both at the
// end of the detect graph, so the host waits once and copies nothing back).
int ensure_detect_out(rtod_handle* h) {
  if (!h->bs_mirror) {
    void* dp = nullptr;
    CU(cudaHostAlloc((void**)&h->bs_mirror, sizeof(BatchState), cudaHostAllocMapped));
    CU(cudaHostGetDevicePointer(&dp, h->bs_mirror, 0));
    h->bs_mirror_dev = (BatchState*)dp;
  }
  if (h->ids_host_cap < h->W) {
    drop_graph(h);
    if (h->ids_host) cudaFreeHost(h->ids_host);
    h->ids_host = h->ids_host_dev = nullptr;
    h->ids_host_cap = 0;
    void* dp = nullptr;
    CU(cudaHostAlloc((void**)&h->ids_host, (size_t)h->W * sizeof(int64_t), cudaHostAllocMapped));
    CU(cudaHostGetDevicePointer(&dp, h->ids_host, 0));
    h->ids_host_dev = (int64_t*)dp;
    h->ids_host_cap = h->W;
  }
  return RTOD_OK;
}

// Room for a stream of `used` points: the handle's run buffer for a host
// stream (*host = true; run_stream copies it in), its keys and features.
int stage_stream(rtod_handle* h, const void* pts, int64_t used, const void** src, bool* host,
                 bool memsets = true, bool* pinned = nullptr) {
  const int64_t D = h->D;
  *src = pts;
  *host = !is_device_ptr(pts);
  if (pinned) *pinned = *host && pinned_host_ptr(pts);
  if (*host) {
    if (h->run_buf_cap < used * D) {
      if (h->run_buf) h->device_bytes -= h->run_buf_cap * h->esz;
      dfree(h->run_buf);
      h->run_buf_cap = 0;
      if (dalloc(&h->run_buf, (size_t)(used * D * h->esz), &h->device_bytes)) return RTOD_ERR_CUDA;
      h->run_buf_cap = used * D;
    }
    *src = h->run_buf;  // filled piece by piece by run_stream
  }
  if (h->run_key_cap < used) {
    if (h->run_keys) h->device_bytes -= h->run_key_cap * 9;
    dfree(h->run_keys);
    dfree(h->run_prev);
    h->run_key_cap = 0;
    if (dalloc(&h->run_keys, (size_t)used, &h->device_bytes) || dalloc(&h->run_prev, (size_t)used, &h->device_bytes))
      return RTOD_ERR_CUDA;
    h->run_key_cap = used;
  }
  const int64_t blocks = used / h->S + 1;
  if (h->run_blk_cap < blocks) {
    if (h->run_blk_lo) h->device_bytes -= h->run_blk_cap * 48;
    dfree(h->run_blk_lo);
    dfree(h->run_blk_hi);
    h->run_blk_cap = 0;
    if (dalloc(&h->run_blk_lo, (size_t)(blocks * 3), &h->device_bytes) ||
        dalloc(&h->run_blk_hi, (size_t)(blocks * 3), &h->device_bytes))
      return RTOD_ERR_CUDA;
    h->run_blk_cap = blocks;
  }
  // +inf / -inf patterns for the atomic min / max of k_keys (without memsets
  // the caller enqueues them)
  if (memsets) {
    CU(cudaMemsetAsync(h->run_blk_lo, 0x7f, (size_t)(blocks * 3) * sizeof(long long), h->stream));
    CU(cudaMemsetAsync(h->run_blk_hi, 0x80, (size_t)(blocks * 3) * sizeof(long long), h->stream));
  }
  return RTOD_OK;
}

// Whether rtod_run uses the span engine: at most SPAN_MAX_BLOCKS slide
// blocks per window.
bool use_span(const rtod_handle* h) {
  return h->engine == RTOD_ENGINE_SPAN && h->W / h->S <= SPAN_MAX_BLOCKS;
}

// Largest batch of the span engine: spans of at most SPAN_MAX_BLOCKS blocks
// and fewer than 2^31 points.
int64_t span_batch_cap(const rtod_handle* h) {
  const int64_t wblk = h->W / h->S;
  return std::max<int64_t>(1, std::min<int64_t>(SPAN_MAX_BLOCKS, ((1ll << 31) - 1) / h->S) - wblk + 1);
}

int pick_batch(const rtod_handle* h, int64_t slides) {
  int64_t b;
  if (use_span(h)) {
    b = std::min<int64_t>(h->cfg.batch ? h->cfg.batch : 32, std::min<int64_t>(h->span_batch_max, span_batch_cap(h)));
  } else {
    b = h->cfg.batch ? std::min(h->cfg.batch, h->batch_max) : h->batch_max;
  }
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, slides));
}

int64_t count_slides(const rtod_handle* h, int64_t n, int64_t max_slides) {
  int64_t sl = n >= h->W ? (n - h->W) / h->S : 0;
  if (max_slides >= 0) sl = std::min(sl, max_slides);
  return sl;
}

// Shared body of rtod_run and rtod_profile_run: the stream is copied in (if
// on the host), its cell keys computed, then the slides are detected in
// batches of B consecutive windows. kev (may be null) gets 8 events per
// batch: one before and one after each kernel (the last one after the
// router's training step, or right after k_compact without router).
// Windows per batch of an rtod_run of `slides` slides from pts. A host
// stream that one span batch would cover runs as two: the copy of the second
// half then overlaps the first batch's detection (a 4 MB page-locked stream
// of 189 slides: 1.14 -> 1.07 us per slide end to end; three batches or more
// lose again to per-batch latency).
int run_batch_size(rtod_handle* h, int64_t slides, const void* pts) {
  const int B = pick_batch(h, slides);
  if (use_span(h) && B >= slides && slides >= 32 && !is_device_ptr(pts)) return (int)((slides + 1) / 2);
  return B;
}

int run_stream(rtod_handle* h, const void* pts, int64_t slides, int64_t ids_cap, cudaEvent_t e_begin,
               cudaEvent_t e_keys, cudaEvent_t e_end, std::vector<cudaEvent_t>* kev, BatchState* out_state,
               std::vector<int32_t>* nout, std::vector<int32_t>* nund, int64_t* out_ids = nullptr,
               bool* direct = nullptr) {
  const int64_t W = h->W, S = h->S;
  const int64_t used = W + slides * S;
  int r;
  const void* src;
  if ((r = ensure_records(h, slides))) return r;
  // Outlier IDs go straight to the caller's buffer when it is memory of this
  // device; otherwise to the handle's buffer and out in one copy by the
  // caller (one bulk copy beats scattered device writes into host memory).
  const bool to_user = out_ids && ids_cap > 0 && is_device_ptr(out_ids) && device_addressable(out_ids, h->device);
  // A page-locked host buffer gets the IDs from k_run_out at the end of the
  // pass, through its device mapping.
  int64_t* mapped_out = nullptr;
  if (out_ids && ids_cap > 0 && !to_user) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, out_ids) == cudaSuccess) {
      if (a.type == cudaMemoryTypeHost && a.devicePointer) mapped_out = static_cast<int64_t*>(a.devicePointer);
    } else {
      cudaGetLastError();
    }
  }
  if (direct) *direct = to_user || mapped_out;
  if (!to_user && (r = ensure_ids(h, std::max<int64_t>(1, std::min(ids_cap, slides * W))))) return r;
  int64_t* const dst = to_user ? out_ids : h->ids;
  const bool span = use_span(h);
  const int B = run_batch_size(h, slides, pts);
  if ((r = ensure_pool(h, B, !span))) return r;
  const int64_t chunk = span ? span_chunk(h, B, slides) : 0;
  if (span && (r = ensure_span(h, W / S + B - 1, chunk))) return r;
  bool host = false, pinned = false;
  if ((r = stage_stream(h, pts, used, &src, &host, false, &pinned))) return r;
  // first detected window: [S, W + S)
  if ((r = configure(h, MODE_RUN, B, S, src, !span, false))) return r;
  const int64_t blocks = used / S + 1;
  // A host stream is copied in pieces on a second stream: piece i holds the
  // points batch i needs beyond the earlier pieces ([0, W + B S) for the
  // first), so detection of a batch overlaps the copy of the next pieces.
  const int64_t nbatch = (slides + B - 1) / B;
  auto piece_end = [&](int64_t i) { return std::min(used, W + (i + 1) * (int64_t)B * S); };
  if (host) {
    if (!h->copy_stream) CU(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (!h->fork_ev) CU(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
    while ((int64_t)h->piece_ev.size() < nbatch) {
      cudaEvent_t e;
      CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      h->piece_ev.push_back(e);
    }
  }
  // the pieces, on the copy stream forked from the library stream
  auto copy_pieces = [&]() -> int {
    CU(cudaEventRecord(h->fork_ev, h->stream));
    CU(cudaStreamWaitEvent(h->copy_stream, h->fork_ev, 0));
    const int64_t D = h->D, es = h->esz;
    for (int64_t i = 0; i < nbatch; ++i) {
      const int64_t a = i ? piece_end(i - 1) : 0, e = piece_end(i);
      CU(cudaMemcpyAsync(h->run_buf + a * D * es, (const unsigned char*)pts + a * D * es, (size_t)((e - a) * D * es),
                         cudaMemcpyHostToDevice, h->copy_stream));
      CU(cudaEventRecord(h->piece_ev[(size_t)i], h->copy_stream));
    }
    return RTOD_OK;
  };
  const unsigned kgrid = (unsigned)h->sm_count * 8;
  // cell keys of points [a, b) (and their slide blocks' coordinate ranges),
  // after their piece has arrived; the span engine computes them in
  // k_span_hist
  auto keys = [&](int64_t i, int64_t a, int64_t b) -> int {
    if (host) CU(cudaStreamWaitEvent(h->stream, h->piece_ev[(size_t)i], 0));
    if (span) return RTOD_OK;
    const unsigned kx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((b - a + 255) / 256, kgrid));
    DISPATCH_DT(h->f64, h->D, CU(launch_k(k_keys<D, T>, dim3(kx), 256, h->stream, (const T*)src, a, b, 1.0 / h->cell,
                                          h->run_keys, h->run_prev, h->bs, h->S, h->run_blk_lo, h->run_blk_hi)));
    h->launches++;
    return RTOD_OK;
  };
  const int64_t out_cap = to_user ? ids_cap : std::min(ids_cap, h->ids_cap);
  const int64_t full = slides / B, rem = slides % B;
  Batch bfull = make_batch(h, B, out_cap, dst);
  const Span sfull = span ? make_span(h, B, src, chunk) : Span{};
  const int64_t chunk_batches = span ? chunk / B : 0;
  EventSet chunk_es;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> chunk_ev;
  if (span) bfull.span = h->span.sc;
  // a whole run as one graph: span engine, a device-resident or pinned host
  // stream (a graph's copy may not read pageable memory), no stage events
  const bool whole = span && (!host || pinned) && h->cfg.use_graph && !kev;
  // the span engine's learned router trains once per pass when due
  const bool train_pass = span && sfull.route && train_now(h);
  // Everything from the scratch resets to the last compaction.
  auto enqueue = [&]() -> int {
    // the pass starts here (a run graph: just before its launch)
    if (e_begin && !whole) CU(cudaEventRecord(e_begin, h->stream));
    if (!span) {  // +inf / -inf patterns for the atomic min / max of k_keys
      CU(cudaMemsetAsync(h->run_blk_lo, 0x7f, (size_t)(blocks * 3) * sizeof(long long), h->stream));
      CU(cudaMemsetAsync(h->run_blk_hi, 0x80, (size_t)(blocks * 3) * sizeof(long long), h->stream));
    }
    CU(launch_k(k_run_init, dim3(1), 256, h->stream, h->ctr, (int32_t)B, S, S, h->bs));
    h->launches++;
    int rr;
    if (host && (rr = copy_pieces())) return rr;
    if (!whole) CU(cudaEventRecord(h->ev[1], h->stream));  // start of the key kernel (profile)
    if ((rr = keys(0, 0, host ? piece_end(0) : used))) return rr;
    if (e_keys && !whole) CU(cudaEventRecord(e_keys, h->stream));
    for (int64_t i = 0; i < full + (rem ? 1 : 0); ++i) {
      Batch b = bfull;
      Span sp = sfull;
      if (i == full) {
        b = make_batch(h, (int)rem, out_cap, dst);
        if (span) {
          b.span = h->span.sc;
          sp = make_span(h, (int)rem, src, chunk);
        }
      }
      const Span* spp = span ? &sp : nullptr;
      if (host && i > 0 && (rr = keys(i, piece_end(i - 1), piece_end(i)))) return rr;
      if (kev) {
        cudaEvent_t* e = &(*kev)[(size_t)i * 8];
        CU(cudaEventRecord(e[0], h->stream));
        rr = launch_batch(h, b, false, e + 1, spp);
      } else {
        rr = (i < full && !whole) ? run_batch(h, b, false, spp) : launch_batch(h, b, false, nullptr, spp);
      }
      if (rr) return rr;
      const bool last = i + 1 == full + (rem ? 1 : 0);
      if (span && ((i + 1) % chunk_batches == 0 || last)) {
        const int64_t s1 = std::min(slides, (i + 1) * (int64_t)B);
        const int64_t s0 = ((s1 - 1) / chunk) * chunk;
        if (kev) {
          chunk_ev.emplace_back(chunk_es.make(), chunk_es.make());
          CU(cudaEventRecord(chunk_ev.back().first, h->stream));
        }
        if ((rr = span_flush(h, sfull, s0, s1 - s0, out_cap, dst))) return rr;
        if (kev) CU(cudaEventRecord(chunk_ev.back().second, h->stream));
      }
    }
    if (train_pass) {
      if ((rr = launch_train(geom_of(h), h->stream))) return rr;
      h->launches += 2;
    }
    // IDs to a page-locked caller buffer, the batch state to the mirror
    const unsigned ox = mapped_out ? (unsigned)h->sm_count * 2 : 1u;
    CU(launch_k(k_run_out, dim3(ox), 256, h->stream, (const int64_t*)dst, mapped_out, out_cap, h->bs,
                h->bs_mirror_dev));
    h->launches++;
    return RTOD_OK;
  };
  if (whole) {
    // key of the captured run: stream, sizes and the batch / span parameters
    std::vector<unsigned char> key(sizeof(void*) + 5 * sizeof(int64_t) + sizeof(Batch) + sizeof(Span));
    unsigned char* k = key.data();
    const int64_t ints[5] = {slides, out_cap, chunk, (int64_t)B, (int64_t)(intptr_t)mapped_out};
    std::memcpy(k, &pts, sizeof(void*));  // the caller's stream (host pieces are copied from it)
    std::memcpy(k + sizeof(void*), ints, sizeof ints);
    std::memcpy(k + sizeof(void*) + sizeof ints, &bfull, sizeof(Batch));
    std::memcpy(k + sizeof(void*) + sizeof ints + sizeof(Batch), &sfull, sizeof(Span));
    cudaGraphExec_t& rg = h->run_graph[train_pass ? 1 : 0];
    if (!rg || key != h->run_graph_key[train_pass ? 1 : 0]) {
      if (rg) cudaGraphExecDestroy(rg);
      rg = nullptr;
      const int64_t l0 = h->launches;
      cudaGraph_t g;
      CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      r = enqueue();
      cudaError_t e = cudaStreamEndCapture(h->stream, &g);
      if (r) return r;
      if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&rg, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
      h->run_graph_key[train_pass ? 1 : 0] = key;
      h->run_graph_kernels[train_pass ? 1 : 0] = h->launches - l0;
      h->launches = l0;
    }
    if (e_begin) CU(cudaEventRecord(e_begin, h->stream));
    CU(cudaGraphLaunch(rg, h->stream));
    h->launches += h->run_graph_kernels[train_pass ? 1 : 0];
    h->graph_replays++;
  } else {
    if ((r = enqueue())) return r;
  }
  if (e_end) CU(cudaEventRecord(e_end, h->stream));
  // Counters and per-slide records: written by the kernels into mapped
  // page-locked memory, read after a single wait.
  CU(cudaStreamSynchronize(h->stream));
  std::memcpy(out_state, h->bs_mirror, sizeof(BatchState));
  nout->assign(h->rec_nout_h, h->rec_nout_h + slides);
  nund->assign(h->rec_undet_h, h->rec_undet_h + slides);
  h->flush_ms = 0;
  for (const auto& pr : chunk_ev) h->flush_ms += elapsed(pr.first, pr.second);
  h->n_pushed = used;
  h->slides_done = slides;
  if ((r = check_device_error(h, *out_state))) return r;
  h->undet_total += out_state->undet_total;
  return RTOD_OK;
}

void free_all(rtod_handle* h) {
  drop_graph(h);
  for (Scratch& s : h->pool) {
    dfree(s.bin_count); dfree(s.bin_start); dfree(s.kmin); dfree(s.kmax); dfree(s.s_off);
    dfree(s.s_ckey); dfree(s.s_x); dfree(s.queue); dfree(s.feat); dfree(s.flags); dfree(s.scan_status);
    dfree(s.cmp_status);
  }
  h->pool.clear();
  free_span(h);
  free_grid(h);
  dfree(h->ctr); dfree(h->jobs_dev); dfree(h->bs); dfree(h->router); dfree(h->bar); dfree(h->ring); dfree(h->ring_keys);
  dfree(h->ring_prev); dfree(h->staging); dfree(h->run_buf); dfree(h->run_keys); dfree(h->run_prev);
  dfree(h->run_blk_lo); dfree(h->run_blk_hi);
  dfree(h->rec_base); dfree(h->ids);
  if (h->rec_host) cudaFreeHost(h->rec_host);
  h->rec_host = nullptr;
  h->rec_nout = h->rec_undet = h->rec_nout_h = h->rec_undet_h = nullptr;
  if (h->bs_mirror) cudaFreeHost(h->bs_mirror);
  h->bs_mirror = h->bs_mirror_dev = nullptr;
  if (h->stage_host) cudaFreeHost(h->stage_host);
  h->stage_host = nullptr;
  if (h->slide_host) cudaFreeHost(h->slide_host);
  h->slide_host = h->slide_host_dev = nullptr;
  if (h->ids_host) cudaFreeHost(h->ids_host);
  h->ids_host = h->ids_host_dev = nullptr;
  h->ids_host_cap = 0;
  if (h->ctr_init) cudaFreeHost(h->ctr_init);
  h->ctr_init = nullptr;
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto e : h->piece_ev) cudaEventDestroy(e);
  h->piece_ev.clear();
  if (h->fork_ev) cudaEventDestroy(h->fork_ev);
  h->fork_ev = nullptr;
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  h->copy_stream = nullptr;
  if (h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Autotuner: coordinate descent over the launch and grid parameters, each
// candidate timed (CUDA events, second of two passes) on a prefix of the
// stream. Results never depend on these parameters; only the time does.
// The best setting is cached per configuration for the rest of the process.
// ---------------------------------------------------------------------------
struct Tuning {
  int n = 2;
  int block_warps = 8;
  int batch = 32;
  float threshold = 0.5f;
  uint32_t max_sweep = 64;
  int engine = RTOD_ENGINE_WINDOW;
  int group = 0;
  int route = 1;  // span engine with the router on: route its counts (0: plain counts)
};

struct TuneEntry {
  rtod_config cfg;
  Tuning t;
};

std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune_cache;

bool same_problem(const rtod_config& a, const rtod_config& b) {
  return a.window == b.window && a.slide == b.slide && a.R == b.R && a.K == b.K && a.dim == b.dim &&
         a.opt == b.opt && a.pred == b.pred && a.router == b.router && a.device == b.device &&
         a.engine == b.engine && a.coord == b.coord && a.count == b.count;
}

int apply_tuning(rtod_handle* h, const Tuning& t) {
  set_grid(h, t.n);
  h->block_warps = t.block_warps;
  h->cfg.batch = t.batch;
  h->threshold = t.threshold;
  h->max_sweep = t.max_sweep;
  h->engine = t.engine;
  h->group = t.group;
  h->span_route = t.route;
  if (h->router) {
    CU(cudaMemcpy((char*)h->router + offsetof(RouterState, threshold), &t.threshold, sizeof(float),
                  cudaMemcpyHostToDevice));
    CU(cudaMemcpy((char*)h->router + offsetof(RouterState, max_sweep), &t.max_sweep, sizeof(uint32_t),
                  cudaMemcpyHostToDevice));
  }
  drop_graph(h);
  return RTOD_OK;
}

// Device ms of one pass over `slides` slides of a device-resident stream.
int time_pass(rtod_handle* h, const void* dev_pts, int64_t slides, float* ms) {
  EventSet es;
  cudaEvent_t a = es.make(), b = es.make();
  float best = 1e30f;
  for (int rep = 0; rep < 2; ++rep) {
    int r = reset_state(h);
    if (r) return r;
    BatchState s{};
    std::vector<int32_t> nout, nund;
    h->tuning_pass = true;  // the router trains between timed passes, not inside them
    CU(cudaEventRecord(a, h->stream));
    r = run_stream(h, dev_pts, slides, slides * h->W, nullptr, nullptr, nullptr, nullptr, &s, &nout, &nund);
    h->tuning_pass = false;
    if (r) return r;
    CU(cudaEventRecord(b, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    best = std::min(best, elapsed(a, b));
  }
  if (h->cfg.router) {  // on the samples the passes left
    if (int r = launch_train(geom_of(h), h->stream)) return r;
    CU(cudaStreamSynchronize(h->stream));
  }
  *ms = best;
  return RTOD_OK;
}

int autotune(rtod_handle* h, const void* pts, int64_t slides_total) {
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& e : g_tune_cache)
      if (same_problem(e.cfg, h->cfg)) {
        h->tuned = true;
        return apply_tuning(h, e.t);
      }
  }
  const int64_t W = h->W, S = h->S, D = h->D;
  const int64_t slides = std::min<int64_t>(slides_total, 256);
  const int64_t used = W + slides * S;
  // A private device copy of the prefix, so that trials never touch the caller's stream buffers.
  void* dev = nullptr;
  CU(cudaMalloc(&dev, (size_t)(used * D * h->esz)));
  struct Free {
    void* p;
    ~Free() { cudaFree(p); }
  } fr{dev};
  CU(cudaMemcpy(dev, pts, (size_t)(used * D * h->esz), cudaMemcpyDefault));
  Tuning best;
  best.batch = h->engine == RTOD_ENGINE_SPAN ? 32 : std::min(32, h->batch_max);
  best.engine = h->engine;
  best.group = h->group;
  int r = apply_tuning(h, best);
  if (r) return r;
  float best_ms;
  if ((r = time_pass(h, dev, slides, &best_ms))) return r;
  auto trial = [&](Tuning t) -> int {
    int rr = apply_tuning(h, t);
    if (rr) return rr;
    float ms;
    if ((rr = time_pass(h, dev, slides, &ms))) return rr;
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
    return RTOD_OK;
  };
  // engine x cells per R (the best cell width differs between the engines)
  {
    const Tuning start = best;
    for (int e : {RTOD_ENGINE_SPAN, RTOD_ENGINE_WINDOW}) {
      if (h->cfg.engine != RTOD_ENGINE_AUTO && e != start.engine) continue;
      for (int n : {1, 2, 3, 4, 6}) {
        if (n > 3 && h->D != 1) continue;
        if (e == start.engine && n == start.n) continue;  // the starting point, timed above
        Tuning t = start;
        t.engine = e;
        t.n = n;
        if ((r = trial(t))) return r;
      }
    }
  }
  if (best.engine == RTOD_ENGINE_WINDOW && h->cfg.count == RTOD_COUNT_AUTO) {
    Tuning t = best;
    t.group = !best.group;
    if ((r = trial(t))) return r;
  }
  for (int bw : {2, 4, 8}) {
    if (bw == best.block_warps) continue;
    Tuning t = best;
    t.block_warps = bw;
    if ((r = trial(t))) return r;
  }
  for (int bt : {8, 16, 32, 64, 128, 256}) {
    if (bt == best.batch || bt > (best.engine == RTOD_ENGINE_SPAN ? h->span_batch_max : h->batch_max)) continue;
    Tuning t = best;
    t.batch = bt;
    if ((r = trial(t))) return r;
  }
  if (h->cfg.router && best.engine == RTOD_ENGINE_SPAN) {
    // the span engine's routing: off (plain counts), every eligible run in
    // delta segments (threshold above 1), or the network's routing at a few
    // thresholds (it has trained on the trial passes so far)
    const Tuning start = best;
    {
      Tuning t = start;
      t.route = 0;
      if ((r = trial(t))) return r;
    }
    for (float th : {2.0f, 0.35f, 0.65f}) {
      Tuning t = start;
      t.route = 1;
      t.threshold = th;
      if ((r = trial(t))) return r;
    }
  }
  if (h->cfg.router && best.engine == RTOD_ENGINE_WINDOW && !best.group) {
    for (float th : {0.3f, 0.7f, 0.9f}) {
      Tuning t = best;
      t.threshold = th;
      if ((r = trial(t))) return r;
    }
    for (uint32_t ms : {32u, 128u, 512u}) {
      Tuning t = best;
      t.max_sweep = ms;
      if ((r = trial(t))) return r;
    }
  }
  if ((r = apply_tuning(h, best))) return r;
  if ((r = reset_state(h))) return r;
  CU(cudaStreamSynchronize(h->stream));
  h->tuned = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache.push_back(TuneEntry{h->cfg, best});
  g_tune_cache.back().cfg.batch = 0;
  return RTOD_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

RTOD_API const char* rtod_version(void) { return "rtod-b200 0.2 (sm_100a)"; }

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
    return fail(RTOD_ERR_NODEV, "device %d is sm_%d%d; this library is built for sm_100a only", cfg->device,
                prop.major, prop.minor);
  CU(cudaSetDevice(cfg->device));

  rtod_handle* h = new (std::nothrow) rtod_handle();
  if (!h) return fail(RTOD_ERR_ARG, "out of host memory");
  h->cfg = *cfg;
  h->device = cfg->device;
  h->sm_count = prop.multiProcessorCount;
  h->block_warps = cfg->block_warps ? cfg->block_warps : 8;
  h->W = cfg->window;
  h->S = cfg->slide;
  h->D = cfg->dim;
  h->f64 = cfg->coord == RTOD_COORD_F64;
  h->esz = h->f64 ? 8 : 4;
  h->Wp = ((h->W + 3) / 4) * 4 + 4;  // padded SoA row: float4 loads stay in bounds
  {
    volatile float rf = (float)cfg->R;
    volatile float r2f = rf * rf;
    h->R2f = r2f;
  }
  set_grid(h, cfg->cells_per_r ? cfg->cells_per_r : 2);
  // Engine of rtod_run: the span engine by default (with the router on, it
  // routes the span engine's counts; the tuner may pick the window engine).
  h->engine = cfg->engine == RTOD_ENGINE_WINDOW ? RTOD_ENGINE_WINDOW : RTOD_ENGINE_SPAN;
  // Engine of push/detect: the streaming grid engine where it applies.
  h->grid.on = grid_wanted(h);
  // Window-engine count: group counts where no cell is ever all-inlier and
  // a window holds enough points for long parts (auto_group), unless the
  // router (which routes single points) is on.
  h->group = cfg->count == RTOD_COUNT_GROUP ||
             (cfg->count == RTOD_COUNT_AUTO && !cfg->router && auto_group(h->D, h->W, h->sm_count));
  // Windows per rtod_run launch: up to 32, within ~1 GiB of scratch.
  const int64_t per_job = (int64_t)NB * 24 + h->W * (4 + 8 + 4 + 4) + h->Wp * h->D * 4 + h->W / 8;
  h->batch_max = (int)std::max<int64_t>(1, std::min<int64_t>(32, (1ll << 30) / per_job));
  if (cfg->batch) h->batch_max = cfg->batch;
  // Span engine: per window of a batch, room for its listed groups (16 bytes
  // each, at most min(W, NB)), one block row of the two per-block tables
  // (2 * 4 * NB bytes) and S points of span arrays; up to kMaxJobs windows
  // within ~2 GiB.
  {
    const int64_t per_win = 16 * std::min<int64_t>(h->W, NB) + 8 * (int64_t)NB + h->S * (4 + 4 * h->D);
    h->span_batch_max = (int)std::max<int64_t>(1, std::min<int64_t>(kMaxJobs, (2ll << 30) / per_win));
  }

  int64_t* c = &h->device_bytes;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && !dalloc(&h->ctr, (size_t)kMaxJobs, c) && !dalloc(&h->jobs_dev, (size_t)kMaxJobs, c) &&
       !dalloc(&h->bs, 1, c) && !dalloc(&h->ring, (size_t)(h->W * h->D * h->esz), c) &&
       !dalloc(&h->ring_keys, (size_t)h->W, c) && !dalloc(&h->ring_prev, (size_t)h->W, c) &&
       !dalloc(&h->staging, (size_t)(h->W * h->D * h->esz), c);
  ok = ok && cudaMallocHost((void**)&h->ctr_init, sizeof(JobCtr) * kMaxJobs) == cudaSuccess;
  ok = ok && !dalloc(&h->router, 1, c) && !dalloc(&h->bar, 1, c) &&
       cudaMemset(h->bar, 0, sizeof(GridBar)) == cudaSuccess;
  if (ok) {
    RouterState* init = new (std::nothrow) RouterState;
    ok = init != nullptr;
    if (ok) {
      init_router(init);
      ok = cudaMemcpy(h->router, init, sizeof(RouterState), cudaMemcpyHostToDevice) == cudaSuccess;
      delete init;
    }
  }
  ok = ok && cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM) ==
                 cudaSuccess;
  if (ok) {
    k_table<<<(TQ0 * TQ1 * TQ2 + 255) / 256, 256, 0, h->stream>>>(h->router);
    ok = cudaGetLastError() == cudaSuccess;
  }
  for (auto& e : h->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
  if (ok) ok = !ensure_pool(h, 1) && !ensure_ids(h, h->W);
  if (ok) ok = !reset_state(h) && cudaStreamSynchronize(h->stream) == cudaSuccess;
  if (!ok) {
    std::string msg = g_last_error.empty() ? "device allocation failed" : g_last_error;
    free_all(h);
    delete h;
    return fail(RTOD_ERR_CUDA, "%s", msg.c_str());
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

RTOD_API int rtod_get_tuning(const rtod_handle* h, int32_t out[5]) {
  if (!h || !out) return fail(RTOD_ERR_ARG, "null argument");
  out[0] = h->n;
  out[1] = h->block_warps;
  out[2] = h->D < 3 ? h->D : 3;
  out[3] = pick_batch(h, INT64_MAX);
  out[4] = use_span(h) ? RTOD_ENGINE_SPAN : RTOD_ENGINE_WINDOW;
  return RTOD_OK;
}

RTOD_API int rtod_get_count_mode(const rtod_handle* h, int32_t* mode) {
  if (!h || !mode) return fail(RTOD_ERR_ARG, "null argument");
  *mode = h->group ? RTOD_COUNT_GROUP : RTOD_COUNT_POINT;
  return RTOD_OK;
}

namespace {
// Tile 1 of a scan whose tile 0 never publishes: the look-back wait runs
// out after its bound, records the timeout and returns a partial prefix.
__global__ void k_wait_check(unsigned long long* status, BatchState* bs, uint32_t* out) {
  const uint32_t ex = warp_lookback(status, 1, 7, bs);
  if (threadIdx.x == 0) *out = ex;
}
}  // namespace

RTOD_API int rtod_check_bounded_wait(int32_t device, int32_t* timed_out, double* ms) {
  if (!timed_out || !ms) return fail(RTOD_ERR_ARG, "null argument");
  *timed_out = 0;
  *ms = 0;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return fail(RTOD_ERR_NODEV, "bad device ordinal %d", device);
  }
  CU(cudaSetDevice(device));
  unsigned long long* status = nullptr;
  BatchState* bs = nullptr;
  uint32_t* out = nullptr;
  int64_t bytes = 0;
  struct Free {
    unsigned long long*& a;
    BatchState*& b;
    uint32_t*& c;
    ~Free() { dfree(a); dfree(b); dfree(c); }
  } fr{status, bs, out};
  if (dalloc(&status, 2, &bytes) || dalloc(&bs, 1, &bytes) || dalloc(&out, 1, &bytes)) return RTOD_ERR_CUDA;
  CU(cudaMemset(status, 0, 2 * sizeof(unsigned long long)));  // tile 0 never publishes
  CU(cudaMemset(bs, 0, sizeof(BatchState)));
  EventSet es;
  cudaEvent_t a = es.make(), b = es.make();
  CU(cudaEventRecord(a, 0));
  k_wait_check<<<1, 32>>>(status, bs, out);
  CU(cudaGetLastError());
  CU(cudaEventRecord(b, 0));
  CU(cudaEventSynchronize(b));
  BatchState hs{};
  CU(cudaMemcpy(&hs, bs, sizeof hs, cudaMemcpyDeviceToHost));
  *ms = elapsed(a, b);
  *timed_out = hs.err == DERR_TIMEOUT ? 1 : 0;
  return RTOD_OK;
}

RTOD_API int rtod_get_stats(const rtod_handle* h, int64_t out[5]) {
  if (!h || !out) return fail(RTOD_ERR_ARG, "null argument");
  out[0] = h->launches;
  out[1] = h->graph_replays;
  out[2] = h->slides_done;
  out[3] = h->undet_total;
  out[4] = h->device_bytes;
  return RTOD_OK;
}

RTOD_API int rtod_get_stream_engine(const rtod_handle* h, int64_t out[4]) {
  if (!h || !out) return fail(RTOD_ERR_ARG, "null argument");
  out[0] = h->grid.on ? RTOD_ENGINE_GRID : RTOD_ENGINE_WINDOW;
  out[1] = h->grid.builds;
  out[2] = h->grid.g.pool;
  out[3] = 0;
  if (h->grid.on && h->grid.g.ctl) {
    GridCtl c{};
    CU(cudaSetDevice(h->device));
    CU(cudaStreamSynchronize(h->stream));
    CU(cudaMemcpy(&c, h->grid.g.ctl, sizeof c, cudaMemcpyDeviceToHost));
    out[3] = c.max_occ;
  }
  return RTOD_OK;
}

RTOD_API int rtod_set_grid_pool(rtod_handle* h, int64_t slots) {
  if (!h) return fail(RTOD_ERR_ARG, "handle is null");
  if (slots < 1024 || (uint64_t)slots > kGridMaxPool)
    return fail(RTOD_ERR_ARG, "pool slots must be in [1024, 2^31]");
  if (h->n_pushed != 0) return fail(RTOD_ERR_STATE, "set the pool before the first push (or after rtod_reset)");
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->stream));
  free_grid_pool(h);
  drop_graph(h);
  h->grid.pool_first = (uint64_t)slots;
  return RTOD_OK;
}

RTOD_API const char* rtod_kernel_name(int32_t i) { return (i >= 0 && i < kPipeKernels) ? kKernelNames[i] : nullptr; }

namespace {

// The coordinate type of a call must be the handle's.
int check_coord(const rtod_handle* h, bool f64) {
  if (h->f64 != (int)f64)
    return fail(RTOD_ERR_ARG, h->f64 ? "this handle stores double coordinates: use the _f64 entry points"
                                     : "this handle stores float coordinates: use the float entry points");
  return RTOD_OK;
}

// Points the streaming job's slide source (Job::stage, read by the ingest
// kernels) at `stage`: the mapped page-locked slide of a host push, or the
// device staging buffer. The job table is read by the kernels at run time,
// so captured graphs stay valid.
int set_ring_stage(rtod_handle* h, const void* stage) {
  if (h->tab_host.empty() || h->tab_host[0].stage == stage) return RTOD_OK;
  h->tab_host[0].stage = stage;
  CU(cudaMemcpyAsync(reinterpret_cast<unsigned char*>(h->jobs_dev) + offsetof(Job, stage), &h->tab_host[0].stage,
                     sizeof(void*), cudaMemcpyHostToDevice, h->stream));
  CU(cudaStreamSynchronize(h->stream));  // the source lives in tab_host, which configure may replace
  return RTOD_OK;
}

int push_impl(rtod_handle* h, const void* pts, int64_t n, bool f64) {
  if (!h || !pts) return fail(RTOD_ERR_ARG, "null argument");
  if (int r = check_coord(h, f64)) return r;
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  CU(cudaSetDevice(h->device));
  const int64_t W = h->W, S = h->S, D = h->D;
  if (h->n_pushed == 0) {
    if (n != W) return fail(RTOD_ERR_STATE, "the first push must hold exactly W=%lld points", (long long)W);
  } else {
    if (h->mode != MODE_RING) return fail(RTOD_ERR_STATE, "the handle is not streaming; call rtod_reset");
    if (h->pending) return fail(RTOD_ERR_STATE, "rtod_detect must follow each slide push");
    if (n != S) return fail(RTOD_ERR_STATE, "a slide push must hold exactly S=%lld points", (long long)S);
  }
  const size_t bytes = (size_t)(n * D * h->esz);
  if (h->n_pushed > 0 && !is_device_ptr(pts)) {
    // A slide from host memory: copied on the host into a mapped page-locked
    // buffer (the caller may reuse its buffer at once) that the detection's
    // ingest kernel reads in place over the bus: no copy operation, whose
    // completion the first kernel would wait for. The previous detection has
    // finished with the buffer: every detection ends with a wait.
    if (!h->slide_host) {
      CU(cudaHostAlloc(&h->slide_host, (size_t)(S * D * h->esz), cudaHostAllocMapped));
      CU(cudaHostGetDevicePointer(&h->slide_host_dev, h->slide_host, 0));
    }
    std::memcpy(h->slide_host, pts, bytes);
    if (int r = set_ring_stage(h, h->slide_host_dev)) return r;
    CU(cudaEventRecord(h->ev[4], h->stream));
    CU(cudaEventRecord(h->ev[5], h->stream));
  } else {
    if (h->n_pushed > 0)
      if (int r = set_ring_stage(h, h->staging)) return r;
    CU(cudaEventRecord(h->ev[4], h->stream));
    CU(cudaMemcpyAsync(h->staging, pts, bytes, cudaMemcpyDefault, h->stream));
    CU(cudaEventRecord(h->ev[5], h->stream));
    // a slide in device memory may be overwritten once the push returns
    if (h->n_pushed > 0) CU(cudaEventSynchronize(h->ev[5]));
  }
  if (h->n_pushed == 0) {
    int r = configure(h, MODE_RING, 1, S, nullptr);  // first detected window: [S, W + S)
    if (r) return r;
    const Batch b = make_batch(h, 1, h->ids_cap);
    const int64_t gx = std::max<int64_t>(1, std::min<int64_t>((W + 255) / 256, h->sm_count * 8));
    DISPATCH_DT(h->f64, h->D, CU(launch_k(k_ingest<D, T>, dim3((unsigned)gx, 1), 256, h->stream, b, 1)));
    h->launches++;
    BatchState s;
    CU(cudaMemcpyAsync(&s, h->bs, sizeof s, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    r = check_device_error(h, s);
    if (r) return r;
    if (h->grid.on && (r = grid_build(h, 0))) return r;
  } else {
    h->pending = true;
    if (h->eager) {
      // the detection follows the copy on the stream at once; rtod_detect waits for it
      if (int r = ensure_detect_out(h)) return r;
      CU(cudaEventRecord(h->ev[0], h->stream));
      if (int r = run_batch(h, make_batch(h, 1, h->ids_cap), true)) return r;
      CU(cudaEventRecord(h->ev[7], h->stream));
      h->launched = true;
    }
  }
  h->n_pushed += n;
  return RTOD_OK;
}

}  // namespace

RTOD_API int rtod_push_slide(rtod_handle* h, const float* pts, int64_t n) { return push_impl(h, pts, n, false); }

RTOD_API int rtod_push_slide_f64(rtod_handle* h, const double* pts, int64_t n) { return push_impl(h, pts, n, true); }


RTOD_API int rtod_detect(rtod_handle* h, int64_t* out_ids, int64_t cap, int64_t* n_out, rtod_times* times) {
  if (!h || !n_out || (cap > 0 && !out_ids)) return fail(RTOD_ERR_ARG, "null argument");
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  if (!h->pending) return fail(RTOD_ERR_STATE, "no pushed slide to detect");
  CU(cudaSetDevice(h->device));
  if (int r0 = ensure_detect_out(h)) return r0;
  const Batch b = make_batch(h, 1, h->ids_cap);
  cudaEvent_t kev[7];
  EventSet es;
  const bool split = times && !h->launched;  // stage events need the detection launched here
  int r = RTOD_OK;
  if (!h->launched) {
    if (split) {
      for (auto& e : kev) e = es.make();
      CU(cudaEventRecord(h->ev[0], h->stream));
    }
    r = split ? launch_batch(h, b, true, kev) : run_batch(h, b, true);
    if (r) return r;
    if (split) CU(cudaEventRecord(h->ev[7], h->stream));
  }
  const bool was_launched = h->launched;
  h->launched = false;
  h->eager = times == nullptr;
  // The IDs and the batch state arrive in the mapped landing buffers
  // (k_run_out, the graph's last kernel): one wait.
  CU(cudaStreamSynchronize(h->stream));
  BatchState s;
  std::memcpy(&s, h->bs_mirror, sizeof s);
  if (s.err == DERR_GRID && h->grid.on) {
    if ((r = grid_recount(h, b))) return r;
    std::memcpy(&s, h->bs_mirror, sizeof s);
  }
  h->pending = false;
  r = check_device_error(h, s);
  if (r) return r;
  h->slides_done++;
  h->undet_total = s.undet_total;
  *n_out = s.out_total;
  if (s.out_total > cap)
    return fail(RTOD_ERR_CAPACITY, "%lld outliers but room for %lld", (long long)s.out_total, (long long)cap);
  if (s.out_total > 0) {
    if (is_device_ptr(out_ids)) {
      CU(cudaMemcpyAsync(out_ids, h->ids, (size_t)s.out_total * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                         h->stream));
      CU(cudaStreamSynchronize(h->stream));
    } else {
      std::memcpy(out_ids, h->ids_host, (size_t)s.out_total * sizeof(int64_t));
    }
  }
  if (times) {
    std::memset(times, 0, sizeof *times);
    times->copy_new_points_h2d = elapsed(h->ev[4], h->ev[5]);
    if (!was_launched) {
      times->prepare_cell = elapsed(h->ev[0], kev[1]);   // ring update + occupancy
      times->build_bvh = elapsed(kev[1], kev[3]);       // scan + scatter
      times->detect_outlier = elapsed(kev[3], kev[5]);  // count + compact
      times->copy_outlier_d2h = elapsed(kev[6], h->ev[7]);  // after the compaction's delivery
    }
    times->total = times->copy_new_points_h2d + elapsed(h->ev[0], h->ev[7]);
    times->undetermined_per_slide = (double)s.undet_total;
    times->slides = 1;
  }
  return RTOD_OK;
}

namespace {

int run_impl(rtod_handle* h, const void* pts, int64_t n, int64_t max_slides, int64_t* out_offsets,
             int64_t* out_ids, int64_t ids_cap, int64_t* slides_out, rtod_times* times, bool f64) {
  if (!h || !pts || !out_offsets || !slides_out || (ids_cap > 0 && !out_ids))
    return fail(RTOD_ERR_ARG, "null argument");
  if (int r = check_coord(h, f64)) return r;
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  if (h->n_pushed != 0) return fail(RTOD_ERR_STATE, "rtod_run needs a fresh handle (call rtod_reset)");
  if (n < 0 || ids_cap < 0) return fail(RTOD_ERR_ARG, "negative size");
  CU(cudaSetDevice(h->device));
  out_offsets[0] = 0;
  const int64_t slides = count_slides(h, n, max_slides);
  *slides_out = slides;
  if (slides == 0) return RTOD_OK;
  if (h->cfg.tuner && !h->tuned) {
    int rt = autotune(h, pts, slides);
    if (rt) return rt;
  }
  EventSet es;
  cudaEvent_t t0 = h->ev[8], t1 = h->ev[9], t2 = h->ev[10], d0 = h->ev[11], d1 = h->ev[12];
  // Stage split (only without graphs): events around every kernel of every batch.
  std::vector<cudaEvent_t> kev;
  const bool stage = times && !h->cfg.use_graph;
  if (stage) {
    const int B = run_batch_size(h, slides, pts);
    kev.resize((size_t)((slides + B - 1) / B) * 8);
    for (auto& e : kev) e = es.make();
  }
  BatchState s{};
  std::vector<int32_t> nout, nund;
  bool direct = false;
  int r = run_stream(h, pts, slides, ids_cap, t0, t1, t2, stage ? &kev : nullptr, &s, &nout, &nund, out_ids,
                     &direct);
  if (r) return r;
  for (int64_t j = 0; j < slides; ++j) out_offsets[j + 1] = out_offsets[j] + nout[j];
  if (out_offsets[slides] != s.out_total) return fail(RTOD_ERR_CUDA, "inconsistent outlier totals");
  // IDs still in the handle's buffer (a pageable host destination): one copy
  const bool copy_out = !direct && s.out_total > 0;
  if (copy_out) {
    CU(cudaEventRecord(d0, h->stream));
    CU(cudaMemcpyAsync(out_ids, h->ids, (size_t)s.out_total * sizeof(int64_t), cudaMemcpyDefault, h->stream));
    CU(cudaEventRecord(d1, h->stream));
    CU(cudaStreamSynchronize(h->stream));
  }
  if (times) {
    std::memset(times, 0, sizeof *times);
    const double inv = 1.0 / (double)slides;
    const double d2h = copy_out ? elapsed(d0, d1) : 0.0;  // otherwise inside the pass (k_run_out)
    times->slides = slides;
    times->copy_outlier_d2h = d2h * inv;
    if (stage) {
      const int64_t nb = (int64_t)kev.size() / 8;
      double pc = elapsed(t0, t1), bb = 0, de = 0;  // input copy + cell keys count as preparing cells
      for (int64_t i = 0; i < nb; ++i) {
        const cudaEvent_t* e = &kev[(size_t)i * 8];
        pc += elapsed(e[0], e[2]);  // hist
        bb += elapsed(e[2], e[4]);  // scan + scatter
        de += elapsed(e[4], e[7]);  // count + compact (+ router training)
      }
      de += h->flush_ms;  // span engine: compaction once per chunk of slides
      times->prepare_cell = pc * inv;
      times->build_bvh = bb * inv;
      times->detect_outlier = de * inv;
    }
    // Everything on the library stream from the start of the pass (input
    // copy, counters) to its last kernel (which also delivers the IDs to a
    // device or page-locked buffer), plus the copy to a pageable buffer; only
    // the host's wait is outside.
    times->total = (elapsed(t0, t2) + d2h) * inv;
    times->undetermined_per_slide = (double)s.undet_total * inv;
  }
  return RTOD_OK;
}

}  // namespace

RTOD_API int rtod_run(rtod_handle* h, const float* pts, int64_t n, int64_t max_slides, int64_t* out_offsets,
                      int64_t* out_ids, int64_t ids_cap, int64_t* slides_out, rtod_times* times) {
  return run_impl(h, pts, n, max_slides, out_offsets, out_ids, ids_cap, slides_out, times, false);
}

RTOD_API int rtod_run_f64(rtod_handle* h, const double* pts, int64_t n, int64_t max_slides, int64_t* out_offsets,
                          int64_t* out_ids, int64_t ids_cap, int64_t* slides_out, rtod_times* times) {
  return run_impl(h, pts, n, max_slides, out_offsets, out_ids, ids_cap, slides_out, times, true);
}


RTOD_API int rtod_profile_run(rtod_handle* h, const float* pts, int64_t n, int64_t max_slides, double* kernel_ms,
                              int32_t n_kernels) {
  if (!h || !pts || !kernel_ms || n_kernels < 1) return fail(RTOD_ERR_ARG, "null argument");
  if (int r = check_coord(h, false)) return r;
  if (h->poisoned) return fail(RTOD_ERR_STATE, "handle is in an error state; call rtod_reset");
  if (h->n_pushed != 0) return fail(RTOD_ERR_STATE, "rtod_profile_run needs a fresh handle");
  CU(cudaSetDevice(h->device));
  const int64_t slides = count_slides(h, n, max_slides);
  if (slides == 0) return fail(RTOD_ERR_ARG, "stream shorter than one slide");
  const int B = run_batch_size(h, slides, pts);
  const int64_t nb = (slides + B - 1) / B;
  EventSet es;
  cudaEvent_t t0 = es.make(), t1 = es.make();
  std::vector<cudaEvent_t> kev((size_t)nb * 8);
  for (auto& e : kev) e = es.make();
  BatchState s{};
  std::vector<int32_t> nout, nund;
  int r = run_stream(h, pts, slides, slides * h->W, t0, t1, nullptr, &kev, &s, &nout, &nund);
  if (r) return r;
  for (int i = 0; i < n_kernels; ++i) kernel_ms[i] = 0;
  kernel_ms[0] = elapsed(h->ev[1], t1);  // cell keys of the stream
  for (int64_t i = 0; i < nb; ++i) {
    const cudaEvent_t* e = &kev[(size_t)i * 8];
    for (int k = 1; k < kPipeKernels && k < n_kernels; ++k) kernel_ms[k] += elapsed(e[k], e[k + 1]);
  }
  if (n_kernels > 6) kernel_ms[6] += h->flush_ms;  // span engine: compaction once per chunk
  for (int i = 0; i < n_kernels; ++i) kernel_ms[i] /= (double)slides;
  return RTOD_OK;
}

// ---------------------------------------------------------------------------
// Router diagnostics and test entry points
// ---------------------------------------------------------------------------

RTOD_API int rtod_router_info(rtod_handle* h, float* params, double info[6]) {
  if (!h || !info) return fail(RTOD_ERR_ARG, "null argument");
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->stream));
  RouterState* r = new (std::nothrow) RouterState;
  if (!r) return fail(RTOD_ERR_ARG, "out of host memory");
  cudaError_t e = cudaMemcpy(r, h->router, sizeof(RouterState), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    delete r;
    return fail(RTOD_ERR_CUDA, "router read failed: %s", cudaGetErrorString(e));
  }
  if (params) std::memcpy(params, r->params, sizeof(float) * MLP_P);
  info[0] = (double)r->steps;
  info[1] = (double)r->last_loss;
  info[2] = (double)r->routed_early;
  info[3] = (double)r->routed_sweep;
  info[4] = (double)r->misrouted;
  info[5] = (double)r->threshold;
  delete r;
  return RTOD_OK;
}

RTOD_API int rtod_router_set_threshold(rtod_handle* h, float threshold) {
  if (!h) return fail(RTOD_ERR_ARG, "handle is null");
  if (!(threshold >= 0.0f) || !(threshold <= 2.0f)) return fail(RTOD_ERR_ARG, "threshold must be in [0, 2]");
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->stream));
  CU(cudaMemcpy((char*)h->router + offsetof(RouterState, threshold), &threshold, sizeof(float),
                cudaMemcpyHostToDevice));
  h->threshold = threshold;
  return RTOD_OK;
}

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

RTOD_API int rtod_mlp_param_count(void) { return MLP_P; }

RTOD_API int rtod_mlp_forward(int32_t device, const float* params, const float* x, int64_t n, float* logits) {
  if (!params || !x || !logits || n < 1 || n > (1 << 24)) return fail(RTOD_ERR_ARG, "bad argument");
  CU(cudaSetDevice(device));
  DevBuf dp, dx, dz;
  CU(cudaMalloc(&dp.p, sizeof(float) * MLP_P));
  CU(cudaMalloc(&dx.p, sizeof(float) * MLP_IN * n));
  CU(cudaMalloc(&dz.p, sizeof(float) * MLP_B * n));
  CU(cudaMemcpy(dp.p, params, sizeof(float) * MLP_P, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dx.p, x, sizeof(float) * MLP_IN * n, cudaMemcpyHostToDevice));
  k_mlp_forward<<<(unsigned)((n + 255) / 256), 256>>>((float*)dp.p, (float*)dx.p, (int)n, (float*)dz.p);
  CU(cudaGetLastError());
  CU(cudaMemcpy(logits, dz.p, sizeof(float) * MLP_B * n, cudaMemcpyDeviceToHost));
  return RTOD_OK;
}

RTOD_API int rtod_mlp_grad(int32_t device, const float* params, const float* x, const int32_t* y, int64_t n,
                           float* grad, float* loss) {
  if (!params || !x || !y || !grad || !loss || n < 1 || n > (1 << 20)) return fail(RTOD_ERR_ARG, "bad argument");
  for (int64_t i = 0; i < n; ++i)
    if (y[i] < 0 || y[i] >= MLP_B) return fail(RTOD_ERR_ARG, "label out of range");
  CU(cudaSetDevice(device));
  CU(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
  DevBuf dp, dx, dy, dg, dl, dyf;
  CU(cudaMalloc(&dp.p, sizeof(float) * MLP_P));
  CU(cudaMalloc(&dx.p, sizeof(float) * MLP_IN * n));
  CU(cudaMalloc(&dy.p, sizeof(int32_t) * n));
  CU(cudaMalloc(&dyf.p, sizeof(float) * n));
  CU(cudaMalloc(&dg.p, sizeof(float) * MLP_P));
  CU(cudaMalloc(&dl.p, sizeof(float)));
  CU(cudaMemcpy(dp.p, params, sizeof(float) * MLP_P, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dx.p, x, sizeof(float) * MLP_IN * n, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dy.p, y, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  k_mlp_grad<<<1, 256, TRAIN_SMEM>>>((float*)dp.p, (float*)dx.p, (int32_t*)dy.p, (int)n, (float*)dg.p,
                                     (float*)dl.p, (float*)dyf.p);
  CU(cudaGetLastError());
  CU(cudaMemcpy(grad, dg.p, sizeof(float) * MLP_P, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
  return RTOD_OK;
}

RTOD_API int rtod_mlp_adam(int32_t device, float* params, float* m, float* v, int32_t t, const float* x,
                           const int32_t* y, int64_t n, float lr, float* loss) {
  if (!params || !m || !v || !x || !y || !loss || n < 1 || n > (1 << 20) || t < 1)
    return fail(RTOD_ERR_ARG, "bad argument");
  for (int64_t i = 0; i < n; ++i)
    if (y[i] < 0 || y[i] >= MLP_B) return fail(RTOD_ERR_ARG, "label out of range");
  CU(cudaSetDevice(device));
  CU(cudaFuncSetAttribute(k_mlp_adam, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM));
  const float beta1 = 0.9f, beta2 = 0.999f;
  float bt[2] = {std::pow(beta1, (float)(t - 1)), std::pow(beta2, (float)(t - 1))};
  DevBuf dp, dm, dv, dbt, dx, dy, dl, dyf;
  CU(cudaMalloc(&dp.p, sizeof(float) * MLP_P));
  CU(cudaMalloc(&dm.p, sizeof(float) * MLP_P));
  CU(cudaMalloc(&dv.p, sizeof(float) * MLP_P));
  CU(cudaMalloc(&dbt.p, sizeof(float) * 2));
  CU(cudaMalloc(&dx.p, sizeof(float) * MLP_IN * n));
  CU(cudaMalloc(&dy.p, sizeof(int32_t) * n));
  CU(cudaMalloc(&dyf.p, sizeof(float) * n));
  CU(cudaMalloc(&dl.p, sizeof(float)));
  CU(cudaMemcpy(dp.p, params, sizeof(float) * MLP_P, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dm.p, m, sizeof(float) * MLP_P, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dv.p, v, sizeof(float) * MLP_P, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dbt.p, bt, sizeof(float) * 2, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dx.p, x, sizeof(float) * MLP_IN * n, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dy.p, y, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  k_mlp_adam<<<1, 256, TRAIN_SMEM>>>((float*)dp.p, (float*)dm.p, (float*)dv.p, (float*)dbt.p, (float*)dx.p,
                                     (int32_t*)dy.p, (int)n, lr, beta1, beta2, 1e-8f, (float*)dl.p, (float*)dyf.p);
  CU(cudaGetLastError());
  CU(cudaMemcpy(params, dp.p, sizeof(float) * MLP_P, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(m, dm.p, sizeof(float) * MLP_P, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(v, dv.p, sizeof(float) * MLP_P, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
  return RTOD_OK;
}

// ---------------------------------------------------------------------------
// Batched streams
// ---------------------------------------------------------------------------

struct rtod_batch {
  int device = 0;
  int n = 0;
  int route = 0;
  int fused = 0;  // RTOD_PIPELINE_FUSED: one cooperative launch per group and step
  cudaStream_t stream = nullptr;
  std::vector<rtod_handle*> hs;
  struct Group {
    Geom geom{};
    std::vector<int> streams;
    Job* jobs = nullptr;
    BatchState* bs = nullptr;
    int64_t* out = nullptr;
    int64_t out_cap = 0;
    int32_t* active = nullptr;    // device [n in group]
    int32_t* active_h = nullptr;  // pinned host
    int32_t* nout = nullptr;      // device [n in group]
    int32_t* nout_h = nullptr;    // pinned host
    BatchState* bs_h = nullptr;   // pinned host
    int64_t cmp_tiles = 0;
    GridBar* bar = nullptr;       // grid barrier of the group's fused launch
    int fused_grid = 0;
    // Autotuner (rtod_config.tuner): settings tried one per step, each timed
    // on the device around the group's launches, `rounds` times over.
    struct Setting {
      int n, bw, group;
    };
    Setting cur{2, 8, 0};
    std::vector<Setting> cand;
    std::vector<float> ms;
    int idx = 0, round = 0;
    bool tuned = true;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;      // the group's branch of a captured step (groups overlap)
    cudaEvent_t join = nullptr;     // end of that branch
  };
  std::vector<Group> groups;
  RouterState* router = nullptr;
  std::vector<char> filled, pending;
  bool tuning = false;   // the autotuner is still trying settings (no graph replay meanwhile)
  int tune_rounds = 2;
  int64_t tune_steps = 0;
  cudaGraphExec_t graphs[2] = {nullptr, nullptr};  // without / with the router's training step
  int64_t graph_kernels[2] = {0, 0};
  int64_t steps = 0, launches = 0, detections = 0;
  cudaEvent_t fork = nullptr;  // start of a captured step whose groups run as parallel branches
};

namespace {

void batch_free(rtod_batch* b) {
  for (auto g : b->graphs)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : b->groups) {
    if (g.e0) cudaEventDestroy(g.e0);
    if (g.e1) cudaEventDestroy(g.e1);
    if (g.join) cudaEventDestroy(g.join);
    if (g.st) cudaStreamDestroy(g.st);
    dfree(g.jobs); dfree(g.bs); dfree(g.out); dfree(g.active); dfree(g.nout); dfree(g.bar);
    if (g.active_h) cudaFreeHost(g.active_h);
    if (g.nout_h) cudaFreeHost(g.nout_h);
    if (g.bs_h) cudaFreeHost(g.bs_h);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  dfree(b->router);
  for (auto* h : b->hs)
    if (h) rtod_destroy(h);
  if (b->stream) cudaStreamDestroy(b->stream);
}

Batch group_batch(const rtod_batch::Group& g, RouterState* router) {
  Batch bt{};
  bt.jobs = g.jobs;
  bt.njobs = (int32_t)g.streams.size();
  bt.bs = g.bs;
  bt.router = router;
  bt.out_ids = g.out;
  bt.out_cap = g.out_cap;
  bt.cmp_tiles = g.cmp_tiles;
  bt.active = g.active;
  bt.job_nout = g.nout;
  return bt;
}

// One step for all groups: active flags in, counters reset, pipeline, counts out.
int batch_enqueue(rtod_batch* b, bool train, int64_t* nk_total, bool timed = false, bool branches = false) {
  int64_t total = 0;
  // branches (a captured step with several groups): each group on its own
  // stream, forked from and joined back into the step's stream, so that the
  // graph runs the groups side by side. The groups share no device state
  // (jobs, counters, outputs and flags are per group) except the router,
  // which every routed group reads and trains: the routed groups form one
  // branch, one after another. Cooperative fused launches keep one branch.
  branches = branches && b->groups.size() > 1 && !b->fused;
  if (branches) CU(cudaEventRecord(b->fork, b->stream));
  cudaStream_t routed_st = nullptr;  // the routed groups' branch
  for (auto& g : b->groups) {
    cudaStream_t st = b->stream;
    if (branches) {
      st = g.st;
      if (g.geom.route) {
        if (routed_st) st = routed_st;  // follows the previous routed group
        else routed_st = st;
      }
      if (st == g.st) CU(cudaStreamWaitEvent(st, b->fork, 0));
    }
    const int ng = (int)g.streams.size();
    CU(cudaMemcpyAsync(g.active, g.active_h, sizeof(int32_t) * ng, cudaMemcpyHostToDevice, st));
    if (timed) CU(cudaEventRecord(g.e0, st));
    int64_t nk = 0;
    int r;
    if (b->fused) {
      r = launch_fused(g.geom, group_batch(g, b->router), g.bar, true, nullptr, 0, nullptr, train, st,
                       &g.fused_grid, &nk);
    } else {
      r = launch_group(g.geom, group_batch(g, b->router), true, train, st, nullptr, &nk);
    }
    if (r) return r;
    total += nk;
    if (timed) CU(cudaEventRecord(g.e1, st));
    CU(cudaMemcpyAsync(g.nout_h, g.nout, sizeof(int32_t) * ng, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(g.bs_h, g.bs, sizeof(BatchState), cudaMemcpyDeviceToHost, st));
    if (branches) CU(cudaEventRecord(g.join, st));
  }
  if (branches)
    for (auto& g : b->groups) CU(cudaStreamWaitEvent(b->stream, g.join, 0));
  *nk_total = total;
  return RTOD_OK;
}

// Job table of a group from its streams' current settings.
int upload_group_jobs(rtod_batch* b, rtod_batch::Group& g) {
  const int ng = (int)g.streams.size();
  std::vector<Job> tab(ng);
  for (int k = 0; k < ng; ++k) tab[k] = make_job(b->hs[g.streams[k]], 0, true, nullptr);
  for (auto& jb : tab) jb.gpts = group_part_size(g.out_cap, b->hs[g.streams[0]]->sm_count);
  CU(cudaMemcpy(g.jobs, tab.data(), sizeof(Job) * ng, cudaMemcpyHostToDevice));
  return RTOD_OK;
}

// Applies a setting to a group: cell width (its streams' ring keys are
// recomputed), count block shape and count mode. Results do not depend on
// any of them.
int apply_group_setting(rtod_batch* b, rtod_batch::Group& g, const rtod_batch::Group::Setting& st,
                        bool rings_filled = true) {
  const bool rekey = st.n != g.cur.n;
  for (int s : g.streams) {
    rtod_handle* h = b->hs[s];
    if (rekey) set_grid(h, st.n);
    h->group = st.group;
    h->block_warps = st.bw;
  }
  if (st.group != g.cur.group) g.fused_grid = 0;  // another kernel instantiation: residency found again
  g.geom.block_warps = st.bw;
  g.geom.group = st.group;
  g.geom.route = b->route && !st.group;
  if (int r = upload_group_jobs(b, g)) return r;
  if (rekey && rings_filled) {
    // the rings of the streams that hold a window
    std::vector<int32_t> filled(g.streams.size());
    for (size_t k = 0; k < g.streams.size(); ++k) filled[k] = b->filled[g.streams[k]] ? 1 : 0;
    CU(cudaMemcpy(g.active, filled.data(), sizeof(int32_t) * filled.size(), cudaMemcpyHostToDevice));
    Batch bt = group_batch(g, b->router);
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((g.geom.Wmax + 255) / 256, 1024));
    DISPATCH_D(g.geom.D, CU(launch_k(k_rekey<D, float>, dim3(gx, (unsigned)g.streams.size()), 256, b->stream, bt)));
  }
  g.cur = st;
  return RTOD_OK;
}

// Candidate settings of a group: cell widths x block shapes (and, beyond 3
// dimensions, both count modes), except what the streams' configs fix.
void init_group_tuning(rtod_batch* b, rtod_batch::Group& g, const rtod_config& c) {
  std::vector<int> ns, bws, gs;
  if (c.cells_per_r) ns = {c.cells_per_r};
  else if (g.geom.D == 1) ns = {2, 3, 4};
  else if (g.geom.D <= 3) ns = {1, 2, 3};
  else ns = {1, 2};
  if (c.block_warps) bws = {c.block_warps};
  else if (g.geom.D <= 3) bws = {2, 4, 8};
  else bws = {4, 8};
  if (c.count != RTOD_COUNT_AUTO || g.geom.D <= 3) gs = {g.cur.group};
  else gs = {1, 0};
  g.cand.clear();
  for (int n : ns)
    for (int gm : gs)
      for (int bw : bws) g.cand.push_back({n, bw, gm});
  g.ms.assign(g.cand.size(), INFINITY);
  g.idx = 0;
  g.round = 0;
  g.tuned = g.cand.size() <= 1;
}

// Records the device time of each group's setting of this step and moves
// the tuners on; the best setting of a finished group is applied.
int advance_tuning(rtod_batch* b) {
  bool all = true;
  for (auto& g : b->groups) {
    if (g.tuned) continue;
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, g.e0, g.e1));
    g.ms[g.idx] = std::min(g.ms[g.idx], ms);
    if (++g.idx == (int)g.cand.size()) {
      g.idx = 0;
      if (++g.round == b->tune_rounds) {
        const size_t best = (size_t)(std::min_element(g.ms.begin(), g.ms.end()) - g.ms.begin());
        g.tuned = true;
        if (int r = apply_group_setting(b, g, g.cand[best])) return r;
        continue;
      }
    }
    if (int r = apply_group_setting(b, g, g.cand[g.idx])) return r;
    all = false;
  }
  if (all) {
    b->tuning = false;
    for (auto& gx : b->graphs)
      if (gx) {
        cudaGraphExecDestroy(gx);
        gx = nullptr;
      }
  }
  return RTOD_OK;
}

}  // namespace

RTOD_API int rtod_batch_create(const rtod_config* cfgs, int32_t n_streams, rtod_batch** out) {
  if (!cfgs || !out || n_streams < 1 || n_streams > 4096) return fail(RTOD_ERR_ARG, "bad argument");
  *out = nullptr;
  for (int i = 0; i < n_streams; ++i) {
    int r = check_config(&cfgs[i]);
    if (r) return r;
    if (cfgs[i].device != cfgs[0].device) return fail(RTOD_ERR_CONFIG, "all streams must use one device");
    if (cfgs[i].coord != RTOD_COORD_F32) return fail(RTOD_ERR_CONFIG, "the multi-stream API takes float coordinates");
  }
  rtod_batch* b = new (std::nothrow) rtod_batch();
  if (!b) return fail(RTOD_ERR_ARG, "out of host memory");
  b->device = cfgs[0].device;
  b->n = n_streams;
  b->route = cfgs[0].router ? 1 : 0;
  b->fused = cfgs[0].pipeline == RTOD_PIPELINE_FUSED;
  b->filled.assign(n_streams, 0);
  b->pending.assign(n_streams, 0);
  auto bail = [&](int code) {
    std::string msg = g_last_error;
    batch_free(b);
    delete b;
    g_last_error = msg;
    return code;
  };
  for (int i = 0; i < n_streams; ++i) {
    rtod_config c = cfgs[i];
    c.batch = 1;
    c.router = b->route;
    c.use_graph = 0;
    c.engine = RTOD_ENGINE_WINDOW;  // the step runs every stream's window as a window-engine job
    rtod_handle* h = nullptr;
    int r = rtod_create(&c, &h);
    if (r) return bail(r);
    b->hs.push_back(h);
  }
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming))
    return bail(fail(RTOD_ERR_CUDA, "stream creation failed"));
  int64_t dummy = 0;
  if (dalloc(&b->router, 1, &dummy)) return bail(RTOD_ERR_CUDA);
  {
    RouterState* init = new (std::nothrow) RouterState;
    if (!init) return bail(fail(RTOD_ERR_ARG, "out of host memory"));
    init_router(init);
    cudaError_t e = cudaMemcpy(b->router, init, sizeof(RouterState), cudaMemcpyHostToDevice);
    delete init;
    if (e != cudaSuccess) return bail(fail(RTOD_ERR_CUDA, "router init failed"));
    k_table<<<(TQ0 * TQ1 * TQ2 + 255) / 256, 256, 0, b->stream>>>(b->router);
    if (cudaGetLastError() != cudaSuccess) return bail(fail(RTOD_ERR_CUDA, "router table failed"));
  }
  // Streams counted with RTOD_COUNT_AUTO follow their (dimension, predicate)
  // group's points: group counts when auto_group holds for all of them, with
  // the router on as well. The router routes the single points of point
  // counts; a group that counts by groups has none to route, runs unrouted
  // and does not train it (measured on the 64-stream step: 8-d streams in
  // routed point counts made the routed step 3.6x slower than the unrouted).
  {
    std::vector<int64_t> pts(n_streams, 0);
    for (int i = 0; i < n_streams; ++i)
      for (int k = 0; k < n_streams; ++k)
        if (cfgs[k].count == RTOD_COUNT_AUTO && b->hs[k]->D == b->hs[i]->D && cfgs[k].pred == cfgs[i].pred)
          pts[i] += b->hs[k]->W;
    for (int i = 0; i < n_streams; ++i)
      if (cfgs[i].count == RTOD_COUNT_AUTO)
        b->hs[i]->group = auto_group(b->hs[i]->D, pts[i], b->hs[i]->sm_count);
  }
  // Group the streams by (dimension, predicate, count mode), at most
  // BATCH_JOBS_MAX streams per group (one launch's count list).
  for (int i = 0; i < n_streams; ++i) {
    const rtod_handle* h = b->hs[i];
    rtod_batch::Group* g = nullptr;
    for (auto& x : b->groups)
      if (x.geom.D == h->D && x.geom.pred == h->cfg.pred && x.geom.group == h->group &&
          (int)x.streams.size() < BATCH_JOBS_MAX)
        g = &x;
    if (!g) {
      b->groups.emplace_back();
      g = &b->groups.back();
      g->geom = Geom{0, 0, h->D, h->cfg.pred, b->route && !h->group, h->sm_count, h->block_warps, b->router, 0,
                     h->group};
    }
    g->streams.push_back(i);
    g->geom.Wmax = std::max(g->geom.Wmax, h->W);
    g->geom.Smax = std::max(g->geom.Smax, h->S);
  }
  for (auto& g : b->groups) {
    const int ng = (int)g.streams.size();
    std::vector<Job> tab(ng);
    for (int k = 0; k < ng; ++k) {
      rtod_handle* h = b->hs[g.streams[k]];
      tab[k] = make_job(h, 0, true, nullptr);
      g.out_cap += h->W;
      g.cmp_tiles += (h->W + CMP_TILE - 1) / CMP_TILE;
    }
    for (auto& jb : tab) jb.gpts = group_part_size(g.out_cap, b->hs[g.streams[0]]->sm_count);
    if (dalloc(&g.jobs, ng, &dummy) || dalloc(&g.bs, 1, &dummy) || dalloc(&g.out, (size_t)g.out_cap, &dummy) ||
        dalloc(&g.active, ng, &dummy) || dalloc(&g.nout, ng, &dummy) || dalloc(&g.bar, 1, &dummy))
      return bail(RTOD_ERR_CUDA);
    if (cudaMemset(g.bar, 0, sizeof(GridBar))) return bail(fail(RTOD_ERR_CUDA, "group setup failed"));
    if (cudaMallocHost((void**)&g.active_h, sizeof(int32_t) * ng) || cudaMallocHost((void**)&g.nout_h, sizeof(int32_t) * ng) ||
        cudaMallocHost((void**)&g.bs_h, sizeof(BatchState)))
      return bail(fail(RTOD_ERR_CUDA, "pinned allocation failed"));
    if (cudaMemcpy(g.jobs, tab.data(), sizeof(Job) * ng, cudaMemcpyHostToDevice) ||
        cudaMemset(g.bs, 0, sizeof(BatchState)))
      return bail(fail(RTOD_ERR_CUDA, "group setup failed"));
  }
  // Autotuner: when any stream asks for it, every group tries its candidate
  // settings over the first steps (one per step, tune_rounds times), then
  // keeps the fastest.
  for (int i = 0; i < n_streams; ++i) b->tuning = b->tuning || cfgs[i].tuner;
  bool any = false;
  for (auto& g : b->groups) {
    const rtod_handle* h0 = b->hs[g.streams[0]];
    g.cur = {h0->n, h0->block_warps, h0->group};
    if (cudaEventCreate(&g.e0) || cudaEventCreate(&g.e1) ||
        cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming) ||
        cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking))
      return bail(fail(RTOD_ERR_CUDA, "event creation failed"));
    if (!b->tuning) continue;
    init_group_tuning(b, g, cfgs[g.streams[0]]);
    if (!g.tuned) {
      any = true;
      if (int r = apply_group_setting(b, g, g.cand[0], false)) return bail(r);
    }
  }
  b->tuning = any;
  *out = b;
  return RTOD_OK;
}

RTOD_API void rtod_batch_destroy(rtod_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_free(b);
  delete b;
}

RTOD_API int rtod_batch_push(rtod_batch* b, int32_t s, const float* pts, int64_t n) {
  if (!b || !pts || s < 0 || s >= b->n) return fail(RTOD_ERR_ARG, "bad argument");
  rtod_handle* h = b->hs[s];
  CU(cudaSetDevice(b->device));
  if (!b->filled[s]) {
    int r = rtod_push_slide(h, pts, n);  // first push: exactly W points, fills the ring
    if (r) return r;
    b->filled[s] = 1;
    return RTOD_OK;
  }
  if (b->pending[s]) return fail(RTOD_ERR_STATE, "stream %d already has a pending slide", s);
  if (n != h->S) return fail(RTOD_ERR_STATE, "stream %d: a slide push must hold exactly S=%lld points", s,
                             (long long)h->S);
  // Host slides go through the stream's page-locked buffer (copied here, so
  // the caller may reuse its buffer at once); the step that follows waits
  // for the DMA before the next push can touch that buffer.
  const size_t bytes = (size_t)(n * h->D) * sizeof(float);
  const void* src = pts;
  if (!is_device_ptr(pts)) {
    if (!h->stage_host) CU(cudaMallocHost(&h->stage_host, bytes));
    std::memcpy(h->stage_host, pts, bytes);
    src = h->stage_host;
  }
  CU(cudaMemcpyAsync(h->staging, src, bytes, cudaMemcpyDefault, b->stream));
  b->pending[s] = 1;
  return RTOD_OK;
}

RTOD_API int rtod_batch_step(rtod_batch* b, int64_t* out_offsets, int64_t* out_ids, int64_t cap, int64_t* n_total) {
  if (!b || !out_offsets || !n_total || (cap > 0 && !out_ids)) return fail(RTOD_ERR_ARG, "null argument");
  CU(cudaSetDevice(b->device));
  int any = 0;
  for (auto& g : b->groups)
    for (size_t k = 0; k < g.streams.size(); ++k) {
      g.active_h[k] = b->pending[g.streams[k]] ? 1 : 0;
      any |= g.active_h[k];
    }
  if (!any) return fail(RTOD_ERR_STATE, "no stream has a pushed slide");
  const bool train = b->route && (b->steps < kTrainWarm || b->steps % kTrainEvery == 0);
  const bool tuning = b->tuning;
  cudaGraphExec_t& gx = b->graphs[train ? 1 : 0];
  int64_t nk = 0;
  if (tuning) {  // direct launches, each group timed on the device
    if (int r = batch_enqueue(b, train, &nk, true)) return r;
    b->tune_steps++;
  } else if (!gx) {
    cudaGraph_t gr;
    CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int64_t nk0 = 0;
    int r = batch_enqueue(b, train, &nk0, false, true);
    cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
    if (r) return r;
    if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&gx, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return fail(RTOD_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    b->graph_kernels[train ? 1 : 0] = nk0;
  }
  if (!tuning) {
    nk = b->graph_kernels[train ? 1 : 0];
    CU(cudaGraphLaunch(gx, b->stream));
  }
  CU(cudaStreamSynchronize(b->stream));
  b->launches += nk;
  b->steps++;
  // Per-stream counts and errors, then the IDs group by group.
  std::vector<int64_t> cnt(b->n, 0);
  std::vector<int64_t> start(b->n, 0);  // offset of the stream's IDs inside its group output
  for (auto& g : b->groups) {
    rtod_handle* h0 = b->hs[g.streams[0]];
    int r = check_device_error(h0, *g.bs_h);
    if (r) {
      for (int s : g.streams) b->hs[s]->poisoned = true;
      return r;
    }
    int64_t off = 0;
    for (size_t k = 0; k < g.streams.size(); ++k) {
      const int s = g.streams[k];
      cnt[s] = g.active_h[k] ? g.nout_h[k] : 0;
      start[s] = off;
      off += cnt[s];
    }
  }
  out_offsets[0] = 0;
  for (int s = 0; s < b->n; ++s) out_offsets[s + 1] = out_offsets[s] + cnt[s];
  *n_total = out_offsets[b->n];
  if (*n_total > cap) return fail(RTOD_ERR_CAPACITY, "%lld outliers but room for %lld", (long long)*n_total,
                                  (long long)cap);
  for (auto& g : b->groups) {
    for (size_t k = 0; k < g.streams.size(); ++k) {
      const int s = g.streams[k];
      if (cnt[s] > 0)
        CU(cudaMemcpyAsync(out_ids + out_offsets[s], g.out + start[s], sizeof(int64_t) * cnt[s], cudaMemcpyDefault,
                           b->stream));
    }
  }
  CU(cudaStreamSynchronize(b->stream));
  for (int s = 0; s < b->n; ++s)
    if (b->pending[s]) {
      b->pending[s] = 0;
      b->hs[s]->slides_done++;
      b->detections++;
    }
  if (tuning) {
    if (int r = advance_tuning(b)) return r;
    CU(cudaStreamSynchronize(b->stream));
  }
  return RTOD_OK;
}

RTOD_API int rtod_batch_get_tuning(const rtod_batch* b, int32_t* out, int32_t cap) {
  if (!b || (cap > 0 && !out)) return fail(RTOD_ERR_ARG, "null argument");
  const int32_t ng = (int32_t)b->groups.size();
  for (int32_t i = 0; i < ng && i < cap; ++i) {
    const auto& g = b->groups[(size_t)i];
    int32_t* o = out + 6 * i;
    o[0] = g.geom.D;
    o[1] = g.geom.pred;
    o[2] = g.cur.n;
    o[3] = g.cur.bw;
    o[4] = g.cur.group ? RTOD_COUNT_GROUP : RTOD_COUNT_POINT;
    o[5] = g.tuned ? 1 : 0;
  }
  return ng;
}

RTOD_API int rtod_batch_stats(const rtod_batch* b, int64_t out[5]) {
  if (!b || !out) return fail(RTOD_ERR_ARG, "null argument");
  out[0] = b->steps;
  out[1] = b->launches;
  out[2] = b->detections;
  out[3] = (int64_t)b->groups.size();
  int64_t tests = 0;
  for (const auto& g : b->groups) tests += (int64_t)g.bs_h->pair_tests;
  out[4] = tests;
  return RTOD_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free detection of one window (rtod_detect_window_static).
//
// Every buffer of the pipeline lives in one file-scope device array. Host code
// only ever sees the array's device address through cudaGetSymbolAddress
// (the symbol itself is a host-side stand-in). Layout, all 256-byte aligned:
// Job, JobCtr, BatchState, block ranges, keys, last counts, bin counts, bin
// starts, bin key minima and maxima, cell-ordered offsets, keys and
// coordinates, queue, outlier bits, look-back words.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kStaticN = RTOD_STATIC_MAX_POINTS;
constexpr int kStaticD = RTOD_STATIC_MAX_DIM;
constexpr int64_t kStaticWp = ((kStaticN + 3) / 4) * 4 + 4;

constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

struct StaticLayout {
  size_t job, ctr, bs, blo, bhi, keys, prev, bcount, bstart, kmin, kmax, soff, sckey, sx, queue, flags, scan, cmp,
      end;
};

constexpr StaticLayout make_layout() {
  StaticLayout L{};
  size_t o = 0;
  L.job = o; o = al256(o + sizeof(Job));
  L.ctr = o; o = al256(o + sizeof(JobCtr));
  L.bs = o; o = al256(o + sizeof(BatchState));
  L.blo = o; o = al256(o + sizeof(long long) * 6);  // blocks 0 and 1
  L.bhi = o; o = al256(o + sizeof(long long) * 6);
  L.keys = o; o = al256(o + sizeof(uint64_t) * kStaticN);
  L.prev = o; o = al256(o + kStaticN);
  L.bcount = o; o = al256(o + sizeof(uint32_t) * NB);
  L.bstart = o; o = al256(o + sizeof(uint32_t) * (NB + 1));
  L.kmin = o; o = al256(o + sizeof(unsigned long long) * NB);
  L.kmax = o; o = al256(o + sizeof(unsigned long long) * NB);
  L.soff = o; o = al256(o + sizeof(uint32_t) * kStaticN);
  L.sckey = o; o = al256(o + sizeof(uint64_t) * kStaticN);
  L.sx = o; o = al256(o + sizeof(float) * kStaticD * kStaticWp);
  L.queue = o; o = al256(o + sizeof(uint32_t) * kStaticN);
  L.flags = o; o = al256(o + sizeof(uint32_t) * (kStaticN / 32));
  L.scan = o; o = al256(o + sizeof(unsigned long long) * SCAN_TILES);
  L.cmp = o; o = al256(o + sizeof(unsigned long long) * ((kStaticN + CMP_TILE - 1) / CMP_TILE));
  L.end = o;
  return L;
}
constexpr StaticLayout kStatic = make_layout();
static_assert(kStatic.end <= RTOD_STATIC_SCRATCH_BYTES, "static scratch too small for its layout");

static __device__ __align__(256) unsigned char g_static_scratch[RTOD_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
unsigned char* g_static_addr[kMaxDevices] = {};
int g_static_sms[kMaxDevices] = {};

// Device address of the scratch array on the current device and its SM
// count, looked up once per device with that device current (the device's
// compute capability is checked at the same time).
int static_scratch(unsigned char** out, int* sm_count) {
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(RTOD_ERR_NODEV, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_addr[dev]) {
    int major = 0, sms = 0;
    CU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (major != 10) return fail(RTOD_ERR_NODEV, "device %d is not sm_100", dev);
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return fail(RTOD_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
    g_static_sms[dev] = sms;
    g_static_addr[dev] = (unsigned char*)p;
  }
  *out = g_static_addr[dev];
  *sm_count = g_static_sms[dev];
  return RTOD_OK;
}

}  // namespace

RTOD_API int rtod_detect_window_static(const float* pts, int64_t n, int32_t dim, double R, int32_t K, int32_t pred,
                                       int64_t* out_ids, int64_t* n_out, void* stream) {
  if (!pts || !out_ids || !n_out) return fail(RTOD_ERR_ARG, "null argument");
  if (n < 1 || n > kStaticN)
    return fail(RTOD_ERR_CAPACITY, "window of %lld points: the allocation-free entry point takes 1..%lld",
                (long long)n, (long long)kStaticN);
  if (dim < 1 || dim > kStaticD)
    return fail(RTOD_ERR_CAPACITY, "dim %d: the allocation-free entry point takes 1..%d", dim, kStaticD);
  if (!(R >= 1e-18) || !(R <= 1e18) || !std::isfinite(R)) return fail(RTOD_ERR_CONFIG, "R must be finite and in [1e-18, 1e18]");
  if (K < 0) return fail(RTOD_ERR_CONFIG, "K must be >= 0");
  if (pred != RTOD_PRED_FP32_LE && pred != RTOD_PRED_F64_LT) return fail(RTOD_ERR_CONFIG, "unknown predicate %d", pred);
  if (!is_device_ptr(pts) || !is_device_ptr(out_ids))
    return fail(RTOD_ERR_ARG, "pts and out_ids must be device memory");
  unsigned char* base = nullptr;
  int sm = 0;
  int r = static_scratch(&base, &sm);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  auto at = [&](size_t off) { return (void*)(base + off); };

  // Clear what must start at zero (the array keeps the previous call's contents).
  CU(cudaMemsetAsync(at(kStatic.ctr), 0, sizeof(JobCtr), st));
  CU(cudaMemsetAsync(at(kStatic.bs), 0, sizeof(BatchState), st));
  CU(cudaMemsetAsync(at(kStatic.blo), 0x7f, sizeof(long long) * 6, st));
  CU(cudaMemsetAsync(at(kStatic.bhi), 0x80, sizeof(long long) * 6, st));
  CU(cudaMemsetAsync(at(kStatic.bcount), 0, sizeof(uint32_t) * NB, st));
  CU(cudaMemsetAsync(at(kStatic.kmin), 0xff, sizeof(unsigned long long) * NB, st));
  CU(cudaMemsetAsync(at(kStatic.kmax), 0, sizeof(unsigned long long) * NB, st));
  CU(cudaMemsetAsync(at(kStatic.flags), 0, sizeof(uint32_t) * ((n + 31) / 32), st));
  CU(cudaMemsetAsync(at(kStatic.scan), 0, sizeof(unsigned long long) * SCAN_TILES, st));
  CU(cudaMemsetAsync(at(kStatic.cmp), 0, sizeof(unsigned long long) * ((kStaticN + CMP_TILE - 1) / CMP_TILE), st));

  const int n_cells = 2;
  Job jb{};
  jb.W = n;
  jb.S = n;  // one window, one slide block
  jb.Wp = ((n + 3) / 4) * 4 + 4;
  jb.inv_cell = 1.0 / (R * (1.0 + std::ldexp(1.0, -12)) / (double)n_cells);
  jb.R = R;
  jb.R2 = R * R;
  {
    volatile float rf = (float)R;
    volatile float r2f = rf * rf;
    jb.R2f = r2f;
  }
  jb.K = K;
  jb.n = n_cells;
  jb.filter = 1;
  jb.ring = 0;
  jb.gpts = 32;
  jb.pts = pts;
  jb.keys = (const uint64_t*)at(kStatic.keys);
  jb.stage = nullptr;
  jb.blk_lo = (const long long*)at(kStatic.blo);
  jb.blk_hi = (const long long*)at(kStatic.bhi);
  jb.prev = (uint8_t*)at(kStatic.prev);
  jb.bin_count = (uint32_t*)at(kStatic.bcount);
  jb.bin_start = (uint32_t*)at(kStatic.bstart);
  jb.kmin = (unsigned long long*)at(kStatic.kmin);
  jb.kmax = (unsigned long long*)at(kStatic.kmax);
  jb.s_off = (uint32_t*)at(kStatic.soff);
  jb.s_ckey = (uint64_t*)at(kStatic.sckey);
  jb.s_x = (float*)at(kStatic.sx);
  jb.queue = (uint32_t*)at(kStatic.queue);
  jb.feat = nullptr;
  jb.flags = (uint32_t*)at(kStatic.flags);
  jb.scan_status = (unsigned long long*)at(kStatic.scan);
  jb.cmp_status = (unsigned long long*)at(kStatic.cmp);
  jb.ctr = (JobCtr*)at(kStatic.ctr);
  jb.rec_nout = nullptr;
  jb.rec_undet = nullptr;
  jb.rec_base = nullptr;
  jb.rec_cap = 0;
  // Pageable source: the copy has been staged when the call returns.
  CU(cudaMemcpyAsync(at(kStatic.job), &jb, sizeof(Job), cudaMemcpyHostToDevice, st));

  Batch b{};
  b.jobs = (const Job*)at(kStatic.job);
  b.njobs = 1;
  b.bs = (BatchState*)at(kStatic.bs);
  b.router = nullptr;
  b.active = nullptr;
  b.job_nout = nullptr;
  b.out_ids = out_ids;
  b.out_cap = n;
  b.cmp_tiles = (n + CMP_TILE - 1) / CMP_TILE;

  const unsigned kx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm * 8));
  DISPATCH_D(dim, CU(launch_k(k_keys<D, float>, dim3(kx), 256, st, pts, (int64_t)0, n, jb.inv_cell, (uint64_t*)at(kStatic.keys),
                               (uint8_t*)at(kStatic.prev), b.bs, n, (long long*)at(kStatic.blo),
                               (long long*)at(kStatic.bhi))));
  const Geom g{n, n, dim, pred, 0, sm, 8, nullptr};
  if ((r = launch_group(g, b, false, false, st, nullptr, nullptr))) return r;
  BatchState s{};
  CU(cudaMemcpyAsync(&s, at(kStatic.bs), sizeof(BatchState), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  switch (s.err) {
    case DERR_NONE: break;
    case DERR_NONFINITE: return fail(RTOD_ERR_INPUT, "non-finite coordinate in the window");
    case DERR_RANGE: return fail(RTOD_ERR_INPUT, "coordinate too large for the grid");
    case DERR_CAPACITY: return fail(RTOD_ERR_CAPACITY, "outlier ID buffer too small");
    case DERR_TIMEOUT: return fail(RTOD_ERR_TIMEOUT, "a bounded device-side wait ran out");
    default: return fail(RTOD_ERR_CUDA, "device error %d", s.err);
  }
  *n_out = s.out_total;
  return RTOD_OK;
}
