// Device code of the detector pipeline (sm_100a), batched over jobs: the
// window engine (one counting sort per window; push/detect, the
// multi-stream API, and rtod_run when chosen). span.cuh holds the span
// engine of rtod_run (one counting sort per batch of consecutive windows),
// which shares this file's cell keys, predicates, scans and finish_batch.
//
// A job is the detection of one window of one stream. Every kernel takes a
// Batch (a table of jobs) and uses blockIdx.y as the job index, so one launch
// serves B windows: consecutive windows of one resident stream (rtod_run),
// the current window of many streams (batched streaming), or the single
// window of a push/detect step. A batch runs five kernels in stream order:
//
//   k_hist     cell occupancy of each window: per-bin point counts and the
//              per-bin key range (a bin holds one cell iff min == max). Replaces the expire /
//              insert bookkeeping of prepare_c_non_points_queue
//              (src/ods/optixScan.cpp:967-981) and FixQueue (state.h:15-57).
//   k_scan     exclusive scan of the bin counts -> bin starts (16 tiles per
//              window chained by a warp-parallel decoupled look-back).
//   k_scatter  counting sort of the window into cell order (window offset,
//              cell key and coordinates as SoA) and classification: points
//              of a bin that holds one cell with more than K points are
//              inliers (safe-inlier skip, the all-inlier cell filter of
//              :983-993); every other point goes to the query queue.
//              k_scan + k_scatter replace kGenAABB (aabb.cu:5-45), the BVH
//              rebuild (:378-426) and the undetermined-point gather
//              (:995-1016).
//   k_count    range count of the queued points, one warp per point, K early
//              exit. Replaces the ray launch and intersection program
//              (optixScan.cu:21-75, :158-199). With the learned router on
//              (router.cuh), k_scatter splits the queue into an early-exit and
//              a full-sweep queue and k_count treats them differently; the
//              router network is trained after the batch by k_train.
//   k_compact  outlier bitset -> sorted global indices appended to the batch
//              output in job order; per-slide records; window advance.
//              Replaces the D2H + host pick of :1083-1101 and :1103-1108.
//
// Points come either from a ring (push/detect streaming: SoA [D][W], ring
// slot = global index % W, filled by k_ingest, which replaces the slide H2D
// and host mirror of :1051-1064) or straight from a stream resident in HBM
// (point-major, keys precomputed by k_keys).
//
// Scratch arrays clean up after themselves for the next batch: k_scatter
// hands bin counts back to zero (it claims positions with atomicSub),
// k_count resets the per-bin key ranges and the compaction look-back words,
// k_compact clears the outlier bits it read, and its last block ends the
// batch (finish_batch: per-slide records, window advance, per-job counters). Consecutive kernels use programmatic dependent launch:
// each kernel lets the next one launch early and waits (griddepcontrol.wait)
// for its predecessor to complete before touching shared data.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

namespace rtod {

constexpr int NB_LOG2 = 16;
constexpr uint32_t NB = 1u << NB_LOG2;  // bins of the cell hash table, per job
constexpr uint32_t NB_MASK = NB - 1;
constexpr unsigned long long EMPTY_KEY = ~0ull;
constexpr int SCAN_TILE = 4096;             // bins per k_scan tile (16 per thread)
constexpr int SCAN_TILES = NB / SCAN_TILE;  // 16
constexpr int SPAN_SCAN_TILE = 1024;        // bins per k_span_scan tile (4 per thread)
constexpr int SPAN_SCAN_TILES = NB / SPAN_SCAN_TILE;  // 64
constexpr int CMP_TILE = 8192;              // window offsets per k_compact tile (32 per thread)
constexpr int SPIN_LIMIT = 1 << 22;         // bounded waits (then DERR_TIMEOUT)

// Device error codes (first one wins).
enum : int32_t {
  DERR_NONE = 0, DERR_NONFINITE = 1, DERR_RANGE = 2, DERR_CAPACITY = 3, DERR_TIMEOUT = 4,
  DERR_GRID = 5  // the streaming grid (grid.cuh) must be rebuilt from the ring: not the caller's error
};

// Per-job counters (device). lo is the first global index of the job's
// window; after each detection it advances by lo_step.
struct JobCtr {
  int64_t lo;
  int64_t lo_step;
  int32_t n_undet;       // queued points: early-exit queue (router on) or the only queue
  int32_t n_out;         // outliers found
  uint32_t scan_ticket;  // k_scan tile tickets
  uint32_t cmp_ticket;   // k_compact tile tickets
  int32_t n_sweep;       // queued points of the full-sweep queue (router on)
  int32_t last_nout;     // outliers of the job's last detected window
  int32_t pure;          // current window: no two of its cells share a bin
  int32_t n_groups;      // parts of bins listed for a group count (group mode)
};

// Per-handle state (device).
struct BatchState {
  int64_t out_total;    // outliers found so far (IDs in out_ids, or pending in bitsets)
  int64_t slides;       // windows detected so far
  int64_t undet_total;  // queued points summed over windows
  int32_t err;          // DERR_*
  uint32_t done;        // finished blocks of the running batch's last kernel
  unsigned long long pair_tests;  // distance tests made by group counts so far
  uint32_t count_ticket;  // next entry of the batch-wide count list (k_count), reset by the batch end
};

// Span engine counters (device), one per handle, and the per-bin arrays
// that k_compact clears after each batch.
struct SpanCtr {
  uint32_t scan_ticket;  // tile tickets of the span's bin scan
  uint32_t n_used;       // bins holding span points
  int32_t pure;          // the span's cells and their sure neighbours map to distinct bins (k_span_scan)
  uint32_t n_groups;     // groups listed for exact counts in the running batch
  uint32_t n_segs;       // delta segments listed (learned router on), from the back of the list
  uint32_t seg_ticket;   // next delta segment for a count warp to take
  uint32_t group_ticket; // next independent group for a count warp to take (router on)
  long long cmin[3];     // per hashed dimension, the span's cell coordinate range (k_span_hist)
  long long cmax[3];
  uint32_t* used;        // [NB] bins in use
  uint32_t* bin_count;   // [NB]
  unsigned long long* kmin;  // [NB]
  unsigned long long* kmax;  // [NB]
};


struct Job {
  int64_t W, S, Wp;  // window, slide, padded SoA row stride (multiple of 4, >= W + 4)
  double inv_cell;   // 1 / cell, cell side = R * (1 + 2^-12) / n
  double R, R2;
  float R2f;         // fl32(fl32(R)^2)
  int32_t K;
  int32_t n;         // cells per R = stencil reach in cells
  int32_t filter;    // safe-inlier skip enabled
  int32_t ring;      // 1: ring source, 0: resident stream
  int32_t gpts;      // group mode: points per listed part of a bin (power of two, >= 32)
  const void* pts;        // coordinates (float or double, the handle's type): ring: SoA
                          // [D][W] by slot; stream: point-major [N][D]
  const uint64_t* keys;   // ring: [W] by slot; stream: [N] by global index
  const void* stage;      // ring: the points k_ingest writes (point-major)
  const long long* blk_lo;  // stream: per slide block (S points), min cell coordinate per
  const long long* blk_hi;  //   hashed dimension ([blocks][3]); null for a ring
  uint8_t* prev;          // last capped count per source position (255 = safe, 254 = none)
  uint32_t* bin_count;    // [NB]
  uint32_t* bin_start;    // [NB + 1]
  unsigned long long* kmin;   // [NB] smallest cell key in a bin (EMPTY_KEY when none)
  unsigned long long* kmax;   // [NB] largest cell key in a bin (0 when none)
  uint32_t* s_off;        // [W] cell-ordered: window offset (global index - lo)
  uint64_t* s_ckey;       // [W] cell-ordered: cell key
  void* s_x;              // [D][Wp] cell-ordered coordinates (the handle's type)
  uint32_t* queue;        // [W] cell-ordered positions that need an exact count; with the
                          // router on, the early-exit queue grows from the front and the
                          // full-sweep queue from the back
  float* feat;            // [W][3] router features, at the same index as the queue entry
  uint32_t* flags;        // [ceil(W / 32)] outlier bit per window offset
  unsigned long long* scan_status;  // [SCAN_TILES]
  unsigned long long* cmp_status;   // [ceil(W / CMP_TILE)]
  JobCtr* ctr;
  int32_t* rec_nout;      // per-slide outlier counts, indexed (lo - S) / S; may be null
  int32_t* rec_undet;
  int64_t* rec_base;      // per-slide output offset of its outlier IDs (span batches)
  int64_t rec_cap;
};

struct RouterState;

// Kernel argument: the jobs of one launch and the shared output.
struct Batch {
  const Job* jobs;
  int32_t njobs;
  BatchState* bs;
  RouterState* router;  // learned router (used when the kernels are built with ROUTE)
  const int32_t* active; // per job: 0 = skip this job in this launch (null: all active)
  int32_t* job_nout;     // per job: outliers of this launch's window (may be null)
  int64_t* out_ids;  // outlier IDs of all jobs, concatenated in job order
  int64_t out_cap;
  int64_t cmp_tiles; // k_compact tiles over all jobs
  SpanCtr* span;     // span engine counters, cleared by the last k_compact tile (null otherwise)
};

__device__ __forceinline__ void set_err(BatchState* bs, int32_t code) { atomicCAS(&bs->err, 0, code); }

__device__ __forceinline__ bool job_active(const Batch& b, uint32_t job) { return !b.active || b.active[job]; }

// Block coordinates of a pipeline stage: x index and extent of the block
// within its job, and the job. A kernel of one stage passes its own
// blockIdx / gridDim; the fused pipeline kernel (fused.cuh) runs each stage
// over a virtual grid of such blocks.
struct VB {
  uint32_t x, y, gx;
};
__device__ __forceinline__ VB hw_block() { return VB{blockIdx.x, blockIdx.y, gridDim.x}; }

// ---------------------------------------------------------------------------
// Grid cells. Cell coordinate k_i = floor(x_i * inv_cell) in double
// precision (inv_cell = fl(1 / cell)), for the first h = min(D, 3)
// dimensions. With cell = R(1+2^-12)/n and |x/cell| below the limits below,
// any pair accepted by either predicate has |k_i(p) - k_i(q)| <= n (the
// stencil), and for D <= 3, n >= 2 two points of one cell are always
// neighbours (so a cell with more than K points is all-inlier). The product
// x * inv_cell is within a relative 1.5 * 2^-52 of x / cell, so the limits
// keep its error below 2^-16 cells.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double coord_limit(int h) {
  return h == 1 ? 34359738368.0 /* 2^35 */ : (h == 2 ? 1073741824.0 /* 2^30 */ : 1048576.0 /* 2^20 */);
}

__device__ __forceinline__ uint64_t pack_key(const int64_t* k, int h) {
  if (h == 1) return (uint64_t)(k[0] + (1ll << 36));
  if (h == 2) return ((uint64_t)(k[0] + (1ll << 30)) << 32) | (uint64_t)(k[1] + (1ll << 30));
  return ((uint64_t)(k[0] + (1ll << 20)) << 42) | ((uint64_t)(k[1] + (1ll << 20)) << 21) |
         (uint64_t)(k[2] + (1ll << 20));
}

__device__ __forceinline__ void unpack_key(uint64_t key, int h, int64_t* k) {
  if (h == 1) {
    k[0] = (int64_t)key - (1ll << 36);
  } else if (h == 2) {
    k[0] = (int64_t)(key >> 32) - (1ll << 30);
    k[1] = (int64_t)(key & 0xffffffffull) - (1ll << 30);
  } else {
    k[0] = (int64_t)(key >> 42) - (1ll << 20);
    k[1] = (int64_t)((key >> 21) & 0x1fffffull) - (1ll << 20);
    k[2] = (int64_t)(key & 0x1fffffull) - (1ll << 20);
  }
}

// Bin of a cell. Consecutive cells along the last hashed dimension land in
// consecutive bins (mod NB), so a stencil row of 2n+1 cells is one run of
// bins; rows of one stencil never share a bin for n <= 3 (1-d: any n).
__device__ __forceinline__ uint32_t bin_of(const int64_t* k, int h) {
  if (h == 1) return (uint32_t)k[0] & NB_MASK;
  if (h == 2) return ((uint32_t)k[1] + ((uint32_t)k[0] << 8)) & NB_MASK;
  return ((uint32_t)k[2] + ((uint32_t)k[1] << 6) + ((uint32_t)k[0] << 12)) & NB_MASK;
}

__device__ __forceinline__ uint32_t bin_of_key(uint64_t key, int h) {
  int64_t k[3];
  unpack_key(key, h, k);
  return bin_of(k, h);
}

template <int D>
struct Hashed {
  static constexpr int value = D < 3 ? D : 3;
};

// Cell key of one point (float or double coordinates); *code =
// DERR_NONFINITE for a non-finite coordinate, DERR_RANGE for one too large
// for the grid (then the key is zero).
template <int D, typename T>
__device__ __forceinline__ uint64_t cell_key(const T* x, double inv_cell, int32_t* code) {
  constexpr int H = Hashed<D>::value;
  const double lim = coord_limit(H);
  bool ok = true;
#pragma unroll
  for (int d = 0; d < D; ++d) ok &= isfinite(x[d]);
  int64_t k[3] = {0, 0, 0};
  bool inr = true;
#pragma unroll
  for (int d = 0; d < H; ++d) {
    const double q = floor(__dmul_rn((double)x[d], inv_cell));
    inr &= (q > -lim) && (q < lim);
    k[d] = inr ? (int64_t)q : 0;
  }
  *code = !ok ? DERR_NONFINITE : (!inr ? DERR_RANGE : DERR_NONE);
  if (*code) k[0] = k[1] = k[2] = 0;
  return pack_key(k, H);
}

// ---------------------------------------------------------------------------
// Neighbour predicates. PRED 0: FP32, each subtract, multiply and add
// rounded on its own (no FMA contraction), summed left to right,
// d2 <= fl32(fl32(R)^2). PRED 1: RTOD's double test
// (src/ods/optixScan.cu:170-190): |dx| < R in 1-d, d^2 < R*R otherwise, on
// float coordinates widened to double or on double coordinates (T = double,
// used only with PRED 1).
// ---------------------------------------------------------------------------
template <int D, int PRED, typename T>
__device__ __forceinline__ bool is_nbr(const T* q, const T* c, float R2f, double R, double R2) {
  if constexpr (PRED == 0) {
    static_assert(sizeof(T) == sizeof(float), "the FP32 predicate runs on float coordinates");
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const float dx = __fsub_rn(q[i], c[i]);
      const float t = __fmul_rn(dx, dx);
      s = (i == 0) ? t : __fadd_rn(s, t);
    }
    return s <= R2f;
  } else {
    if constexpr (D == 1) {
      return fabs(__dsub_rn((double)q[0], (double)c[0])) < R;
    } else {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const double dx = __dsub_rn((double)q[i], (double)c[i]);
        const double t = __dmul_rn(dx, dx);
        s = (i == 0) ? t : __dadd_rn(s, t);
      }
      return s < R2;
    }
  }
}

// The FP32 predicate (PRED 0) for two candidates at once, with sm_100's
// paired single-precision instructions: each half of sub/mul/add.rn.f32x2 is
// the IEEE single-precision operation rounded to nearest on its own (no
// contraction: the instructions are explicit), so each half's sum is
// bit-identical to is_nbr<D, 0> on that candidate. q2[i] holds the query's
// coordinate i twice; c2[i] holds coordinate i of the two candidates.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}

template <int D>
__device__ __forceinline__ void is_nbr_f32x2(const unsigned long long* q2, const unsigned long long* c2, float R2f,
                                             bool& n0, bool& n1) {
  unsigned long long s = 0;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    unsigned long long dx, t;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(dx) : "l"(q2[i]), "l"(c2[i]));
    asm("mul.rn.f32x2 %0, %1, %1;" : "=l"(t) : "l"(dx));
    if (i == 0) s = t;
    else asm("add.rn.f32x2 %0, %1, %2;" : "=l"(s) : "l"(s), "l"(t));
  }
  float s0, s1;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(s0), "=f"(s1) : "l"(s));
  n0 = s0 <= R2f;
  n1 = s1 <= R2f;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch, release/acquire and single-pass scans.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

__device__ __forceinline__ void st_release(unsigned long long* a, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* a) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
  return v;
}

constexpr unsigned long long LB_AGG = 1ull << 62;     // tile total published
constexpr unsigned long long LB_PREFIX = 2ull << 62;  // inclusive prefix published

// Exclusive prefix of `tile` over all earlier tiles of one scan, computed by
// one full warp: publishes the tile total, then inspects the 32 nearest
// predecessors at once and sums back to the nearest published prefix, then
// publishes its own inclusive prefix. Tiles are claimed in ticket order, so
// every predecessor is running or done and the chain always resolves; each
// wait is still bounded (DERR_TIMEOUT, partial sum used).
static __device__ uint32_t warp_lookback(unsigned long long* status, uint32_t tile, uint32_t total,
                                  BatchState* bs) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_release(&status[0], LB_PREFIX | total);
    return 0;
  }
  if (lane == 0) st_release(&status[tile], LB_AGG | total);
  uint32_t acc = 0;
  int64_t base = (int64_t)tile - 1;
  while (true) {
    const int64_t idx = base - lane;
    unsigned long long v = LB_PREFIX;  // before tile 0: an empty prefix
    if (idx >= 0) {
      int it = 0;
      while (((v = ld_acquire(&status[idx])) >> 62) == 0) {
        if (++it > SPIN_LIMIT) {
          set_err(bs, DERR_TIMEOUT);
          v = LB_PREFIX;
          break;
        }
        __nanosleep(32);
      }
    }
    const unsigned pref = __ballot_sync(0xffffffffu, (v >> 62) == 2);
    const int stop = pref ? __ffs(pref) - 1 : 31;
    uint32_t val = lane <= stop ? (uint32_t)(v & 0xffffffffull) : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
    acc += val;
    if (pref) break;
    base -= 32;
  }
  if (lane == 0) st_release(&status[tile], LB_PREFIX | (acc + total));
  return acc;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total, uint32_t* smem33) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) smem33[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const uint32_t w = lane < nw ? smem33[lane] : 0;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    smem33[lane] = wi - w;
    if (lane == 31) smem33[32] = wi;
  }
  __syncthreads();
  const uint32_t r = smem33[wid] + inc - v;
  *total = smem33[32];
  __syncthreads();
  return r;
}

// Window offset i of a job -> source position (ring slot or global index).
__device__ __forceinline__ int64_t source_pos(const Job& jb, int64_t lo, int64_t i) {
  const int64_t g = lo + i;
  return jb.ring ? g % jb.W : g;
}

template <int D, typename T>
__device__ __forceinline__ void load_point(const Job& jb, int64_t src, T* x) {
  const T* pts = static_cast<const T*>(jb.pts);
  if (jb.ring) {
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = pts[(int64_t)d * jb.W + src];
  } else {
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = pts[src * D + d];
  }
}

// Coordinate row d of a job's cell-ordered SoA.
template <typename T>
__device__ __forceinline__ T* sx_row(const Job& jb, int d) {
  return static_cast<T*>(jb.s_x) + (int64_t)d * jb.Wp;
}

// Four consecutive coordinates starting at a multiple of 4 (rows are
// aligned to 16 bytes for float, 32 for double).
__device__ __forceinline__ void load4(const float* p, float* v) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, double* v) {
  const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

}  // namespace rtod

#include "router.cuh"
#include "group.cuh"

namespace rtod {

// ---------------------------------------------------------------------------
// k_keys: cell keys of a resident stream, global indices [g0, g1).
// ---------------------------------------------------------------------------
template <int D, typename T>
__global__ void __launch_bounds__(256) k_keys(const T* pts, int64_t g0, int64_t g1, double inv_cell,
                                              uint64_t* keys, uint8_t* prev, BatchState* bs, int64_t S,
                                              long long* blk_lo, long long* blk_hi) {
  pdl_trigger();
  pdl_wait();
  constexpr int H = Hashed<D>::value;
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = g0 + (int64_t)blockIdx.x * blockDim.x; base < g1; base += stride) {
    const int64_t g = base + threadIdx.x;
    const bool valid = g < g1;
    int64_t k[3] = {0, 0, 0};
    int64_t blk = -1;
    if (valid) {
      T x[D];
#pragma unroll
      for (int d = 0; d < D; ++d) x[d] = pts[g * D + d];
      int32_t code;
      const uint64_t key = cell_key<D, T>(x, inv_cell, &code);
      keys[g] = key;
      prev[g] = 254;
      if (code) set_err(bs, code);
      unpack_key(key, H, k);
      blk = g / S;
    }
    // Per slide block, the range of cell coordinates: reduced over the lanes
    // of each block present in the warp, then one atomic per block and dim.
    unsigned todo = __ballot_sync(0xffffffffu, valid);
    while (todo) {
      const int ld = __ffs(todo) - 1;
      const int64_t bid = __shfl_sync(0xffffffffu, blk, ld);
      const unsigned grp = __ballot_sync(0xffffffffu, valid && blk == bid);
      todo &= ~grp;
      const bool in = (grp >> lane) & 1;
#pragma unroll
      for (int d = 0; d < H; ++d) {
        long long mn = in ? k[d] : LLONG_MAX, mx = in ? k[d] : LLONG_MIN;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
          mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if (lane == ld) {
          atomicMin(&blk_lo[bid * 3 + d], mn);
          atomicMax(&blk_hi[bid * 3 + d], mx);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k_ingest: ring update of every job. fill = 1 writes the first W points
// (global indices [0, W)); otherwise the S newest points of the job's window
// [lo, lo + W), i.e. [lo + W - S, lo + W). Slot = global index % W.
// ---------------------------------------------------------------------------
template <int D, typename T>
__device__ __forceinline__ void ingest_body(const Batch& b, int32_t fill, VB v) {
  if (!job_active(b, v.y)) return;
  const Job& jb = b.jobs[v.y];
  T* ring = static_cast<T*>(const_cast<void*>(jb.pts));
  const T* stage = static_cast<const T*>(jb.stage);
  uint64_t* keys = const_cast<uint64_t*>(jb.keys);
  const int64_t n_new = fill ? jb.W : jb.S;
  const int64_t base = fill ? 0 : jb.ctr->lo + jb.W - jb.S;
  const int64_t stride = (int64_t)v.gx * blockDim.x;
  for (int64_t i = (int64_t)v.x * blockDim.x + threadIdx.x; i < n_new; i += stride) {
    const int64_t slot = (base + i) % jb.W;
    T x[D];
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = stage[i * D + d];
    int32_t code;
    const uint64_t key = cell_key<D, T>(x, jb.inv_cell, &code);
    if (code) set_err(b.bs, code);
#pragma unroll
    for (int d = 0; d < D; ++d) ring[(int64_t)d * jb.W + slot] = x[d];
    keys[slot] = key;
    jb.prev[slot] = 254;
  }
}

template <int D, typename T>
__global__ void __launch_bounds__(256) k_ingest(Batch b, int32_t fill) {
  pdl_trigger();
  pdl_wait();
  ingest_body<D, T>(b, fill, hw_block());
}

// k_rekey: the cell key of every ring slot of every job, recomputed from the
// ring's coordinates with the job's current cell (after the multi-stream
// autotuner changed a group's cell width). Grid (x, jobs).
template <int D, typename T>
__global__ void __launch_bounds__(256) k_rekey(Batch b) {
  pdl_trigger();
  pdl_wait();
  if (!job_active(b, blockIdx.y)) return;
  const Job& jb = b.jobs[blockIdx.y];
  const T* ring = static_cast<const T*>(jb.pts);
  uint64_t* keys = const_cast<uint64_t*>(jb.keys);
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < jb.W; s += (int64_t)gridDim.x * blockDim.x) {
    T x[D];
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = ring[(int64_t)d * jb.W + s];
    int32_t code;
    keys[s] = cell_key<D, T>(x, jb.inv_cell, &code);
    if (code) set_err(b.bs, code);
  }
}

// ---------------------------------------------------------------------------
// k_hist: per-bin counts and the smallest / largest cell key per bin (a bin
// holds a single cell iff they are equal), warp-aggregated, with atomics
// whose results are not needed (no round trip on the critical path).
// ---------------------------------------------------------------------------
// Points handled per lane per loop iteration by k_hist and k_scatter: their
// loads and atomics are all issued before any result is used.
template <int D>
struct Unroll {
  static constexpr int value = D <= 3 ? 2 : 1;  // measured: half of 4 / 2 is 7-9% faster
};

// Whether no two cells of slide blocks [b0, b0 + nb) of a resident stream
// can share a bin, nor a cell share one with a neighbour within margin/2 of
// another, from the per-block coordinate ranges (a ring has none). The bin
// map is injective on boxes of at most 65536 cells (1-d), 256 x 256 (2-d)
// or 16 x 64 x 64 (3-d). One warp computes it.
// Whether cells within [mn_d - margin/2, mx_d + margin/2] per dimension map
// to distinct bins: then no two cells of the range share a bin, and a
// neighbour k + d (|d_i| <= margin/2) of a cell k of the range lies in a bin
// that holds cell k + d or nothing.
template <int H>
__device__ __forceinline__ bool box_pure(const long long* mn, const long long* mx, int margin) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < H; ++d) {
    const long long span = mx[d] - mn[d] + 1 + margin;
    const long long cap = H == 1 ? 65536 : (H == 2 ? 256 : (d == 0 ? 16 : 64));
    ok &= span <= cap;
  }
  return ok;
}

template <int H>
__device__ __forceinline__ bool range_pure(const long long* blk_lo, const long long* blk_hi, int64_t b0,
                                           int64_t nb, int margin) {
  if (!blk_lo || nb > 4096) return false;
  const int lane = threadIdx.x & 31;
  long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  for (int64_t t = lane; t < nb; t += 32) {
#pragma unroll
    for (int d = 0; d < H; ++d) {
      mn[d] = min(mn[d], blk_lo[(b0 + t) * 3 + d]);
      mx[d] = max(mx[d], blk_hi[(b0 + t) * 3 + d]);
    }
  }
#pragma unroll
  for (int d = 0; d < H; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  }
  return box_pure<H>(mn, mx, margin);
}

// The same test for the job's current window, with room for the 1-d group
// rule's neighbours (cells within n-2).
template <int H>
__device__ __forceinline__ bool window_pure(const Job& jb, int64_t lo) {
  return range_pure<H>(jb.blk_lo, jb.blk_hi, lo / jb.S, jb.W / jb.S, 2 * max(jb.n - 2, 0));
}



constexpr int HIST_BITS = 8;                  // slot index bits of the table below
constexpr int HIST_SLOTS = 1 << HIST_BITS;  // block-local aggregation table of k_hist and k_scatter

// k_hist: per-bin counts (and, unless the window is pure, the per-bin key
// range), aggregated first per warp, then per block in a shared-memory hash
// table, then flushed to global memory with one atomic per bin per block.
// With INGEST (a ring job of the fused pipeline), the S newest points of the
// window are taken from the staged slide instead: their keys are computed
// here and they are written into the ring (k_ingest's work, folded in).
template <int D, typename T = float, bool INGEST = false>
__device__ __forceinline__ void hist_body(const Batch& b, VB v) {
  __shared__ uint32_t hbin[HIST_SLOTS];
  __shared__ uint32_t hcnt[HIST_SLOTS];
  __shared__ unsigned long long hmin[HIST_SLOTS], hmax[HIST_SLOTS];
  __shared__ int s_pure;
  if (!job_active(b, v.y)) return;
  constexpr int H = Hashed<D>::value;
  constexpr int U = Unroll<D>::value;
  const Job& jb = b.jobs[v.y];
  const int64_t lo = jb.ctr->lo;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
    const bool pure = window_pure<H>(jb, lo);
    if (threadIdx.x == 0) {
      s_pure = pure;
      if (v.x == 0) jb.ctr->pure = pure;
    }
  }
  for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
    hbin[t] = 0xffffffffu;
    hcnt[t] = 0;
    hmin[t] = EMPTY_KEY;
    hmax[t] = 0;
  }
  __syncthreads();
  const bool pure = s_pure;
  const int64_t chunk = (int64_t)blockDim.x * U;
  const int64_t first_new = jb.W - jb.S;  // window offset of the staged slide (INGEST)
  for (int64_t c0 = (int64_t)v.x * chunk; c0 < jb.W; c0 += (int64_t)v.gx * chunk) {
    const int64_t w0 = c0 + (int64_t)(threadIdx.x >> 5) * 32 * U;
    uint64_t key[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = w0 + u * 32 + lane;
      if (INGEST && i >= first_new && i < jb.W) {
        const int64_t slot = source_pos(jb, lo, i);
        const T* stage = static_cast<const T*>(jb.stage) + (i - first_new) * D;
        T* ring = static_cast<T*>(const_cast<void*>(jb.pts));
        T x[D];
#pragma unroll
        for (int d = 0; d < D; ++d) x[d] = stage[d];
        int32_t code;
        key[u] = cell_key<D, T>(x, jb.inv_cell, &code);
        if (code) set_err(b.bs, code);
#pragma unroll
        for (int d = 0; d < D; ++d) ring[(int64_t)d * jb.W + slot] = x[d];
        const_cast<uint64_t*>(jb.keys)[slot] = key[u];
        jb.prev[slot] = 254;
      } else {
        key[u] = i < jb.W ? jb.keys[source_pos(jb, lo, i)] : EMPTY_KEY;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool valid = key[u] != EMPTY_KEY;
      const uint32_t bin = valid ? bin_of_key(key[u], H) : 0xffffffffu;
      const unsigned peers = __match_any_sync(0xffffffffu, bin);
      const int leader = __ffs(peers) - 1;
      const uint64_t lkey = __shfl_sync(0xffffffffu, key[u], leader);
      const bool mixed_grp = (__ballot_sync(0xffffffffu, key[u] != lkey) & peers) != 0;
      int slot = -1;
      if (valid && lane == leader) {
        const uint32_t c = (uint32_t)__popc(peers);
        uint32_t sl = (bin * 2654435761u) >> (32 - HIST_BITS);
#pragma unroll 1
        for (int probe = 0; probe < 8; ++probe) {
          const uint32_t old = atomicCAS(&hbin[sl], 0xffffffffu, bin);
          if (old == 0xffffffffu || old == bin) {
            atomicAdd(&hcnt[sl], c);
            slot = (int)sl;
            break;
          }
          sl = (sl + 1) & (HIST_SLOTS - 1);
        }
        if (slot < 0) atomicAdd(&jb.bin_count[bin], c);
      }
      if (!pure) {
        // key range of the bin: the leader alone when the group's keys agree
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (valid && (mixed_grp || lane == leader)) {
          if (slot >= 0) {
            atomicMin(&hmin[slot], (unsigned long long)key[u]);
            atomicMax(&hmax[slot], (unsigned long long)key[u]);
          } else {
            atomicMin(&jb.kmin[bin], (unsigned long long)key[u]);
            atomicMax(&jb.kmax[bin], (unsigned long long)key[u]);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
    const uint32_t bin = hbin[t];
    if (bin != 0xffffffffu) {
      atomicAdd(&jb.bin_count[bin], hcnt[t]);
      if (!pure) {
        atomicMin(&jb.kmin[bin], hmin[t]);
        atomicMax(&jb.kmax[bin], hmax[t]);
      }
    }
  }
}

template <int D>
__global__ void __launch_bounds__(256) k_hist(Batch b) {
  pdl_trigger();
  pdl_wait();
  hist_body<D>(b, hw_block());
}

// k_hist of ring jobs with the slide's ingest folded in (the S newest points
// keyed from the staged slide and written into the ring); with reset_out it
// also starts the batch output at zero (read by the compaction).
template <int D, typename T>
__global__ void __launch_bounds__(256) k_hist_ingest(Batch b, int32_t reset_out) {
  pdl_trigger();
  pdl_wait();
  if (reset_out && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) b.bs->out_total = 0;
  hist_body<D, T, true>(b, hw_block());
}

// ---------------------------------------------------------------------------
// k_scan: exclusive scan of each job's NB bin counts. Grid (NB / TILE, jobs),
// 256 threads; each thread owns TILE / 256 consecutive bins (coalesced
// uint4 loads). The window engine uses 4096-bin tiles, the span engine
// 1024-bin tiles (measured: 64 smaller tiles are 1-2% faster for a span's one
// scan per batch, 4% slower for the window engine's scan per window).
// ---------------------------------------------------------------------------
template <int TILE>
__device__ __forceinline__ void scan_bins(const uint32_t* bin_count, uint32_t* bin_start,
                                          unsigned long long* status, uint32_t* ticket, BatchState* bs) {
  constexpr int Q = TILE / 1024;  // uint4 per thread
  __shared__ uint32_t sm[33];
  __shared__ uint32_t s_tile, s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t b0 = tile * TILE + threadIdx.x * 4 * Q;
  uint4 v[Q];
  uint32_t sum = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    v[q] = *reinterpret_cast<const uint4*>(bin_count + b0 + 4 * q);
    sum += v[q].x + v[q].y + v[q].z + v[q].w;
  }
  uint32_t total;
  const uint32_t ex = block_exclusive_scan(sum, &total, sm);
  if (threadIdx.x < 32) {
    const uint32_t pre = warp_lookback(status, tile, total, bs);
    if (threadIdx.x == 0) {
      s_prefix = pre;
      if (tile == NB / TILE - 1) {
        bin_start[NB] = pre + total;
        *ticket = 0;
      }
    }
  }
  __syncthreads();
  uint32_t run = s_prefix + ex;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    uint4 o;
    o.x = run; run += v[q].x;
    o.y = run; run += v[q].y;
    o.z = run; run += v[q].z;
    o.w = run; run += v[q].w;
    *reinterpret_cast<uint4*>(bin_start + b0 + 4 * q) = o;
  }
}

__device__ __forceinline__ void scan_body(const Batch& b, VB v) {
  if (!job_active(b, v.y)) return;
  const Job& jb = b.jobs[v.y];
  scan_bins<SCAN_TILE>(jb.bin_count, jb.bin_start, jb.scan_status, &jb.ctr->scan_ticket, b.bs);
}

static __global__ void __launch_bounds__(256) k_scan(Batch b) {
  pdl_trigger();
  pdl_wait();
  scan_body(b, hw_block());
}

// ---------------------------------------------------------------------------
// Stencil runs: the sorted-position ranges holding every point of the cells
// within n of cell k along each hashed dimension. f(rs, re) returns true to
// stop early.
// ---------------------------------------------------------------------------
template <int h, typename F>
__device__ __forceinline__ bool for_each_run(const uint32_t* bin_start, const int64_t* k, int n, F&& f) {
  const int rows = (h == 1) ? 1 : (h == 2 ? 2 * n + 1 : (2 * n + 1) * (2 * n + 1));
  for (int r = 0; r < rows; ++r) {
    int64_t c[3];
    if (h == 1) {
      c[0] = k[0] - n;
    } else if (h == 2) {
      c[0] = k[0] + r - n;
      c[1] = k[1] - n;
    } else {
      c[0] = k[0] + r / (2 * n + 1) - n;
      c[1] = k[1] + r % (2 * n + 1) - n;
      c[2] = k[2] - n;
    }
    const uint32_t b0 = bin_of(c, h);
    const uint32_t b1 = (b0 + 2 * n) & NB_MASK;
    if (b0 <= b1) {
      if (f(bin_start[b0], bin_start[b1 + 1])) return true;
    } else {
      if (f(bin_start[b0], bin_start[NB])) return true;
      if (f(bin_start[0], bin_start[b1 + 1])) return true;
    }
  }
  return false;
}

// ---------------------------------------------------------------------------
// k_scatter: window -> cell-ordered SoA (counting sort, warp-aggregated;
// positions are claimed with atomicSub so the bin counts end at zero),
// safe-inlier classification and the query queue.
// ---------------------------------------------------------------------------
// 1-d group filter. With cells of R(1+2^-12)/n, any n-1 consecutive cells
// span less than R (with the same margin argument as one cell for n = 2),
// and every point of the 2n-3 cells within n-2 of a cell lies within
// (n-1)/n (1+2^-12) R < R of every point of that cell. So a point is an
// inlier if those 2n-3 cells, or some run of n-1 consecutive cells containing
// its cell, hold more than K points, provided every bin involved holds
// exactly its expected cell (or nothing). Returns true when that holds.
__device__ __forceinline__ bool group_safe_1d(const Job& jb, uint64_t key, uint32_t b, bool pure) {
  const int m = jb.n - 1;
  if (m < 2 || b < (uint32_t)(m - 1) || b + m > NB - 1) return false;
  constexpr int MMAX = 7;
  uint32_t bs[2 * MMAX];
  bool ok[2 * MMAX - 1];
#pragma unroll
  for (int t = 0; t < 2 * MMAX; ++t)
    if (t < 2 * m) bs[t] = jb.bin_start[b - m + 1 + t];
#pragma unroll
  for (int t = 0; t < 2 * MMAX - 1; ++t) {
    if (t < 2 * m - 1) {
      const uint32_t j = b - m + 1 + t;
      const unsigned long long want = key + (unsigned long long)(t - (m - 1));
      ok[t] = pure || bs[t + 1] == bs[t] || (jb.kmin[j] == want && jb.kmax[j] == want);
    }
  }
  {  // the whole neighbourhood of 2n-3 cells: bins b-m+1 .. b+m-1
    bool all = true;
#pragma unroll
    for (int t = 0; t < 2 * MMAX - 1; ++t)
      if (t < 2 * m - 1) all &= ok[t];
    if (all && bs[2 * m - 1] - bs[0] > (uint32_t)jb.K) return true;
  }
#pragma unroll
  for (int g = 0; g < MMAX; ++g) {
    if (g < m) {
      bool pure = true;
#pragma unroll
      for (int t = 0; t < MMAX; ++t)
        if (t < m) pure &= ok[g + t];
      if (pure && bs[g + m] - bs[g] > (uint32_t)jb.K) return true;
    }
  }
  return false;
}

template <int D, bool ROUTE, typename T, bool GROUP = false>
__device__ __forceinline__ void scatter_body(const Batch& b, VB v) {
  // Block-local table: bin, points of the chunk in the bin, claimed base.
  __shared__ uint32_t tbin[HIST_SLOTS];
  __shared__ uint32_t tcnt[HIST_SLOTS];
  __shared__ uint32_t tbase[HIST_SLOTS];
  __shared__ unsigned long long s_routed[2];  // router statistics, flushed once per block
  if (!job_active(b, v.y)) return;
  if (ROUTE && threadIdx.x < 2) s_routed[threadIdx.x] = 0;
  constexpr int H = Hashed<D>::value;
  constexpr int U = Unroll<D>::value;
  const Job& jb = b.jobs[v.y];
  const int64_t lo = jb.ctr->lo;
  const bool pure = jb.ctr->pure;
  if (v.x == 0 && threadIdx.x < SCAN_TILES) jb.scan_status[threadIdx.x] = 0;
  for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
    tbin[t] = 0xffffffffu;
    tcnt[t] = 0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int64_t chunk = (int64_t)blockDim.x * U;
  for (int64_t c0 = (int64_t)v.x * chunk; c0 < jb.W; c0 += (int64_t)v.gx * chunk) {
    const int64_t w0 = c0 + (int64_t)(threadIdx.x >> 5) * 32 * U;
    int64_t src[U];
    uint64_t key[U];
    uint32_t bin[U], peers[U], goff[U];
    int leader[U], slot[U];
    // 1. keys of U chunks of 32
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = w0 + u * 32 + lane;
      src[u] = i < jb.W ? source_pos(jb, lo, i) : -1;
      key[u] = src[u] >= 0 ? jb.keys[src[u]] : EMPTY_KEY;
    }
    // 2. per warp group: slot in the block table and offset inside the block's share
#pragma unroll
    for (int u = 0; u < U; ++u) {
      bin[u] = src[u] >= 0 ? bin_of_key(key[u], H) : 0xffffffffu;
      peers[u] = __match_any_sync(0xffffffffu, bin[u]);
      leader[u] = __ffs(peers[u]) - 1;
      int sl_found = -1;
      uint32_t off = 0;
      if (src[u] >= 0 && lane == leader[u]) {
        const uint32_t c = (uint32_t)__popc(peers[u]);
        uint32_t sl = (bin[u] * 2654435761u) >> (32 - HIST_BITS);
#pragma unroll 1
        for (int probe = 0; probe < 8; ++probe) {
          const uint32_t old = atomicCAS(&tbin[sl], 0xffffffffu, bin[u]);
          if (old == 0xffffffffu || old == bin[u]) {
            off = atomicAdd(&tcnt[sl], c);
            sl_found = (int)sl;
            break;
          }
          sl = (sl + 1) & (HIST_SLOTS - 1);
        }
        if (sl_found < 0) {  // table full: claim directly
          const uint32_t top = atomicSub(&jb.bin_count[bin[u]], c);
          off = top - c;
        }
      }
      slot[u] = __shfl_sync(0xffffffffu, sl_found, leader[u]);
      goff[u] = __shfl_sync(0xffffffffu, off, leader[u]) + __popc(peers[u] & lt);
    }
    __syncthreads();
    // 3. one claim per bin of the chunk (positions [top - cnt, top) of the bin)
    for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
      const uint32_t bb = tbin[t];
      if (bb != 0xffffffffu) {
        const uint32_t c = tcnt[t];
        tbase[t] = atomicSub(&jb.bin_count[bb], c) - c;
        tbin[t] = 0xffffffffu;
        tcnt[t] = 0;
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool valid = src[u] >= 0;
      const int64_t i = w0 + u * 32 + lane;
      bool safe = false;
      uint32_t pos = 0, cnt = 0, bs0 = 0;
      if (valid) {
        bs0 = jb.bin_start[bin[u]];
        const uint32_t bs1 = jb.bin_start[bin[u] + 1];
        pos = bs0 + goff[u] + (slot[u] >= 0 ? tbase[slot[u]] : 0u);
        T x[D];
        load_point<D, T>(jb, src[u], x);
        jb.s_off[pos] = (uint32_t)i;
        jb.s_ckey[pos] = key[u];
#pragma unroll
        for (int d = 0; d < D; ++d) sx_row<T>(jb, d)[pos] = x[d];
        cnt = bs1 - bs0;
        if (jb.filter) {
          safe = cnt > (uint32_t)jb.K && (pure || jb.kmin[bin[u]] == jb.kmax[bin[u]]);
          if constexpr (H == 1) {
            if (!safe && jb.n >= 3) safe = group_safe_1d(jb, key[u], bin[u], pure);
          }
        }
        if (safe) jb.prev[src[u]] = 255;
      }
      const bool need = valid && !safe;
      if constexpr (GROUP) {
        // Group mode: a bin that needs counting (safety is decided per bin, so
        // every point of it does) is listed as parts of jb.gpts points, each
        // by the point at the part's first position.
        const bool emit = need && ((pos - bs0) & (uint32_t)(jb.gpts - 1)) == 0;
        const unsigned em = __ballot_sync(0xffffffffu, emit);
        if (em) {
          const uint32_t pts = __reduce_add_sync(0xffffffffu, emit && pos == bs0 ? cnt : 0u);
          const int ql = __ffs(em) - 1;
          uint32_t gb = 0;
          if (lane == ql) {
            gb = atomicAdd(reinterpret_cast<uint32_t*>(&jb.ctr->n_groups), (uint32_t)__popc(em));
            if (pts) atomicAdd(&jb.ctr->n_undet, (int)pts);
          }
          gb = __shfl_sync(0xffffffffu, gb, ql);
          if (emit) jb.queue[gb + __popc(em & lt)] = pos;
        }
        continue;
      }
      bool sweep = false;
      float f[MLP_IN] = {0.0f, 0.0f, 0.0f};
      if constexpr (ROUTE) {
        if (need) {
          // Router features (own bin, stencil row, last count) and one table lookup.
          int64_t k[3];
          unpack_key(key[u], H, k);
          int64_t c[3] = {k[0], k[1], k[2]};
          c[H - 1] -= jb.n;
          const uint32_t r0 = bin_of(c, H), r1 = r0 + 2 * jb.n + 1;
          const uint32_t row = r1 <= NB ? jb.bin_start[r1] - jb.bin_start[r0] : 0xffffffu;
          f[0] = log2f(1.0f + (float)cnt) * 0.125f;
          f[1] = log2f(1.0f + (float)row) * 0.125f;
          f[2] = prev_feature(jb.prev[src[u]], jb.K);
          const uint32_t rows = H == 1 ? 1u : (H == 2 ? 2u * jb.n + 1u : (2u * jb.n + 1u) * (2u * jb.n + 1u));
          sweep = row * rows <= b.router->max_sweep && !route_early(b.router, f);
        }
      }
      const unsigned need_e = __ballot_sync(0xffffffffu, need && !sweep);
      if (need_e) {
        uint32_t qb = 0;
        const int ql = __ffs(need_e) - 1;
        if (lane == ql) qb = (uint32_t)atomicAdd(&jb.ctr->n_undet, __popc(need_e));
        qb = __shfl_sync(0xffffffffu, qb, ql);
        if (need && !sweep) {
          const uint32_t q = qb + __popc(need_e & lt);
          jb.queue[q] = pos;
          if constexpr (ROUTE) {
#pragma unroll
            for (int j = 0; j < MLP_IN; ++j) jb.feat[(int64_t)q * MLP_IN + j] = f[j];
          }
        }
      }
      if constexpr (ROUTE) {
        const unsigned need_s = __ballot_sync(0xffffffffu, sweep);
        if (need_s) {
          uint32_t qb = 0;
          const int ql = __ffs(need_s) - 1;
          if (lane == ql) qb = (uint32_t)atomicAdd(&jb.ctr->n_sweep, __popc(need_s));
          qb = __shfl_sync(0xffffffffu, qb, ql);
          if (sweep) {
            const uint32_t q = (uint32_t)jb.W - 1 - (qb + __popc(need_s & lt));
            jb.queue[q] = pos;
#pragma unroll
            for (int j = 0; j < MLP_IN; ++j) jb.feat[(int64_t)q * MLP_IN + j] = f[j];
          }
        }
        if (lane == 0 && (need_e || need_s)) {
          atomicAdd(&s_routed[0], (unsigned long long)__popc(need_e));
          atomicAdd(&s_routed[1], (unsigned long long)__popc(need_s));
        }
      }
    }
  }
  if constexpr (ROUTE) {
    __syncthreads();
    if (threadIdx.x == 0 && s_routed[0]) atomicAdd(&b.router->routed_early, s_routed[0]);
    if (threadIdx.x == 1 && s_routed[1]) atomicAdd(&b.router->routed_sweep, s_routed[1]);
  }
}

template <int D, bool ROUTE, typename T, bool GROUP = false>
__global__ void __launch_bounds__(256) k_scatter(Batch b) {
  pdl_trigger();
  pdl_wait();
  scatter_body<D, ROUTE, T, GROUP>(b, hw_block());
}

// Counts the neighbours of query qx among the candidates of one run
// [rs, re), 128 per step: each lane loads 4 consecutive candidates per
// dimension with one float4, the warp tallies them with ballot/popc.
// Returns true once the running total exceeds K.
template <int D, int PRED, typename T>
__device__ __forceinline__ bool count_run(const Job& jb, const T* qx, uint32_t rs, uint32_t re,
                                          int& total) {
  const int lane = threadIdx.x & 31;
  for (uint32_t b = rs & ~3u; b < re; b += 128) {
    const uint32_t c0 = b + 4 * lane;
    bool in[4] = {false, false, false, false};
    if (c0 < re) {
      T v[D][4];
#pragma unroll
      for (int d = 0; d < D; ++d) load4(sx_row<T>(jb, d) + c0, v[d]);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        T cx[D];
#pragma unroll
        for (int d = 0; d < D; ++d) cx[d] = v[d][e];
        const uint32_t c = c0 + e;
        in[e] = c >= rs && c < re && is_nbr<D, PRED, T>(qx, cx, jb.R2f, jb.R, jb.R2);
      }
    }
    total += __popc(__ballot_sync(0xffffffffu, in[0])) + __popc(__ballot_sync(0xffffffffu, in[1])) +
             __popc(__ballot_sync(0xffffffffu, in[2])) + __popc(__ballot_sync(0xffffffffu, in[3]));
    if (total > jb.K) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Row-parallel count for 2 and 3 hashed dimensions. The (2n+1)^(h-1) stencil
// rows are taken nearest first (centre row, then by distance); lane r fetches
// the bounds of rows r and r+32 in one round trip, a warp scan turns the row
// lengths into offsets of one virtual concatenated candidate list, and the
// warp consumes that list 128 candidates per step across row boundaries (each
// lane finds the row of its candidates by binary search over the offsets).
// Returns false in *ok when a row wraps around the end of the bin table; the
// caller then uses the row-by-row count.
// ---------------------------------------------------------------------------
static __constant__ uint8_t c_rows2[3][7] = {{1, 0, 2}, {2, 1, 3, 0, 4}, {3, 2, 4, 1, 5, 0, 6}};
static __constant__ uint8_t c_rows3[3][49] = {
    {4, 3, 5, 1, 7, 0, 2, 6, 8},
    {12, 11, 13, 7, 17, 6, 8, 16, 18, 10, 14, 2, 22, 5, 9, 15, 19, 1, 3, 21, 23, 0, 4, 20, 24},
    {24, 23, 25, 17, 31, 16, 18, 30, 32, 22, 26, 10, 38, 15, 19, 29, 33, 9, 11, 37, 39, 8, 12, 36, 40,
     21, 27, 3, 45, 14, 20, 28, 34, 2, 4, 44, 46, 7, 13, 35, 41, 1, 5, 43, 47, 0, 6, 42, 48}};

template <int D, int PRED, typename T>
__device__ __forceinline__ bool count_query_rows(const Job& jb, uint32_t pos, int& total, bool* ok) {
  constexpr int H = Hashed<D>::value;
  static_assert(H >= 2, "row-parallel count needs 2 or 3 hashed dimensions");
  const int lane = threadIdx.x & 31;
  const int n = jb.n, span = 2 * n + 1;
  const int rows = (H == 2) ? span : span * span;
  T qx[D];
#pragma unroll
  for (int d = 0; d < D; ++d) qx[d] = sx_row<T>(jb, d)[pos];
  int64_t k[3];
  unpack_key(jb.s_ckey[pos], H, k);
  uint32_t rs[2] = {0, 0}, len[2] = {0, 0};
  bool wrap = false;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int slot = lane + 32 * t;
    if (slot < rows) {
      const int r = (H == 2) ? c_rows2[n - 1][slot] : c_rows3[n - 1][slot];
      int64_t c[3];
      if (H == 2) {
        c[0] = k[0] + r - n;
        c[1] = k[1] - n;
      } else {
        c[0] = k[0] + r / span - n;
        c[1] = k[1] + r % span - n;
        c[2] = k[2] - n;
      }
      const uint32_t b0 = bin_of(c, H);
      if (b0 + 2 * n > NB_MASK) {
        wrap = true;
      } else {
        rs[t] = jb.bin_start[b0];
        len[t] = jb.bin_start[b0 + 2 * n + 1] - rs[t];
      }
    }
  }
  total = 0;
  *ok = !__any_sync(0xffffffffu, wrap);
  if (!*ok) return false;
  // exclusive offsets of the 64 row slots (slot = lane + 32 t)
  uint32_t off[2], ncand = 0;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    uint32_t inc = len[t];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    off[t] = ncand + inc - len[t];
    ncand += __shfl_sync(0xffffffffu, inc, 31);
  }
  for (uint32_t v0 = 0; v0 < ncand; v0 += 128) {
    bool in[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const uint32_t v = v0 + 32 * e + lane;
      in[e] = false;
      // row slot holding v: the last slot whose offset is <= v (binary search over 64 slots)
      int lo_s = 0;
#pragma unroll
      for (int step = 32; step > 0; step >>= 1) {
        const int cand = lo_s + step;
        const uint32_t o0 = __shfl_sync(0xffffffffu, off[0], cand & 31);
        const uint32_t o1 = __shfl_sync(0xffffffffu, off[1], cand & 31);
        const uint32_t oc = cand < 32 ? o0 : o1;
        if (cand < 64 && oc <= v) lo_s = cand;
      }
      const uint32_t base0 = __shfl_sync(0xffffffffu, rs[0], lo_s & 31);
      const uint32_t base1 = __shfl_sync(0xffffffffu, rs[1], lo_s & 31);
      const uint32_t oo0 = __shfl_sync(0xffffffffu, off[0], lo_s & 31);
      const uint32_t oo1 = __shfl_sync(0xffffffffu, off[1], lo_s & 31);
      if (v < ncand) {
        const uint32_t c = (lo_s < 32 ? base0 : base1) + (v - (lo_s < 32 ? oo0 : oo1));
        T cx[D];
#pragma unroll
        for (int d = 0; d < D; ++d) cx[d] = sx_row<T>(jb, d)[c];
        in[e] = is_nbr<D, PRED, T>(qx, cx, jb.R2f, jb.R, jb.R2);
      }
    }
    total += __popc(__ballot_sync(0xffffffffu, in[0])) + __popc(__ballot_sync(0xffffffffu, in[1])) +
             __popc(__ballot_sync(0xffffffffu, in[2])) + __popc(__ballot_sync(0xffffffffu, in[3]));
    if (total > jb.K) return true;
  }
  return false;
}

// Exact count of one queued point by the whole warp: `total` receives the
// count (capped just above K); returns true if it exceeded K.
template <int D, int PRED, typename T>
__device__ __forceinline__ bool count_query(const Job& jb, uint32_t pos, int& total) {
  constexpr int H = Hashed<D>::value;
  if constexpr (H >= 2) {
    bool ok;
    const bool r = count_query_rows<D, PRED, T>(jb, pos, total, &ok);
    if (ok) return r;
  }
  T qx[D];
#pragma unroll
  for (int d = 0; d < D; ++d) qx[d] = sx_row<T>(jb, d)[pos];
  int64_t k[3];
  unpack_key(jb.s_ckey[pos], H, k);
  total = 0;
  return for_each_run<H>(jb.bin_start, k, jb.n, [&](uint32_t rs, uint32_t re) {
    return count_run<D, PRED, T>(jb, qx, rs, re, total);
  });
}

// Exact count of one queued point by one lane (full-sweep queue): the
// candidates are read 8 at a time, so that their loads are in flight together.
template <int D, int PRED, typename T>
__device__ __forceinline__ bool count_query_lane(const Job& jb, uint32_t pos, int& total) {
  constexpr int H = Hashed<D>::value;
  T qx[D];
#pragma unroll
  for (int d = 0; d < D; ++d) qx[d] = sx_row<T>(jb, d)[pos];
  int64_t k[3];
  unpack_key(jb.s_ckey[pos], H, k);
  total = 0;
  return for_each_run<H>(jb.bin_start, k, jb.n, [&](uint32_t rs, uint32_t re) {
    for (uint32_t c0 = rs; c0 < re; c0 += 8) {
      T cx[8][D];
#pragma unroll
      for (int e = 0; e < 8; ++e)
#pragma unroll
        for (int d = 0; d < D; ++d) cx[e][d] = c0 + e < re ? sx_row<T>(jb, d)[c0 + e] : T(0);
#pragma unroll
      for (int e = 0; e < 8; ++e) total += (c0 + e < re) && is_nbr<D, PRED, T>(qx, cx[e], jb.R2f, jb.R, jb.R2);
      if (total > jb.K) return true;
    }
    return false;
  });
}

// Records the result of one counted point (one thread).
__device__ __forceinline__ void record_count(const Job& jb, int64_t lo, uint32_t pos, bool inlier, int total) {
  const uint32_t i = jb.s_off[pos];
  if (!inlier) {
    atomicOr(&jb.flags[i >> 5], 1u << (i & 31));
    atomicAdd(&jb.ctr->n_out, 1);
  }
  jb.prev[source_pos(jb, lo, i)] = (uint8_t)(total < 253 ? total : 253);
}

// Block-local buffer of router training samples and misroute count of
// k_count, flushed to the router state once per block.
constexpr int BLOCK_SAMPLES = 64;
struct SampleBuf {
  float s[BLOCK_SAMPLES][4];
  uint32_t n;
  uint32_t misrouted;
};

// Training sample of one routed point (one thread): its features and the
// bucket of its exact capped count. Inliers (most points) are thinned to one
// in INLIER_THIN by queue index so that the buckets are closer to balanced.
__device__ __forceinline__ void record_sample(const Job& jb, SampleBuf& sb, int64_t q, int total,
                                              bool routed_early) {
  const int lab = count_bucket(total, jb.K);
  if ((lab == 3) != routed_early) atomicAdd(&sb.misrouted, 1u);
  if (lab == 3 && (q % INLIER_THIN) != 0) return;
  const uint32_t s = atomicAdd(&sb.n, 1u);
  if (s >= BLOCK_SAMPLES) return;
#pragma unroll
  for (int j = 0; j < MLP_IN; ++j) sb.s[s][j] = jb.feat[q * MLP_IN + j];
  sb.s[s][3] = (float)lab;
}

__device__ __forceinline__ void flush_samples(SampleBuf& sb, RouterState* rs) {
  __syncthreads();
  __shared__ uint32_t s_base;
  const uint32_t n = min(sb.n, (uint32_t)BLOCK_SAMPLES);
  if (threadIdx.x == 0) {
    if (sb.misrouted) atomicAdd(&rs->misrouted, (unsigned long long)sb.misrouted);
    s_base = (n && *(volatile uint32_t*)&rs->n_samples < TRAIN_CAP) ? atomicAdd(&rs->n_samples, n) : TRAIN_CAP;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t dst = s_base + i;
    if (dst < TRAIN_CAP)
#pragma unroll
      for (int j = 0; j < 4; ++j) rs->samples[dst][j] = sb.s[i][j];
  }
}

// Per-job cleanup done by k_count: per-bin key ranges and compaction
// look-back words.
__device__ __forceinline__ void reset_bins(const Job& jb, VB v) {
  const int64_t stride = (int64_t)v.gx * blockDim.x;
  for (int64_t t = (int64_t)v.x * blockDim.x + threadIdx.x; t < NB; t += stride) {
    jb.kmin[t] = EMPTY_KEY;
    jb.kmax[t] = 0;
  }
  const int64_t tiles = (jb.W + CMP_TILE - 1) / CMP_TILE;
  for (int64_t t = (int64_t)v.x * blockDim.x + threadIdx.x; t < tiles; t += stride)
    jb.cmp_status[t] = 0;
}

// ---------------------------------------------------------------------------
// Batch-wide count list. The count work of every job of a launch (parts of
// bins in group mode, runs of queued points otherwise) forms one list,
// job after job, that warps take entry by entry from BatchState::count_ticket.
// Every warp of the launch keeps working while any job has work left: a
// job with many entries (a long or dense window among short ones) is not
// left to the blocks that the grid assigns to it alone.
// ---------------------------------------------------------------------------
constexpr int BATCH_JOBS_MAX = 256;  // jobs per launch (the host's limit is checked against it)
constexpr uint32_t COUNT_RUN = 16;   // queued points per entry of a point-count list

// s_pre[j] = entries of jobs 0..j-1 (inactive jobs hold none); returns the
// total. Every thread of the block calls it.
template <class Entries>
__device__ __forceinline__ uint32_t count_list_prefix(const Batch& b, uint32_t* s_pre, uint32_t* s_scan,
                                                      Entries entries) {
  const int nj = b.njobs;
  const int per = (nj + (int)blockDim.x - 1) / (int)blockDim.x;
  const int j0 = min(nj, (int)threadIdx.x * per), j1 = min(nj, j0 + per);
  uint32_t mine = 0;
  for (int j = j0; j < j1; ++j)
    if (job_active(b, j)) mine += entries(b.jobs[j]);
  uint32_t total;
  uint32_t ex = block_exclusive_scan(mine, &total, s_scan);
  for (int j = j0; j < j1; ++j) {
    s_pre[j] = ex;
    if (job_active(b, j)) ex += entries(b.jobs[j]);
  }
  __syncthreads();
  return total;
}

// The job of list entry t < total: the last j with s_pre[j] <= t (jobs
// without entries repeat their successor's offset and are skipped).
__device__ __forceinline__ int count_list_job(const uint32_t* s_pre, int nj, uint32_t t) {
  int lo = 0, hi = nj;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s_pre[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Next list entry for the calling warp (the same on every lane).
__device__ __forceinline__ uint32_t count_list_take(BatchState* bs) {
  uint32_t t = 0;
  if ((threadIdx.x & 31) == 0) t = atomicAdd(&bs->count_ticket, 1u);
  return __shfl_sync(0xffffffffu, t, 0);
}

// ---------------------------------------------------------------------------
// k_count: the exact count always decides: outlier iff count <= K.
//   plain (ROUTE = false): one warp per queued point, stencil rows in order;
//     a single job's warps stride over its queue, the jobs of a multi-job
//     launch share the batch-wide list in runs of COUNT_RUN points.
//   group mode: one warp per listed part of a bin, parts taken from the
//     batch-wide list.
//   routed: early-exit queue as above; full-sweep queue one lane per point,
//     32 points per warp, each lane sweeping its own (short) candidate list;
//     every counted point becomes a training sample of the router.
// ---------------------------------------------------------------------------
template <int D, int PRED, bool ROUTE, typename T, bool GROUP = false>
__device__ __forceinline__ void count_body(const Batch& b, VB v) {
  __shared__ SampleBuf sb;
  const bool home = job_active(b, v.y);
  if constexpr (GROUP || !ROUTE) {
    if (GROUP || b.njobs > 1) {
      // the batch-wide list: this block's share of its own job's resets,
      // then entries of any job until the list runs out
      __shared__ uint32_t s_pre[BATCH_JOBS_MAX];
      __shared__ uint32_t s_scan[33];
      if (home) reset_bins(b.jobs[v.y], v);
      const int lane = threadIdx.x & 31;
      if constexpr (GROUP) {
        // one warp per listed part of a bin: its points share the stencil (count_group)
        constexpr int H = Hashed<D>::value;
        const uint32_t total =
            count_list_prefix(b, s_pre, s_scan, [](const Job& j) { return (uint32_t)j.ctr->n_groups; });
        for (;;) {
          const uint32_t t = count_list_take(b.bs);
          if (t >= total) break;
          const int j = count_list_job(s_pre, b.njobs, t);
          const Job& J = b.jobs[j];
          const uint32_t p = J.queue[t - s_pre[j]];
          const uint32_t bin = bin_of_key(J.s_ckey[p], H);
          const uint32_t nq = min((uint32_t)J.gpts, J.bin_start[bin + 1] - p);
          const GroupArgs ga{p,   nq,   bin,  J.n,  J.K, J.R2f, J.R, J.R2, J.Wp, J.ctr->pure && D <= 3,
                             &b.bs->pair_tests};
          const int nout = count_group<D, PRED, T>(
              static_cast<const T*>(J.s_x), ga,
              [&](uint32_t sb2, uint32_t& rs, uint32_t& len) {
                rs = J.bin_start[sb2];
                len = J.bin_start[sb2 + 1] - rs;
              },
              [&](uint32_t pos) {
                const uint32_t i = J.s_off[pos];
                atomicOr(&J.flags[i >> 5], 1u << (i & 31));
              });
          if (lane == 0 && nout) atomicAdd(&J.ctr->n_out, nout);
        }
      } else {
        const uint32_t total = count_list_prefix(b, s_pre, s_scan, [](const Job& j) {
          return ((uint32_t)j.ctr->n_undet + COUNT_RUN - 1) / COUNT_RUN;
        });
        for (;;) {
          const uint32_t t = count_list_take(b.bs);
          if (t >= total) break;
          const int j = count_list_job(s_pre, b.njobs, t);
          const Job& J = b.jobs[j];
          const int64_t lo = J.ctr->lo;
          const uint32_t q0 = (t - s_pre[j]) * COUNT_RUN;
          const uint32_t q1 = min((uint32_t)J.ctr->n_undet, q0 + COUNT_RUN);
          for (uint32_t q = q0; q < q1; ++q) {
            const uint32_t pos = J.queue[q];
            int cnt;
            const bool inlier = count_query<D, PRED, T>(J, pos, cnt);
            if (lane == 0) record_count(J, lo, pos, inlier, cnt);
          }
        }
      }
      return;
    }
  }
  if (!home) return;
  const Job& jb = b.jobs[v.y];
  if (ROUTE && threadIdx.x == 0) {
    sb.n = 0;
    sb.misrouted = 0;
  }
  if (ROUTE) __syncthreads();
  reset_bins(jb, v);
  const int lane = threadIdx.x & 31;
  const int64_t lo = jb.ctr->lo;
  const int64_t warp = ((int64_t)v.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)v.gx * blockDim.x) >> 5;
  const int64_t nq = jb.ctr->n_undet;
  for (int64_t q = warp; q < nq; q += nwarps) {
    const uint32_t pos = jb.queue[q];
    int total;
    const bool inlier = count_query<D, PRED, T>(jb, pos, total);
    if (lane == 0) {
      record_count(jb, lo, pos, inlier, total);
      if constexpr (ROUTE) record_sample(jb, sb, q, total, true);
    }
  }
  if constexpr (ROUTE) {
    const int64_t ns = jb.ctr->n_sweep;
    for (int64_t c0 = warp * 32; c0 < ns; c0 += nwarps * 32) {
      const int64_t idx = c0 + lane;
      if (idx < ns) {
        const int64_t q = jb.W - 1 - idx;
        const uint32_t pos = jb.queue[q];
        int total;
        const bool inlier = count_query_lane<D, PRED, T>(jb, pos, total);
        record_count(jb, lo, pos, inlier, total);
        record_sample(jb, sb, q, total, false);
      }
    }
    flush_samples(sb, b.router);
  }
}

template <int D, int PRED, bool ROUTE, typename T, bool GROUP = false>
__global__ void __launch_bounds__(256) k_count(Batch b) {
  pdl_trigger();
  pdl_wait();
  count_body<D, PRED, ROUTE, T, GROUP>(b, hw_block());
}

// ---------------------------------------------------------------------------
// End of a batch, run by the block of the batch's last kernel that finishes
// last (after a fence): per-slide records (outlier count, counted points and,
// where kept, the slide's output offset in window order), window advance,
// per-job counter reset and the batch totals. Every thread of the block
// calls it.
// ---------------------------------------------------------------------------
static __device__ void finish_batch(const Batch& b) {
  __shared__ int64_t s_red[3][32];
  __shared__ int64_t s_scan[33];
  BatchState* bs = b.bs;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  __threadfence();
  // jobs in contiguous runs per thread, so that an exclusive scan over the
  // threads gives each slide its output offset in window order
  const int per = (b.njobs + (int)blockDim.x - 1) / (int)blockDim.x;
  const int j0 = min(b.njobs, (int)threadIdx.x * per), j1 = min(b.njobs, j0 + per);
  int64_t mine = 0;
  for (int j = j0; j < j1; ++j)
    if (!b.active || b.active[j]) mine += *(volatile int32_t*)&b.jobs[j].ctr->n_out;
  int64_t inc = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_scan[wid] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t run = bs->out_total;  // IDs of the earlier batches
    for (int w = 0; w < nw; ++w) {
      const int64_t t = s_scan[w];
      s_scan[w] = run;
      run += t;
    }
  }
  __syncthreads();
  int64_t base = s_scan[wid] + inc - mine;
  int64_t add = 0, und = 0, nact = 0;
  for (int j = j0; j < j1; ++j) {
    if (b.active && !b.active[j]) {
      if (b.job_nout) b.job_nout[j] = 0;
      continue;
    }
    const Job& J = b.jobs[j];
    JobCtr* c = J.ctr;
    const int32_t nout = *(volatile int32_t*)&c->n_out;
    const int32_t nund = *(volatile int32_t*)&c->n_undet + *(volatile int32_t*)&c->n_sweep;
    const int64_t slide = (c->lo - J.S) / J.S;
    if (J.rec_nout && slide >= 0 && slide < J.rec_cap) {
      J.rec_nout[slide] = nout;
      J.rec_undet[slide] = nund;
      if (J.rec_base) J.rec_base[slide] = base;
    }
    base += nout;
    add += nout;
    und += nund;
    nact += 1;
    c->last_nout = nout;
    if (b.job_nout) b.job_nout[j] = nout;
    c->lo += c->lo_step;
    c->n_out = 0;
    c->n_undet = 0;
    c->n_sweep = 0;
    c->n_groups = 0;
    c->cmp_ticket = 0;
  }
#pragma unroll
  for (int o2 = 16; o2 > 0; o2 >>= 1) {
    add += __shfl_xor_sync(0xffffffffu, add, o2);
    und += __shfl_xor_sync(0xffffffffu, und, o2);
    nact += __shfl_xor_sync(0xffffffffu, nact, o2);
  }
  if (lane == 0) {
    s_red[0][wid] = add;
    s_red[1][wid] = und;
    s_red[2][wid] = nact;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t ta = 0, tu = 0, tn = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      ta += s_red[0][w];
      tu += s_red[1][w];
      tn += s_red[2][w];
    }
    bs->out_total += ta;
    bs->undet_total += tu;
    bs->slides += tn;
    bs->done = 0;
    bs->count_ticket = 0;
    if (b.span) {
      b.span->n_used = 0;
      b.span->n_groups = 0;
      b.span->n_segs = 0;
      b.span->seg_ticket = 0;
      b.span->group_ticket = 0;
      for (int d = 0; d < 3; ++d) {
        b.span->cmin[d] = LLONG_MAX;
        b.span->cmax[d] = LLONG_MIN;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Head and tail of an rtod_run pass (kernels, so that a captured run has no
// host copy at either end).
// k_run_init: job j's counters start at window lo = first_lo + j*S and
// advance by jobs*S per batch; the batch state is cleared.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(256) k_run_init(JobCtr* ctr, int32_t jobs, int64_t first_lo, int64_t S,
                                                  BatchState* bs) {
  pdl_trigger();
  pdl_wait();
  for (int j = threadIdx.x; j < jobs; j += blockDim.x) {
    JobCtr c{};
    c.lo = first_lo + (int64_t)j * S;
    c.lo_step = (int64_t)jobs * S;
    ctr[j] = c;
  }
  if (threadIdx.x == 0) *bs = BatchState{};
}

// k_run_out: the outlier IDs (at most cap) into a caller's page-locked host
// buffer through its device mapping (consecutive 8-byte writes, one per
// thread), then the batch state into the handle's mapped mirror.
static __global__ void __launch_bounds__(256) k_run_out(const int64_t* ids, int64_t* host_ids, int64_t cap,
                                                 const BatchState* bs, BatchState* mirror) {
  pdl_trigger();
  pdl_wait();
  if (host_ids) {
    const int64_t n = min(bs->out_total, cap);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      host_ids[i] = ids[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *mirror = *bs;
}

// ---------------------------------------------------------------------------
// k_compact: outlier bits in window order -> sorted global indices, appended
// to the batch output after the outliers of the earlier jobs. Grid
// (max tiles per job, jobs); a tile covers CMP_TILE window offsets, one
// 32-bit word per thread, tiles chained by decoupled look-back. The last
// tile of the batch records per-slide counts, advances every job's window
// and resets the per-job counters.
// ---------------------------------------------------------------------------
// Returns true in the block that ran finish_batch.
__device__ __forceinline__ bool compact_body(const Batch& b, VB v) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t s_tile, s_prefix, s_last;
  __shared__ int64_t s_jobbase;
  const Job& jb = b.jobs[v.y];
  const int64_t ntiles = (jb.W + CMP_TILE - 1) / CMP_TILE;
  if (v.x >= ntiles) return false;  // smaller job in a mixed batch
  BatchState* bs = b.bs;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool act = job_active(b, v.y);
  if (act && wid == 0) {
    // Output base of this job: IDs of all earlier jobs of the batch come first.
    int64_t part = 0;
    for (int j = lane; j < (int)v.y; j += 32) part += b.jobs[j].ctr->n_out;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) {
      s_jobbase = bs->out_total + part;
      s_tile = atomicAdd(&jb.ctr->cmp_ticket, 1u);
    }
  }
  __syncthreads();
  if (act) {
    const uint32_t tile = s_tile;
    const int64_t lo = jb.ctr->lo;
    const int64_t wi = ((int64_t)tile * CMP_TILE >> 5) + threadIdx.x;  // bitset word
    const int64_t nwords = (jb.W + 31) >> 5;
    uint32_t bits = 0;
    if (wi < nwords) {
      bits = jb.flags[wi];
      if (bits) jb.flags[wi] = 0;
    }
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(__popc(bits), &total, sm);
    if (wid == 0) {
      const uint32_t pre = warp_lookback(jb.cmp_status, tile, total, bs);
      if (lane == 0) s_prefix = pre;
    }
    __syncthreads();
    int64_t o = s_jobbase + s_prefix + ex;
    while (bits) {
      const int e = __ffs(bits) - 1;
      bits &= bits - 1;
      if (o < b.out_cap) b.out_ids[o] = lo + wi * 32 + e;
      else set_err(bs, DERR_CAPACITY);
      ++o;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&bs->done, 1u) == (uint32_t)(b.cmp_tiles - 1));
  __syncthreads();
  if (!s_last) return false;
  finish_batch(b);
  return true;
}

static __global__ void __launch_bounds__(256) k_compact(Batch b) {
  pdl_trigger();
  pdl_wait();
  compact_body(b, hw_block());
}

// ---------------------------------------------------------------------------
// k_compact_one: the compaction of windows of at most COMPACT1_MAX offsets,
// one block of 1024 threads per job (grid = jobs): the job's whole bitset in
// one block scan (CMP1_WPT words per thread), no look-back chain between
// tiles. The block that finishes last ends the batch (finish_batch) and, for
// a streaming detection, writes the IDs and the batch state into the mapped
// page-locked landing buffers (k_run_out's work, folded in). A thread's 8
// bitset words are one 32-byte sector, read and cleared as two 16-byte
// vectors; the job's IDs are gathered in shared memory (up to CMP1_SMEM_IDS)
// and written out by consecutive threads: one thread's run of single 8-byte
// stores held the block about 9 us on B200, the coalesced copy 2-3 us.
// ---------------------------------------------------------------------------
constexpr int CMP1_WPT = 8;
constexpr int64_t COMPACT1_MAX = 1024 * 32 * CMP1_WPT;  // 262144 window offsets
constexpr uint32_t CMP1_SMEM_IDS = 4096;

static __global__ void __launch_bounds__(1024) k_compact_one(Batch b, int64_t* ids_host, int64_t ids_host_cap,
                                                             BatchState* mirror) {
  __shared__ uint32_t sm[33];
  __shared__ int64_t s_jobbase;
  __shared__ uint32_t s_last;
  __shared__ int64_t s_ids[CMP1_SMEM_IDS];
  pdl_trigger();
  pdl_wait();
  const uint32_t job = blockIdx.x;
  const Job& jb = b.jobs[job];
  BatchState* bs = b.bs;
  if (*(volatile int32_t*)&bs->err == DERR_GRID) {
    // the streaming grid could not take the slide and nothing was counted:
    // no batch end; the host rebuilds the grid and counts the window again
    if (blockIdx.x == 0 && threadIdx.x == 0 && mirror) *mirror = *bs;
    return;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool act = job_active(b, job);
  if (act && wid == 0) {
    // Output base of this job: IDs of all earlier jobs of the batch come first.
    int64_t part = 0;
    for (int j = lane; j < (int)job; j += 32)
      if (job_active(b, j)) part += b.jobs[j].ctr->n_out;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) s_jobbase = bs->out_total + part;
  }
  __syncthreads();
  if (act) {
    const int64_t lo = jb.ctr->lo;
    const int64_t nwords = (jb.W + 31) >> 5;
    const int64_t w0 = (int64_t)threadIdx.x * CMP1_WPT;
    uint32_t bits[CMP1_WPT];
    uint32_t cnt = 0;
    if (w0 + CMP1_WPT <= nwords) {  // bitsets start 256-byte aligned
      uint4* f4 = reinterpret_cast<uint4*>(jb.flags + w0);
      const uint4 a = f4[0], c = f4[1];
      bits[0] = a.x; bits[1] = a.y; bits[2] = a.z; bits[3] = a.w;
      bits[4] = c.x; bits[5] = c.y; bits[6] = c.z; bits[7] = c.w;
      if ((a.x | a.y | a.z | a.w | c.x | c.y | c.z | c.w) != 0u) {
        f4[0] = make_uint4(0u, 0u, 0u, 0u);
        f4[1] = make_uint4(0u, 0u, 0u, 0u);
      }
    } else {
#pragma unroll
      for (int e = 0; e < CMP1_WPT; ++e) {
        bits[e] = w0 + e < nwords ? jb.flags[w0 + e] : 0u;
        if (bits[e]) jb.flags[w0 + e] = 0;
      }
    }
#pragma unroll
    for (int e = 0; e < CMP1_WPT; ++e) cnt += __popc(bits[e]);
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(cnt, &total, sm);
    if (total <= CMP1_SMEM_IDS && s_jobbase + total <= b.out_cap) {
      uint32_t k = ex;
#pragma unroll
      for (int e = 0; e < CMP1_WPT; ++e) {
        uint32_t v = bits[e];
        while (v) {
          const int f = __ffs(v) - 1;
          v &= v - 1;
          s_ids[k++] = lo + (w0 + e) * 32 + f;
        }
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) b.out_ids[s_jobbase + i] = s_ids[i];
    } else {
      int64_t o = s_jobbase + ex;
#pragma unroll
      for (int e = 0; e < CMP1_WPT; ++e) {
        uint32_t v = bits[e];
        while (v) {
          const int f = __ffs(v) - 1;
          v &= v - 1;
          if (o < b.out_cap) b.out_ids[o] = lo + (w0 + e) * 32 + f;
          else set_err(bs, DERR_CAPACITY);
          ++o;
        }
      }
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&bs->done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  finish_batch(b);
  if (ids_host || mirror) {
    __syncthreads();
    __threadfence();
    if (ids_host) {
      const int64_t n = min(bs->out_total, ids_host_cap);
      for (int64_t i = threadIdx.x; i < n; i += blockDim.x) ids_host[i] = b.out_ids[i];
    }
    __syncthreads();
    // No system-scope fence: the host reads the landing buffers only after
    // its stream wait, by which time the kernel's writes are visible (a
    // fence here held the block for about 20 us on B200).
    if (mirror && threadIdx.x == 0) *mirror = *bs;
  }
}

}  // namespace rtod
