// Device code of the per-slide detector pipeline (sm_100a).
//
// One slide runs six kernels, in stream order:
//   k_ingest   ring-buffer window update: the S new points go to their ring
//              slots (slot = global index % W) as SoA, each gets its packed
//              grid-cell key; per-slide bins and flags are cleared.
//              Replaces the H2D at src/ods/optixScan.cpp:1051-1058, the host
//              mirror at :1062-1064 and the resets at :1047-1050.
//   k_hist     cell occupancy: per-bin point counts and a "bin holds more
//              than one cell" flag. Replaces the expire/insert bookkeeping of
//              prepare_c_non_points_queue (:967-981) and FixQueue (state.h).
//   k_scan     exclusive scan of the bin counts -> bin starts.
//   k_scatter  counting sort of the window into cell order (slot, key and
//              coordinates as SoA). Together with k_scan this replaces
//              kGenAABB (aabb.cu:5-45) and the BVH rebuild (:378-426).
//   k_count    range count with K early exit and safe-inlier skip. Replaces
//              the ray launch and intersection program (optixScan.cu:21-75,
//              :158-199) and the all-inlier cell filter (:983-993).
//   k_compact  outlier flags -> sorted global indices, per-slide counters;
//              replaces the D2H + host pick at :1083-1101 and advances the
//              window (:1103-1108).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rtod {

constexpr int NB_LOG2 = 16;
constexpr uint32_t NB = 1u << NB_LOG2;  // bins of the cell hash table
constexpr uint32_t NB_MASK = NB - 1;
constexpr uint64_t EMPTY_KEY = ~0ull;

// Device error codes (first one wins).
enum : int32_t { DERR_NONE = 0, DERR_NONFINITE = 1, DERR_RANGE = 2, DERR_CAPACITY = 3 };

// Stream state that lives on the device, so that a captured slide graph can
// be replayed without host-side parameter changes.
struct DevState {
  int64_t n_ingested;   // points written to the ring so far (= next global index)
  int64_t out_total;    // outlier IDs appended to out_ids so far
  int64_t slide;        // slides detected so far
  int64_t undet_total;  // counted (undetermined) points summed over slides
  int32_t err;          // DERR_*
  int32_t n_out;        // outliers of the last slide
  int32_t n_undet;      // counted points of the last slide
  int32_t pad;
};

struct KParams {
  int64_t W, S;
  int32_t D;       // dimensions
  int32_t h;       // hashed dimensions (min(D, 3))
  int32_t n;       // cells per R: cell side = R*(1+2^-12)/n, stencil reach n cells
  int32_t K;
  int32_t filter;  // safe-inlier skip (grid filter) enabled
  int32_t src_staging;  // 1: src holds exactly the points being ingested
  double cell;
  double R, R2;
  float R2f;
  const float* src;     // points to ingest, point-major
  float* ring;          // [D][W]
  uint64_t* ckey;       // [W] packed cell key per ring slot
  uint32_t* bin_count;  // [NB]
  uint32_t* bin_start;  // [NB + 1]
  uint32_t* cursor;     // [NB]
  uint64_t* owner;      // [NB] first cell key seen in a bin
  uint8_t* mixed;       // [NB] bin holds points of more than one cell
  uint32_t* s_slot;     // [W] cell-ordered: ring slot
  uint64_t* s_ckey;     // [W] cell-ordered: cell key
  float* s_x;           // [D][W] cell-ordered coordinates
  uint8_t* flags;       // [W] per ring slot: outlier this slide
  uint8_t* prev;        // [W] per ring slot: capped count of the last slide
  DevState* state;
  int64_t* out_ids;     // appended sorted outlier IDs
  int64_t out_cap;
  int32_t* slide_nout;  // per-slide outlier counts (run mode), may be null
  int32_t* slide_undet; // per-slide counted points (run mode), may be null
  int64_t slide_rec_cap;
};

__device__ __forceinline__ void set_err(DevState* st, int32_t code) {
  atomicCAS(&st->err, 0, code);
}

// ---------------------------------------------------------------------------
// Grid cells. Cell coordinate k_i = floor(x_i / cell) in double precision,
// for the first h = min(D, 3) dimensions. With cell = R(1+2^-12)/n and
// |x/cell| below the limits below, any pair accepted by either predicate has
// |k_i(p) - k_i(q)| <= n (the stencil), and for D <= 3, n >= 2 two points of
// one cell are always neighbours (so a cell with more than K points is
// all-inlier). Limits keep the double rounding of x/cell below 2^-16 cells.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double coord_limit(int h) {
  return h == 1 ? 68719476736.0 /* 2^36 */ : (h == 2 ? 1073741824.0 /* 2^30 */ : 1048576.0 /* 2^20 */);
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
// bins; rows of one stencil never share a bin for n <= 3.
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

// ---------------------------------------------------------------------------
// Neighbour predicates (see rtod.h). PRED 0: FP32, each subtract, multiply and
// add rounded on its own (no FMA contraction), summed left to right,
// d2 <= R2f. PRED 1: RTOD's double test (src/ods/optixScan.cu:170-190).
// ---------------------------------------------------------------------------
template <int D, int PRED>
__device__ __forceinline__ bool is_nbr(const float* q, const float* c, float R2f, double R, double R2) {
  if constexpr (PRED == 0) {
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      float dx = __fsub_rn(q[i], c[i]);
      float t = __fmul_rn(dx, dx);
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
        double dx = __dsub_rn((double)q[i], (double)c[i]);
        double t = __dmul_rn(dx, dx);
        s = (i == 0) ? t : __dadd_rn(s, t);
      }
      return s < R2;
    }
  }
}

template <int D>
struct Hashed {
  static constexpr int value = D < 3 ? D : 3;
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------------------
// k_ingest: ring update (+ per-slide resets).
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(256) k_ingest(KParams p, int64_t n_new) {
  DevState* st = p.state;
  const int64_t base = st->n_ingested;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if (tid == 0) st->n_undet = 0;
  for (int64_t i = tid; i < NB; i += stride) {
    p.bin_count[i] = 0;
    p.owner[i] = EMPTY_KEY;
    p.mixed[i] = 0;
  }
  for (int64_t i = tid; i < p.W; i += stride) p.flags[i] = 0;
  constexpr int H = Hashed<D>::value;
  const double lim = coord_limit(H);
  for (int64_t i = tid; i < n_new; i += stride) {
    const int64_t g = base + i;
    const int64_t slot = g % p.W;
    const float* s = p.src + (p.src_staging ? i : g) * D;
    float x[D];
    bool ok = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      x[d] = s[d];
      ok &= isfinite(x[d]);
    }
    int64_t k[3] = {0, 0, 0};
    bool inr = true;
#pragma unroll
    for (int d = 0; d < H; ++d) {
      double qd = floor(__ddiv_rn((double)x[d], p.cell));
      inr &= (qd > -lim) && (qd < lim);
      k[d] = inr ? (int64_t)qd : 0;
    }
    if (!ok) set_err(st, DERR_NONFINITE);
    else if (!inr) set_err(st, DERR_RANGE);
#pragma unroll
    for (int d = 0; d < D; ++d) p.ring[(int64_t)d * p.W + slot] = x[d];
    p.ckey[slot] = pack_key(k, H);
    p.prev[slot] = 254;  // no count yet
  }
}

// Window commit for the initial fill (no detection).
__global__ void k_advance(DevState* st, int64_t n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->n_ingested += n;
}

// ---------------------------------------------------------------------------
// k_hist: per-bin counts, warp-aggregated; "mixed" marks bins shared by cells.
// ---------------------------------------------------------------------------
template <int H>
__global__ void __launch_bounds__(256) k_hist(KParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w0 = warp * 32; w0 < p.W; w0 += nwarps * 32) {
    const int64_t slot = w0 + lane;
    const bool valid = slot < p.W;
    const uint64_t key = valid ? p.ckey[slot] : EMPTY_KEY;
    const uint32_t bin = valid ? bin_of_key(key, H) : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    const int leader = __ffs(peers) - 1;
    const uint64_t lkey = __shfl_sync(0xffffffffu, key, leader);
    const unsigned diff = __ballot_sync(0xffffffffu, key != lkey) & peers;
    if (valid && lane == leader) {
      atomicAdd(&p.bin_count[bin], (uint32_t)__popc(peers));
      const unsigned long long old =
          atomicCAS((unsigned long long*)&p.owner[bin], (unsigned long long)EMPTY_KEY,
                    (unsigned long long)key);
      if (diff || (old != EMPTY_KEY && old != key)) p.mixed[bin] = 1;
    }
  }
}

// ---------------------------------------------------------------------------
// k_scan: exclusive scan of NB bin counts, one block of 1024 threads.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_scan(KParams p) {
  constexpr int PER = NB / 1024;  // 64 bins per thread
  __shared__ uint32_t wsum[32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const uint4* src = reinterpret_cast<const uint4*>(p.bin_count + t * PER);
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < PER / 4; ++j) {
    uint4 v = src[j];
    sum += v.x + v.y + v.z + v.w;
  }
  uint32_t inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t v = wsum[lane], vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, vi, o);
      if (lane >= o) vi += y;
    }
    wsum[lane] = vi - v;
  }
  __syncthreads();
  uint32_t run = wsum[wid] + inc - sum;
  uint4* dst = reinterpret_cast<uint4*>(p.bin_start + t * PER);
  uint4* cur = reinterpret_cast<uint4*>(p.cursor + t * PER);
#pragma unroll
  for (int j = 0; j < PER / 4; ++j) {
    uint4 v = src[j], o;
    o.x = run; run += v.x;
    o.y = run; run += v.y;
    o.z = run; run += v.z;
    o.w = run; run += v.w;
    dst[j] = o;
    cur[j] = o;
  }
  if (t == 1023) p.bin_start[NB] = run;
}

// ---------------------------------------------------------------------------
// k_scatter: window -> cell-ordered SoA (counting sort, warp-aggregated).
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(256) k_scatter(KParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w0 = warp * 32; w0 < p.W; w0 += nwarps * 32) {
    const int64_t slot = w0 + lane;
    const bool valid = slot < p.W;
    const uint64_t key = valid ? p.ckey[slot] : EMPTY_KEY;
    const uint32_t bin = valid ? bin_of_key(key, Hashed<D>::value) : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (valid && lane == leader) base = atomicAdd(&p.cursor[bin], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (valid) {
      const uint32_t pos = base + __popc(peers & lanemask_lt());
      p.s_slot[pos] = (uint32_t)slot;
      p.s_ckey[pos] = key;
#pragma unroll
      for (int d = 0; d < D; ++d) p.s_x[(int64_t)d * p.W + pos] = p.ring[(int64_t)d * p.W + slot];
    }
  }
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
// k_count (plain): one warp per 32 cell-ordered points. Points of a bin that
// holds a single cell with more than K points are inliers without any test
// (safe-inlier skip). Every other point is counted by the whole warp:
// 32 candidates per step, tested with the predicate, tallied with
// ballot/popc, stopping as soon as the count exceeds K.
// ---------------------------------------------------------------------------
template <int D, int PRED>
__global__ void __launch_bounds__(256) k_count(KParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t pos = warp * 32 + lane;
  const bool valid = pos < p.W;
  if (warp * 32 >= p.W) return;
  constexpr int H = Hashed<D>::value;
  const uint64_t key = valid ? p.s_ckey[pos] : 0;
  const uint32_t slot = valid ? p.s_slot[pos] : 0;
  bool need = valid;
  if (valid && p.filter) {
    const uint32_t b = bin_of_key(key, H);
    const uint32_t cnt = p.bin_start[b + 1] - p.bin_start[b];
    if (cnt > (uint32_t)p.K && !p.mixed[b]) need = false;
  }
  if (valid && !need) p.prev[slot] = 255;
  float x[D];
#pragma unroll
  for (int d = 0; d < D; ++d) x[d] = valid ? p.s_x[(int64_t)d * p.W + pos] : 0.0f;
  unsigned todo = __ballot_sync(0xffffffffu, need);
  if (lane == 0 && todo) atomicAdd(&p.state->n_undet, __popc(todo));
  while (todo) {
    const int q = __ffs(todo) - 1;
    todo &= todo - 1;
    float qx[D];
#pragma unroll
    for (int d = 0; d < D; ++d) qx[d] = __shfl_sync(0xffffffffu, x[d], q);
    const uint64_t qkey = __shfl_sync(0xffffffffu, key, q);
    const uint32_t qslot = __shfl_sync(0xffffffffu, slot, q);
    int64_t k[3];
    unpack_key(qkey, H, k);
    int total = 0;
    const bool done = for_each_run<H>(p.bin_start, k, p.n, [&](uint32_t rs, uint32_t re) {
      for (uint32_t b = rs; b < re; b += 32) {
        const uint32_t c = b + lane;
        bool in = false;
        if (c < re) {
          float cx[D];
#pragma unroll
          for (int d = 0; d < D; ++d) cx[d] = p.s_x[(int64_t)d * p.W + c];
          in = is_nbr<D, PRED>(qx, cx, p.R2f, p.R, p.R2);
        }
        total += __popc(__ballot_sync(0xffffffffu, in));
        if (total > p.K) return true;
      }
      return false;
    });
    if (lane == 0) {
      if (!done) p.flags[qslot] = 1;
      p.prev[qslot] = (uint8_t)(total < 253 ? total : 253);
    }
  }
}

// ---------------------------------------------------------------------------
// k_compact: outlier flags in ring order -> sorted global indices, appended to
// out_ids; per-slide counters; window advance. One block of 1024 threads.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_compact(KParams p) {
  __shared__ uint32_t wsum[32];
  __shared__ int64_t s_base;
  __shared__ int s_fail;
  DevState* st = p.state;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int64_t lo = st->n_ingested + p.S - p.W;  // first index of the detected window
  const int64_t slot0 = lo % p.W;
  const int64_t per = (p.W + 1023) / 1024;
  const int64_t i0 = min((int64_t)t * per, p.W), i1 = min(i0 + per, p.W);
  uint32_t cnt = 0;
  for (int64_t i = i0; i < i1; ++i) {
    int64_t s = slot0 + i;
    if (s >= p.W) s -= p.W;
    cnt += p.flags[s];
  }
  uint32_t inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t v = wsum[lane], vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, vi, o);
      if (lane >= o) vi += y;
    }
    wsum[lane] = vi - v;
    if (lane == 31) {
      const int64_t total = vi;
      const int64_t base = st->out_total;
      s_base = base;
      s_fail = (base + total > p.out_cap);
      if (s_fail) set_err(st, DERR_CAPACITY);
      st->n_out = (int32_t)total;
    }
  }
  __syncthreads();
  if (!s_fail) {
    int64_t o = s_base + wsum[wid] + inc - cnt;
    for (int64_t i = i0; i < i1; ++i) {
      int64_t s = slot0 + i;
      if (s >= p.W) s -= p.W;
      if (p.flags[s]) p.out_ids[o++] = lo + i;
    }
  }
  __syncthreads();
  if (t == 0) {
    const int64_t j = st->slide;
    const int32_t nout = st->n_out;
    if (p.slide_nout && j < p.slide_rec_cap) {
      p.slide_nout[j] = nout;
      p.slide_undet[j] = st->n_undet;
    }
    if (!s_fail) st->out_total += nout;
    st->undet_total += st->n_undet;
    st->slide = j + 1;
    st->n_ingested += p.S;
  }
}

}  // namespace rtod
