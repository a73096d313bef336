// Streaming grid engine of push/detect (sm_100a): the window's cell grid is
// kept on the device from slide to slide and updated by the slide's points,
// instead of a counting sort of the whole window per slide (the window
// engine of kernels.cuh). It replaces, for one stream, RTOD's per-slide
// expire / insert bookkeeping and grid filter (prepare_c_non_points_queue and
// FixQueue, src/ods/optixScan.cpp:967-1017, src/ods/state.h:15-57), the
// BVH rebuild (:378-426) and the ray launch (:727-750, src/ods/optixScan.cu:21-75).
//
// Layout. Each bin of the cell hash (the bin map of kernels.cuh, NB bins)
// holds its window points as a FIFO of entries numbered by two monotonic
// counters head <= tail: entry e is live while head <= e < tail. Window
// points leave in the order they came in, one slide block at a time, so a
// slide's expiry is head += (points of the leaving block in the bin) and its
// insertion tail += (points of the new block in the bin): no sort, no scan.
// A bin's entries live in a region of 2 * cap pool slots (cap a power of
// two, 0 for a bin that never held points): entry e is written at slots
// e % cap and cap + e % cap (a mirrored ring), so whenever tail - head <= cap
// the live entries are the contiguous slots [head % cap, head % cap + tail
// - head) of the region. That run is what the group count (group.cuh) reads
// as the bin's candidate range. Per slot: D coordinates (rows of `pool`
// slots) and the ring slot of the point (global index % W).
//
// Per slide, four launches replayed as one graph:
//   k_grid_ingest  one thread per slide point: expiry of the point that its
//                  ring slot held (W points earlier), cell key, ring write,
//                  append to its bin. An entry that does not fit its bin's
//                  region goes to an overflow list; the block that finishes
//                  last moves every overflowed bin into a region of at least
//                  twice its occupancy (pool bump allocation), places the
//                  overflow list, and decides from the per-slide-block cell
//                  ranges whether the window's cells map to distinct bins.
//   k_grid_classify one lane per bin: all-inlier when the bin holds more than
//                  K points of one cell (cells of side R(1+2^-12)/n, n >= 2,
//                  D <= 3: a cell's diagonal is below R) or when its sure
//                  stencil cells do; all-outlier when its whole stencil holds
//                  at most K points; otherwise its points are listed as count
//                  parts of up to GRID_PART consecutive entries.
//   k_grid_count   one warp per part: the group count of group.cuh over the
//                  runs of the bin's stencil bins (candidates shared by the
//                  part's points), early exit past K; outliers set their
//                  window-offset bit.
//   k_compact_one  bitset -> sorted global IDs in the mapped landing buffers,
//                  end of the detection (kernels.cuh).
// Abandoned regions are not reused; when the pool runs out the detection
// reports DERR_GRID and the host rebuilds the grid from the ring (regions
// sized to the current occupancy, compacted) and counts the window again.
//
// A bin's `mixed` counter is the number of its live entries whose cell key
// differs from the bin's reference key `ref` (set by the first entry into an
// empty bin, cleared by the count once the bin is empty): mixed == 0 means the
// bin holds one cell, which the all-inlier rule needs when the window as a
// whole is not known to be alias-free.
#pragma once

#include "kernels.cuh"  // includes group.cuh

namespace rtod {

constexpr uint32_t GRID_MIN_CAP = 64;     // smallest capacity of a grown region (entries)
constexpr uint32_t GRID_FRESH_CAP = 16;   // capacity of an empty bin's region at a build
constexpr int GRID_INGEST_THREADS = 256;
constexpr int GRID_COUNT_THREADS = 256;   // 8 warps, one tile of 32 bins each
constexpr uint32_t GRID_PART = 64;        // points of a bin per listed count part (one warp each)
constexpr int GRID_SLOT_BATCH = 8;        // stencil bins whose occupancy loads are in flight together
constexpr int GRID_COPY_UNROLL = 4;       // entries per lane in flight when a region moves

// Grid control block (device).
struct GridCtl {
  uint32_t done;       // finished blocks of the running ingest or insert launch
  uint32_t n_grow;     // bins listed to grow
  uint32_t n_ovf;      // entries listed as overflow
  int32_t pure;        // the window's cells (with the 1-d rule's margin) map to distinct bins
  unsigned long long pool_top;  // pool slots handed out
  int32_t fail;        // the pool ran out: the grid must be rebuilt
  uint32_t max_occ;    // largest bin occupancy of the last counted window
  uint32_t n_queue;    // count parts listed by k_grid_classify (up to GRID_PART points of a bin each)
  long long cmin[3];   // the window's cell-coordinate box (grid_purity)
  long long cmax[3];
};

// Kernel argument: the grid of one stream.
struct Grid {
  GridCtl* ctl;
  uint32_t* head;            // [NB]
  uint32_t* tail;            // [NB]
  uint32_t* base;            // [NB] first pool slot of the bin's region
  uint32_t* cap;             // [NB] region capacity (power of two, or 0)
  unsigned long long* ref;   // [NB] reference cell key (EMPTY_KEY: none)
  uint32_t* mixed;           // [NB] live entries of another cell than ref
  uint32_t* growflag;        // [NB] listed to grow in the running launch
  void* px;                  // [D][pool] coordinates (the handle's type)
  uint32_t* pslot;           // [pool] ring slot of the entry's point
  uint32_t pool;             // slots of the pool (row stride of px)
  uint32_t ovf_cap;          // room of the overflow and grow lists (S)
  uint32_t* grow;            // [ovf_cap] bins to grow
  uint32_t* grow_to;         // [2 ovf_cap] their new regions: first pool slot, capacity
  uint32_t* ovf_bin;         // [ovf_cap]
  uint32_t* ovf_pos;         // [ovf_cap] entry number
  uint32_t* ovf_slot;        // [ovf_cap] ring slot
  void* ovf_x;               // [D][ovf_cap] coordinates
  uint32_t* qpos;            // [W] count parts: pool slot of the part's first point
  uint32_t* qbin;            // [W] and its bin | points << 16
  long long* brange;         // [nslots][6] per slide block (block t at t % nslots):
                             // smallest then largest cell coordinate per hashed dimension
  int32_t nslots;            // W / S + 1
};

__device__ __forceinline__ uint32_t pow2_at_least(uint32_t v) {
  return v <= 1u ? 1u : 1u << (32 - __clz(v - 1u));
}

template <typename T>
__device__ __forceinline__ T* grid_row(const Grid& g, int d) {
  return static_cast<T*>(g.px) + (size_t)d * g.pool;
}

// Block slot of slide block t.
__device__ __forceinline__ int grid_bslot(const Grid& g, int64_t t) { return (int)(t % g.nslots); }

// Cell-coordinate range of one slide block: per warp reduction, one atomic
// per dimension and warp.
template <int H>
__device__ __forceinline__ void grid_block_range(const Grid& g, int bslot, bool valid, uint64_t key) {
  const int lane = threadIdx.x & 31;
  int64_t k[3] = {0, 0, 0};
  if (valid) unpack_key(key, H, k);
  const bool any = __ballot_sync(0xffffffffu, valid) != 0;
  if (!any) return;
#pragma unroll
  for (int d = 0; d < H; ++d) {
    long long mn = valid ? k[d] : LLONG_MAX, mx = valid ? k[d] : LLONG_MIN;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
      atomicMin(&g.brange[bslot * 6 + d], mn);
      atomicMax(&g.brange[bslot * 6 + 3 + d], mx);
    }
  }
}

// Appends one point per valid lane to its bin (whole warp). Lanes of one
// bin are aggregated: one reference-key check and one tail increment per bin.
template <int D, typename T>
__device__ __forceinline__ void grid_append(const Grid& g, bool valid, uint64_t key, const T* x, uint32_t slot) {
  constexpr int H = Hashed<D>::value;
  const int lane = threadIdx.x & 31;
  const uint32_t bin = valid ? bin_of_key(key, H) : 0xffffffffu;
  const unsigned peers = __match_any_sync(0xffffffffu, bin);
  const int leader = __ffs(peers) - 1;
  unsigned long long r = 0;
  uint32_t pos0 = 0;
  if (valid && lane == leader) {
    r = *(volatile unsigned long long*)&g.ref[bin];
    if (r == EMPTY_KEY) {
      const unsigned long long prev = atomicCAS(&g.ref[bin], EMPTY_KEY, (unsigned long long)key);
      r = prev == EMPTY_KEY ? (unsigned long long)key : prev;
    }
    pos0 = atomicAdd(&g.tail[bin], (uint32_t)__popc(peers));
  }
  r = __shfl_sync(0xffffffffu, r, leader);
  const uint32_t pos = __shfl_sync(0xffffffffu, pos0, leader) + (uint32_t)__popc(peers & lanemask_lt());
  if (!valid) return;
  if ((unsigned long long)key != r) atomicAdd(&g.mixed[bin], 1u);
  // head only grows, so this read is a lower bound of the final head: an
  // entry written here never lands on a live entry's slots.
  const uint32_t h = *(volatile uint32_t*)&g.head[bin];
  const uint32_t c = g.cap[bin];
  if (pos - h < c) {
    const uint32_t s0 = g.base[bin] + (pos & (c - 1u));
#pragma unroll
    for (int d = 0; d < D; ++d) {
      T* row = grid_row<T>(g, d);
      row[s0] = x[d];
      row[s0 + c] = x[d];
    }
    g.pslot[s0] = slot;
    g.pslot[s0 + c] = slot;
  } else {
    const uint32_t o = atomicAdd(&g.ctl->n_ovf, 1u);
    if (o < g.ovf_cap) {
      g.ovf_bin[o] = bin;
      g.ovf_pos[o] = pos;
      g.ovf_slot[o] = slot;
#pragma unroll
      for (int d = 0; d < D; ++d) static_cast<T*>(g.ovf_x)[(size_t)d * g.ovf_cap + o] = x[d];
    }
    if (atomicExch(&g.growflag[bin], 1u) == 0u) {
      const uint32_t gi = atomicAdd(&g.ctl->n_grow, 1u);
      if (gi < g.ovf_cap) g.grow[gi] = bin;
    }
  }
}

// Expires one point per valid lane (its cell key) from its bin (whole warp).
template <int H>
__device__ __forceinline__ void grid_expire(const Grid& g, bool valid, uint64_t key) {
  const int lane = threadIdx.x & 31;
  const uint32_t bin = valid ? bin_of_key(key, H) : 0xffffffffu;
  const unsigned peers = __match_any_sync(0xffffffffu, bin);
  if (!valid) return;
  if (lane == __ffs(peers) - 1) atomicAdd(&g.head[bin], (uint32_t)__popc(peers));
  // ref is fixed while the bin holds entries (this one included)
  if ((unsigned long long)key != g.ref[bin]) atomicSub(&g.mixed[bin], 1u);
}

// Run by the last block of an ingest or insert launch (all threads), after
// every other block's appends: grows the listed bins and places the overflow
// entries. Phases separated by block barriers, each a few dependent memory
// round trips: new regions (a thread per bin), live entries moved (a warp
// per bin, GRID_COPY_UNROLL entries per lane in flight), the bins' region
// fields updated, overflow entries placed (4 per thread in flight). On pool
// exhaustion nothing moves and the grid is marked failed (DERR_GRID).
template <int D, typename T>
__device__ void grid_fixup(const Grid& g, BatchState* bs) {
  GridCtl* ctl = g.ctl;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  const uint32_t n_grow = min(*(volatile uint32_t*)&ctl->n_grow, g.ovf_cap);
  const uint32_t n_ovf = min(*(volatile uint32_t*)&ctl->n_ovf, g.ovf_cap);
  if (n_grow == 0) return;
  __shared__ int s_fail;
  if (threadIdx.x == 0) s_fail = 0;
  __syncthreads();
  for (uint32_t gi = threadIdx.x; gi < n_grow; gi += blockDim.x) {
    const uint32_t bin = g.grow[gi];
    const uint32_t occ = g.tail[bin] - g.head[bin];
    const uint32_t nc = pow2_at_least(max(2u * occ, GRID_MIN_CAP));
    const unsigned long long nb = atomicAdd(&ctl->pool_top, 2ull * nc);
    if (nb + 2ull * nc > (unsigned long long)g.pool) s_fail = 1;
    g.grow_to[2 * gi] = (uint32_t)nb;
    g.grow_to[2 * gi + 1] = nc;
  }
  __syncthreads();
  if (s_fail) {
    if (threadIdx.x == 0) {
      ctl->fail = 1;
      set_err(bs, DERR_GRID);
    }
    return;
  }
  // live entries from the old regions (an overflowed entry reads a stale
  // slot here and is rewritten from the overflow list below)
  for (uint32_t gi = (uint32_t)wid; gi < n_grow; gi += (uint32_t)nw) {
    const uint32_t bin = g.grow[gi];
    const uint32_t oc = g.cap[bin];
    if (!oc) continue;
    const uint32_t nb = g.grow_to[2 * gi], nc = g.grow_to[2 * gi + 1];
    const uint32_t ob = g.base[bin], h = g.head[bin], occ = g.tail[bin] - h;
    for (uint32_t e0 = 0; e0 < occ; e0 += 32u * GRID_COPY_UNROLL) {
      T v[GRID_COPY_UNROLL][D];
      uint32_t sl[GRID_COPY_UNROLL];
#pragma unroll
      for (int u = 0; u < GRID_COPY_UNROLL; ++u) {
        const uint32_t k = e0 + 32u * u + (uint32_t)lane;
        const uint32_t src = ob + ((h + k) & (oc - 1u));
#pragma unroll
        for (int d = 0; d < D; ++d) v[u][d] = k < occ ? grid_row<T>(g, d)[src] : T(0);
        sl[u] = k < occ ? g.pslot[src] : 0u;
      }
#pragma unroll
      for (int u = 0; u < GRID_COPY_UNROLL; ++u) {
        const uint32_t k = e0 + 32u * u + (uint32_t)lane;
        if (k >= occ) continue;
        const uint32_t dst = nb + ((h + k) & (nc - 1u));
#pragma unroll
        for (int d = 0; d < D; ++d) {
          T* row = grid_row<T>(g, d);
          row[dst] = v[u][d];
          row[dst + nc] = v[u][d];
        }
        g.pslot[dst] = sl[u];
        g.pslot[dst + nc] = sl[u];
      }
    }
  }
  __syncthreads();
  for (uint32_t gi = threadIdx.x; gi < n_grow; gi += blockDim.x) {
    const uint32_t bin = g.grow[gi];
    g.base[bin] = g.grow_to[2 * gi];
    g.cap[bin] = g.grow_to[2 * gi + 1];
    g.growflag[bin] = 0;
  }
  __syncthreads();
  for (uint32_t o0 = 0; o0 < n_ovf; o0 += 4u * blockDim.x) {
    uint32_t bin[4], pos[4], sl[4], c[4], base[4];
    T v[4][D];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t o = o0 + (uint32_t)u * blockDim.x + threadIdx.x;
      const bool ok = o < n_ovf;
      bin[u] = ok ? g.ovf_bin[o] : 0u;
      pos[u] = ok ? g.ovf_pos[o] : 0u;
      sl[u] = ok ? g.ovf_slot[o] : 0u;
#pragma unroll
      for (int d = 0; d < D; ++d) v[u][d] = ok ? static_cast<const T*>(g.ovf_x)[(size_t)d * g.ovf_cap + o] : T(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool ok = o0 + (uint32_t)u * blockDim.x + threadIdx.x < n_ovf;
      c[u] = ok ? g.cap[bin[u]] : 0u;
      base[u] = ok ? g.base[bin[u]] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (o0 + (uint32_t)u * blockDim.x + threadIdx.x >= n_ovf) continue;
      const uint32_t s0 = base[u] + (pos[u] & (c[u] - 1u));
#pragma unroll
      for (int d = 0; d < D; ++d) {
        T* row = grid_row<T>(g, d);
        row[s0] = v[u][d];
        row[s0 + c[u]] = v[u][d];
      }
      g.pslot[s0] = sl[u];
      g.pslot[s0 + c[u]] = sl[u];
    }
  }
  if (threadIdx.x == 0) {
    ctl->n_grow = 0;
    ctl->n_ovf = 0;
  }
}

// Purity of the window whose newest slide block is t (blocks t - m + 1 .. t,
// m = nslots - 1): whether its cells, widened by the 1-d rule's margin of
// n - 2 cells, map to distinct bins (box_pure). One warp.
template <int H>
__device__ __forceinline__ void grid_purity(const Grid& g, int64_t t, int n) {
  const int lane = threadIdx.x & 31;
  const int m = g.nslots - 1;
  long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  for (int i = lane; i < m; i += 32) {
    const int bs = grid_bslot(g, t - i);
#pragma unroll
    for (int d = 0; d < H; ++d) {
      mn[d] = min(mn[d], g.brange[bs * 6 + d]);
      mx[d] = max(mx[d], g.brange[bs * 6 + 3 + d]);
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
  const bool pure = box_pure<H>(mn, mx, 2 * max(n - 2, 0));
  if (lane == 0) {
    g.ctl->pure = pure ? 1 : 0;
    for (int d = 0; d < 3; ++d) {
      g.ctl->cmin[d] = d < H ? mn[d] : 0;
      g.ctl->cmax[d] = d < H ? mx[d] : 0;
    }
  }
}

// Whether this block finished last among the launch's blocks (every thread
// gets the answer; the counter is rearmed by the last block).
__device__ __forceinline__ bool grid_last_block(GridCtl* ctl) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&ctl->done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (s_last) __threadfence();
  return s_last != 0;
}

// ---------------------------------------------------------------------------
// k_grid_ingest: one slide of the stream's only job. The window being
// detected is [lo, lo + W); its newest block t holds global indices
// [lo + W - S, lo + W), staged point-major in jb.stage; ring slot s of a new
// point held the point W positions earlier, which leaves the window now.
// ---------------------------------------------------------------------------
template <int D, typename T>
__global__ void __launch_bounds__(GRID_INGEST_THREADS) k_grid_ingest(Batch b, Grid g, int32_t reset_out) {
  pdl_trigger();
  pdl_wait();
  constexpr int H = Hashed<D>::value;
  const Job& jb = b.jobs[0];
  const int64_t lo = jb.ctr->lo;
  const int64_t g0 = lo + jb.W - jb.S;
  const int64_t t = g0 / jb.S;
  const int bslot = grid_bslot(g, t);
  if (blockIdx.x == 0 && threadIdx.x < 6) {  // the leaving block's range slot, reused by block t + 1
    const int rs = grid_bslot(g, t + 1);
    g.brange[rs * 6 + threadIdx.x] = threadIdx.x < 3 ? LLONG_MAX : LLONG_MIN;
  }
  if (reset_out && blockIdx.x == 0 && threadIdx.x == 0) b.bs->out_total = 0;
  T* ring = static_cast<T*>(const_cast<void*>(jb.pts));
  uint64_t* keys = const_cast<uint64_t*>(jb.keys);
  const T* stage = static_cast<const T*>(jb.stage);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < jb.S; i0 += stride) {
    const int64_t i = i0 + threadIdx.x;
    const bool valid = i < jb.S;
    const int64_t s = valid ? (g0 + i) % jb.W : 0;
    grid_expire<H>(g, valid, valid ? keys[s] : 0ull);
    T x[D];
    uint64_t key = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = valid ? stage[i * D + d] : T(0);
    if (valid) {
      int32_t code;
      key = cell_key<D, T>(x, jb.inv_cell, &code);
      if (code) set_err(b.bs, code);
#pragma unroll
      for (int d = 0; d < D; ++d) ring[(int64_t)d * jb.W + s] = x[d];
      keys[s] = key;
      jb.prev[s] = 254;
    }
    grid_append<D, T>(g, valid, key, x, (uint32_t)s);
    grid_block_range<H>(g, bslot, valid, key);
  }
  if (!grid_last_block(g.ctl)) return;
  grid_fixup<D, T>(g, b.bs);
  if (threadIdx.x < 32) grid_purity<H>(g, t, jb.n);
  if (threadIdx.x == 0) g.ctl->done = 0;
}

// ---------------------------------------------------------------------------
// Grid build from the ring (first window of a stream, and rebuilds):
// occupancy per bin, one region per occupied bin, then the window's slide
// blocks appended oldest first (one launch each, so that a bin's entries
// keep block order).
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(256) k_grid_occ(Batch b, Grid g, int64_t lo) {
  pdl_trigger();
  pdl_wait();
  constexpr int H = Hashed<D>::value;
  const Job& jb = b.jobs[0];
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < jb.W; i0 += stride) {
    const int64_t i = i0 + threadIdx.x;
    const bool valid = i < jb.W;
    const uint32_t bin = valid ? bin_of_key(jb.keys[(lo + i) % jb.W], H) : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(&g.tail[bin], (uint32_t)__popc(peers));
  }
}

// One region per bin: twice the occupancy (the counts that k_grid_occ left
// in tail, which restarts at zero) for an occupied bin, GRID_FRESH_CAP
// entries for an empty one, so that a cell the stream enters later rarely
// needs the ingest's growth step.
static __global__ void __launch_bounds__(256) k_grid_alloc(Grid g, BatchState* bs) {
  pdl_trigger();
  pdl_wait();
  for (uint32_t bin = blockIdx.x * blockDim.x + threadIdx.x; bin < NB; bin += gridDim.x * blockDim.x) {
    const uint32_t occ = g.tail[bin];
    g.tail[bin] = 0;
    const uint32_t nc = occ ? pow2_at_least(max(2u * occ, GRID_MIN_CAP)) : GRID_FRESH_CAP;
    const unsigned long long nb = atomicAdd(&g.ctl->pool_top, 2ull * nc);
    if (nb + 2ull * nc > (unsigned long long)g.pool) {
      g.ctl->fail = 1;
      set_err(bs, DERR_GRID);
      continue;
    }
    g.base[bin] = (uint32_t)nb;
    g.cap[bin] = nc;
  }
}

// Appends the ring's slide block t (global indices [tS, tS + S)).
template <int D, typename T>
__global__ void __launch_bounds__(GRID_INGEST_THREADS) k_grid_insert(Batch b, Grid g, int64_t t) {
  pdl_trigger();
  pdl_wait();
  constexpr int H = Hashed<D>::value;
  const Job& jb = b.jobs[0];
  if (g.ctl->fail) return;
  const T* ring = static_cast<const T*>(jb.pts);
  const int bslot = grid_bslot(g, t);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < jb.S; i0 += stride) {
    const int64_t i = i0 + threadIdx.x;
    const bool valid = i < jb.S;
    const int64_t s = valid ? (t * jb.S + i) % jb.W : 0;
    T x[D];
    uint64_t key = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = valid ? ring[(int64_t)d * jb.W + s] : T(0);
    if (valid) key = jb.keys[s];
    grid_append<D, T>(g, valid, key, x, (uint32_t)s);
    grid_block_range<H>(g, bslot, valid, key);
  }
  if (!grid_last_block(g.ctl)) return;
  grid_fixup<D, T>(g, b.bs);
  if (threadIdx.x == 0) g.ctl->done = 0;
}

// Purity of the window whose newest block is t, after a build.
template <int D>
__global__ void __launch_bounds__(32) k_grid_purity(Batch b, Grid g, int64_t t) {
  pdl_trigger();
  pdl_wait();
  grid_purity<Hashed<D>::value>(g, t, b.jobs[0].n);
}

// Starting state: empty bins without regions, pool empty, block ranges empty.
static __global__ void __launch_bounds__(256) k_grid_reset(Grid g) {
  pdl_trigger();
  pdl_wait();
  for (uint32_t bin = blockIdx.x * blockDim.x + threadIdx.x; bin < NB; bin += gridDim.x * blockDim.x) {
    g.head[bin] = 0;
    g.tail[bin] = 0;
    g.base[bin] = 0;
    g.cap[bin] = 0;
    g.ref[bin] = EMPTY_KEY;
    g.mixed[bin] = 0;
    g.growflag[bin] = 0;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.nslots * 6; i += gridDim.x * blockDim.x)
    g.brange[i] = (i % 6) < 3 ? LLONG_MAX : LLONG_MIN;
  if (blockIdx.x == 0 && threadIdx.x == 0) *g.ctl = GridCtl{};
}

// ---------------------------------------------------------------------------
// k_grid_classify: one lane per bin (tiles of 32 bins per warp). A bin is
// decided without tests when it holds more than K points of one cell
// (all-inlier), or, for short stencils, when its sure stencil cells hold more
// than K points (all-inlier) or its whole stencil holds at most K points
// (all-outlier: marked here); the points of every other bin are listed for an
// exact count. Empty bins drop their reference key.
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(GRID_COUNT_THREADS) k_grid_classify(Batch b, Grid g) {
  pdl_trigger();
  pdl_wait();
  constexpr int H = Hashed<D>::value;
  if (*(volatile int32_t*)&g.ctl->fail) return;
  const Job& jb = b.jobs[0];
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t lo_mod = (uint32_t)(jb.ctr->lo % jb.W), Wu = (uint32_t)jb.W;
  const bool pure = g.ctl->pure != 0;
  const bool can_sure = jb.filter && pure && D <= 3;
  const int w = 2 * jb.n + 1;
  const int slots = H == 1 ? w : (H == 2 ? w * w : w * w * w);
  // Short stencils (1-d, 2-d with one cell per R) are summed here, a lane per
  // bin, to decide whole bins without a count; longer ones are left to the
  // count's warp-wide pass over the stencil, which decides the same bins.
  const bool sums = slots <= 2 * GRID_SLOT_BATCH;
  // An alias-free window's points all lie in its cell box: only the box's
  // bins are visited (in rows along the last hashed dimension, whose bins are
  // consecutive); otherwise every bin.
  uint32_t ext[3] = {1, 1, 1};
  uint64_t vol = NB;
  if (pure) {
    vol = 1;
#pragma unroll
    for (int d = 0; d < H; ++d) {
      ext[d] = (uint32_t)(g.ctl->cmax[d] - g.ctl->cmin[d] + 1);
      vol *= ext[d];
    }
  }
  const uint32_t row = pure ? ext[H - 1] : 32u;
  const uint32_t row_tiles = (row + 31) / 32;
  const uint32_t ntiles = (uint32_t)(vol / row) * row_tiles;
  int nout = 0;
  uint32_t occmax = 0, queued = 0;
  for (uint32_t tile = warp; tile < ntiles; tile += nwarps) {
    uint32_t bin;
    bool in = true;
    if (pure) {
      const uint32_t r = tile / row_tiles, x = (tile % row_tiles) * 32 + (uint32_t)lane;
      in = x < row;
      int64_t k[3] = {g.ctl->cmin[0], g.ctl->cmin[1], g.ctl->cmin[2]};
      if constexpr (H == 1) {
        k[0] += x;
      } else if constexpr (H == 2) {
        k[0] += r;
        k[1] += x;
      } else {
        k[0] += r / ext[1];
        k[1] += r % ext[1];
        k[2] += x;
      }
      bin = bin_of(k, H);
    } else {
      bin = tile * 32 + (uint32_t)lane;
    }
    const uint32_t h = in ? g.head[bin] : 0u, c = in ? g.tail[bin] - h : 0u;
    occmax = max(occmax, c);
    bool queue = false;
    if (c == 0) {
      if (in && g.ref[bin] != EMPTY_KEY) {  // empty: the next entry sets a new reference
        g.ref[bin] = EMPTY_KEY;
        g.mixed[bin] = 0;
      }
    } else if (!(jb.filter && c > (uint32_t)jb.K && (pure || g.mixed[bin] == 0)) && !sums) {
      queue = true;  // the group count takes the stencil sums, 32 bins per round
    } else if (!(jb.filter && c > (uint32_t)jb.K && (pure || g.mixed[bin] == 0))) {
      // stencil occupancy, GRID_SLOT_BATCH bins' loads in flight at a time
      uint32_t given = 0, total = 0;
      for (int s0 = 0; s0 < slots; s0 += GRID_SLOT_BATCH) {
        uint32_t hh[GRID_SLOT_BATCH], tt[GRID_SLOT_BATCH];
        bool su[GRID_SLOT_BATCH];
#pragma unroll
        for (int e = 0; e < GRID_SLOT_BATCH; ++e) {
          hh[e] = 0;
          tt[e] = 0;
          su[e] = false;
          if (s0 + e < slots) {
            int d[3] = {0, 0, 0};
            const uint32_t sb = (bin + (uint32_t)slot_cell<H>(s0 + e, jb.n, d)) & NB_MASK;
            su[e] = can_sure && slot_sure<H>(d, jb.n);
            hh[e] = g.head[sb];
            tt[e] = g.tail[sb];
          }
        }
#pragma unroll
        for (int e = 0; e < GRID_SLOT_BATCH; ++e) {
          const uint32_t len = tt[e] - hh[e];
          given += su[e] ? len : 0u;
          total += len;
        }
      }
      if (given > (uint32_t)jb.K) {
        // all inliers
      } else if (total <= (uint32_t)jb.K) {  // all outliers
        const uint32_t own = g.base[bin] + (h & (g.cap[bin] - 1u));
        for (uint32_t i = 0; i < c; ++i) {
          const uint32_t sl = g.pslot[own + i];
          const uint32_t off = sl >= lo_mod ? sl - lo_mod : sl + Wu - lo_mod;
          atomicOr(&jb.flags[off >> 5], 1u << (off & 31));
        }
        nout += (int)c;
      } else {
        queue = true;
      }
    }
    // the bin's points as count parts of up to GRID_PART points; one queue
    // reservation per warp
    const uint32_t np = queue ? (c + GRID_PART - 1u) / GRID_PART : 0u;
    uint32_t inc = np;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    const uint32_t wtot = __shfl_sync(0xffffffffu, inc, 31);
    if (wtot) {
      uint32_t q0 = 0;
      if (lane == 31) q0 = atomicAdd(&g.ctl->n_queue, wtot);
      q0 = __shfl_sync(0xffffffffu, q0, 31) + inc - np;
      if (queue) {
        const uint32_t own = g.base[bin] + (h & (g.cap[bin] - 1u));
        for (uint32_t k = 0; k < np; ++k) {
          g.qpos[q0 + k] = own + k * GRID_PART;
          g.qbin[q0 + k] = bin | (min(GRID_PART, c - k * GRID_PART) << 16);
        }
        queued += c;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    occmax = max(occmax, __shfl_xor_sync(0xffffffffu, occmax, o));
    nout += __shfl_xor_sync(0xffffffffu, nout, o);
    queued += __shfl_xor_sync(0xffffffffu, queued, o);
  }
  if (lane == 0) {
    if (nout) atomicAdd(&jb.ctr->n_out, nout);
    if (occmax) atomicMax(&g.ctl->max_occ, occmax);
  }
  if (lane == 0 && queued) atomicAdd(&jb.ctr->n_undet, (int)queued);
}

// ---------------------------------------------------------------------------
// k_grid_count: exact counts of the listed parts, one warp per part (warps
// striding over the list). A part's points are consecutive entries of one
// bin, so they share the bin's stencil: count_group (group.cuh) reads its
// candidates (the live runs of the stencil bins, one virtual list) 32 x CPL
// at a time into registers and tests every undecided point of the part
// against them, early exit past K. The last block to finish rearms the list
// for the next slide.
// ---------------------------------------------------------------------------
template <int D, int PRED, typename T>
__global__ void __launch_bounds__(GRID_COUNT_THREADS) k_grid_count(Batch b, Grid g) {
  pdl_trigger();
  pdl_wait();
  if (*(volatile int32_t*)&g.ctl->fail) return;
  const Job& jb = b.jobs[0];
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t lo_mod = (uint32_t)(jb.ctr->lo % jb.W), Wu = (uint32_t)jb.W;
  const bool can_sure = jb.filter && g.ctl->pure != 0 && D <= 3;
  const uint32_t nq = *(volatile uint32_t*)&g.ctl->n_queue;
  const T* px = static_cast<const T*>(g.px);
  int nout = 0;
  for (uint32_t q = warp; q < nq; q += nwarps) {
    const uint32_t p = g.qpos[q], pb = g.qbin[q];
    const GroupArgs ga{p, pb >> 16, pb & 0xffffu, jb.n, jb.K, jb.R2f, jb.R, jb.R2, (int64_t)g.pool, can_sure, nullptr};
    nout += count_group<D, PRED, T>(
        px, ga,
        [&](uint32_t sb, uint32_t& rs, uint32_t& len) {
          const uint32_t sh = g.head[sb];
          len = g.tail[sb] - sh;
          rs = len ? g.base[sb] + (sh & (g.cap[sb] - 1u)) : 0u;
        },
        [&](uint32_t pos) {
          const uint32_t sl = g.pslot[pos];
          const uint32_t o = sl >= lo_mod ? sl - lo_mod : sl + Wu - lo_mod;
          atomicOr(&jb.flags[o >> 5], 1u << (o & 31));
        });
  }
  if (lane == 0 && nout) atomicAdd(&jb.ctr->n_out, nout);
  if (grid_last_block(g.ctl)) {
    if (threadIdx.x == 0) {
      g.ctl->n_queue = 0;
      g.ctl->done = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Host side (grid.cu): launches of the engine's kernels for one stream.
// ---------------------------------------------------------------------------
struct GridKind {
  int D;
  int pred;
  int f64;
};

cudaError_t grid_launch_ingest(const GridKind& k, const Batch& b, const Grid& g, int64_t S, int sm_count,
                               cudaStream_t st);
// k_grid_classify then k_grid_count.
cudaError_t grid_launch_count(const GridKind& k, const Batch& b, const Grid& g, int sm_count, cudaStream_t st);
// Builds the grid of window [lo, lo + W) from the ring (reset, occupancy,
// regions, W / S block appends, purity): W / S + 4 launches.
cudaError_t grid_launch_build(const GridKind& k, const Batch& b, const Grid& g, int64_t lo, int64_t W, int64_t S,
                              int sm_count, cudaStream_t st);

}  // namespace rtod
