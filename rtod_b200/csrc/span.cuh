// Span engine: one counting sort per batch of B consecutive windows instead
// of one per window.
//
// The B windows of a batch, [lo0 + jS, lo0 + jS + W) for j < B, cover the
// span [lo0, lo0 + W + (B-1)S): nblk = W/S + B - 1 slide blocks of S points,
// and every window is a union of W/S whole blocks. The span is sorted once by
// bin, and inside each bin by block (points of one block in any order):
//
//   position of a point of block t in bin b
//     = bin_start[b] + pre[b][t] + (its claim among the block's points in b),
//   pre[b][t] = points of bin b in blocks before t (a bin's row of blocks is
//   contiguous, stride ts).
//
// So window j's points of bin b are the contiguous positions
// [bin_start[b] + pre[b][j], bin_start[b] + pre[b][j + W/S]), and its count
// of bin b is pre[b][j + W/S] - pre[b][j]: classification needs no per-point
// work, and a queued point's candidates are (2n+1)^h such ranges (h = hashed
// dimensions, min(D, 3)); all points of a bin share them.
//
// Kernels per batch: k_span_hist (per-block bin counts), k_span_scan
// (bin_start, list of bins in use), k_span_prefix (pre), k_span_scatter (sorted
// span), k_span_classify (per window and bin in use: safe, or listed) and
// k_span_count (exact counts of the listed bins' window points into
// per-slide outlier bitsets; its last block ends the batch). Once per chunk
// of slides, k_span_compact turns the bitsets into sorted outlier IDs.
//
// The safe-inlier rule is the window engine's (count > K in one cell, plus
// the 1-d group rule) and, for 2-3 hashed dimensions in a pure span, the
// cells within R of every point of a cell; "single cell" is judged over the
// whole span: a bin whose span holds two cells queues its points even in a
// window where it holds one. That only queues more points; every result is
// an exact count.
#pragma once

#include "kernels.cuh"

namespace rtod {

constexpr int64_t SPAN_MAX_BLOCKS = 2047;  // slide blocks of one span (tables of (blocks + 1) x NB)

struct Span {
  int64_t S;       // slide = block size
  int64_t Wp;      // row stride of s_x (multiple of 4, >= span points + 4)
  int64_t nblk;    // blocks in the span: W/S + B - 1
  int32_t wblk;    // blocks per window: W/S
  int32_t K, n, filter;
  int32_t h;       // hashed dimensions (1..3)
  int32_t n_sure;  // stencil cells within R of every point of the centre cell (pure spans, D <= 3)
  int32_t sure_delta[16];  // their bin offsets
  double R, R2;
  float R2f;
  const void* pts;          // resident stream, point-major [N][D] (the handle's coordinate type)
  uint64_t* keys;           // cell keys of the stream, by global index (written by k_span_hist)
  double inv_cell;          // 1 / cell side
  uint32_t* bin_count;          // [NB] span points per bin
  uint32_t* bin_start;          // [NB + 1]
  unsigned long long* kmin;     // [NB] smallest / largest cell key of a bin over the span
  unsigned long long* kmax;
  uint32_t* cnt;    // [NB][ts] points of bin b in block t (claims count them back to zero)
  uint32_t* pre;    // [NB][ts] points of bin b in the blocks before t, t <= nblk (bins in use only)
  int64_t ts;       // row stride of cnt and pre (>= nblk + 1): a bin's blocks are contiguous
  uint32_t* used;   // [NB] bins holding span points, n_used of them, in no particular order
  uint32_t* s_off;  // [span] bin-ordered: offset from the span start
  void* s_x;        // [D][Wp] bin-ordered coordinates (the handle's coordinate type)
  unsigned long long* scan_status;  // [SPAN_SCAN_TILES]
  SpanCtr* sc;
  uint4* groups;    // [B * min(W, NB)] listed groups: first position, points, bin, window
  uint32_t* bits;   // [chunk][words] outlier bits per window offset, row = slide % chunk
  int64_t words;    // ceil(W / 32)
  int64_t chunk;    // slides per bitset chunk (a multiple of the batch)
  int32_t route;    // learned router on: groups routed to delta segments or independent counts
  uint32_t gcap;    // entries of `groups`: groups from the front, delta segments from the back
};

// First global index of the span: the window of the batch's first job.
__device__ __forceinline__ int64_t span_lo(const Batch& b) { return b.jobs[0].ctr->lo; }

// Window j's per-bin counts from the prefix table: bin b's points in blocks
// before block t are pre[b * ts + t], and window j covers blocks [j, j + wblk).
struct WinPre {
  const uint32_t* pre;
  int64_t ts;
  int32_t j, wblk;
  __device__ __forceinline__ uint32_t count(uint32_t b) const {
    const uint32_t* row = pre + (int64_t)b * ts + j;
    return row[wblk] - row[0];
  }
};

// ---------------------------------------------------------------------------
// k_span_hist: the cell key of every span point (from its coordinates,
// stored for k_span_scatter), the span's cell-coordinate range (its purity
// is decided by k_span_scan), points per (block, bin) and per bin, and the
// per-bin key range (a bin holds one cell iff min == max). Aggregated per
// warp, then per block in a shared-memory table keyed by bin * ts + block,
// then one atomic per entry.
// ---------------------------------------------------------------------------
template <int D, typename T>
__global__ void __launch_bounds__(256) k_span_hist(Batch b, Span sp) {
  constexpr int H = Hashed<D>::value;
  __shared__ uint32_t hkey[HIST_SLOTS];
  __shared__ uint32_t hcnt[HIST_SLOTS];
  __shared__ unsigned long long hmin[HIST_SLOTS], hmax[HIST_SLOTS];
  __shared__ long long s_cr[2][3][8];  // per warp: the cell-coordinate range
  pdl_trigger();
  pdl_wait();
  constexpr int U = 2;  // points per thread and step (measured: 2 beats 1 and 4)
  const int64_t lo0 = span_lo(b);
  const int64_t npts = sp.nblk * sp.S;
  const int lane = threadIdx.x & 31;
  const T* pts = static_cast<const T*>(sp.pts);
  long long cmn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, cmx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
    hkey[t] = 0xffffffffu;
    hcnt[t] = 0;
    hmin[t] = EMPTY_KEY;
    hmax[t] = 0;
  }
  __syncthreads();
  const uint32_t S32 = (uint32_t)sp.S;
  const int64_t chunk = (int64_t)blockDim.x * U;
  for (int64_t c0 = (int64_t)blockIdx.x * chunk; c0 < npts; c0 += (int64_t)gridDim.x * chunk) {
    const int64_t w0 = c0 + (int64_t)(threadIdx.x >> 5) * 32 * U;
    uint64_t key[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = w0 + u * 32 + lane;
      key[u] = EMPTY_KEY;
      if (i < npts) {
        T x[D];
#pragma unroll
        for (int d = 0; d < D; ++d) x[d] = pts[(lo0 + i) * D + d];
        int32_t code;
        key[u] = cell_key<D, T>(x, sp.inv_cell, &code);
        if (code) set_err(b.bs, code);
        sp.keys[lo0 + i] = key[u];
        int64_t k[3];
        unpack_key(key[u], H, k);
#pragma unroll
        for (int d = 0; d < H; ++d) {
          cmn[d] = min(cmn[d], (long long)k[d]);
          cmx[d] = max(cmx[d], (long long)k[d]);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = w0 + u * 32 + lane;
      const bool valid = key[u] != EMPTY_KEY;
      const uint32_t bin = valid ? bin_of_key(key[u], H) : 0u;
      const uint32_t comp = valid ? bin * (uint32_t)sp.ts + (uint32_t)i / S32 : 0xffffffffu;
      const unsigned peers = __match_any_sync(0xffffffffu, comp);
      const int leader = __ffs(peers) - 1;
      const uint64_t lkey = __shfl_sync(0xffffffffu, key[u], leader);
      const bool mixed_grp = (__ballot_sync(0xffffffffu, key[u] != lkey) & peers) != 0;
      int slot = -1;
      if (valid && lane == leader) {
        const uint32_t c = (uint32_t)__popc(peers);
        uint32_t sl = (comp * 2654435761u) >> (32 - HIST_BITS);
#pragma unroll 1
        for (int probe = 0; probe < 8; ++probe) {
          const uint32_t old = atomicCAS(&hkey[sl], 0xffffffffu, comp);
          if (old == 0xffffffffu || old == comp) {
            atomicAdd(&hcnt[sl], c);
            slot = (int)sl;
            break;
          }
          sl = (sl + 1) & (HIST_SLOTS - 1);
        }
        if (slot < 0) {
          atomicAdd(&sp.cnt[comp], c);
          atomicAdd(&sp.bin_count[bin], c);
        }
      }
      // key range of the bin: the leader alone when the group's keys agree
      slot = __shfl_sync(0xffffffffu, slot, leader);
      if (valid && (mixed_grp || lane == leader)) {
        if (slot >= 0) {
          atomicMin(&hmin[slot], (unsigned long long)key[u]);
          atomicMax(&hmax[slot], (unsigned long long)key[u]);
        } else {
          atomicMin(&sp.kmin[bin], (unsigned long long)key[u]);
          atomicMax(&sp.kmax[bin], (unsigned long long)key[u]);
        }
      }
    }
  }
#pragma unroll
  for (int d = 0; d < H; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cmn[d] = min(cmn[d], __shfl_xor_sync(0xffffffffu, cmn[d], o));
      cmx[d] = max(cmx[d], __shfl_xor_sync(0xffffffffu, cmx[d], o));
    }
    if (lane == 0) {
      s_cr[0][d][threadIdx.x >> 5] = cmn[d];
      s_cr[1][d][threadIdx.x >> 5] = cmx[d];
    }
  }
  __syncthreads();
  if (threadIdx.x < H) {
    const int d = threadIdx.x;
    long long mn = LLONG_MAX, mx = LLONG_MIN;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      mn = min(mn, s_cr[0][d][w]);
      mx = max(mx, s_cr[1][d][w]);
    }
    if (mn <= mx) {
      atomicMin(&sp.sc->cmin[d], mn);
      atomicMax(&sp.sc->cmax[d], mx);
    }
  }
  for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
    const uint32_t comp = hkey[t];
    if (comp != 0xffffffffu) {
      const uint32_t bin = comp / (uint32_t)sp.ts;
      atomicAdd(&sp.cnt[comp], hcnt[t]);
      atomicAdd(&sp.bin_count[bin], hcnt[t]);
      atomicMin(&sp.kmin[bin], hmin[t]);
      atomicMax(&sp.kmax[bin], hmax[t]);
    }
  }
}

// ---------------------------------------------------------------------------
// k_span_prefix: one warp per bin in use (the list k_span_scan built),
// striding over the list. The bin's block counts are one contiguous row of
// cnt: the warp reads it 32 blocks per load (8 loads in flight), scans each
// 32-block step with a warp scan plus the running carry, and writes the
// bin's row of pre (pre[b][nblk] = all its span points).
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(256) k_span_prefix(Batch b, Span sp) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const uint32_t nu = sp.sc->n_used;
  const int64_t nblk = sp.nblk;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t u = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < nu; u += warps) {
    const uint32_t bin = sp.used[u];
    const uint32_t* __restrict__ cnt = sp.cnt + (int64_t)bin * sp.ts;
    uint32_t* __restrict__ pre = sp.pre + (int64_t)bin * sp.ts;
    uint32_t carry = 0;
    for (int64_t r0 = 0; r0 < nblk; r0 += 256) {
      uint32_t v[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int64_t t = r0 + 32 * e + lane;
        v[e] = t < nblk ? cnt[t] : 0u;
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        uint32_t inc = v[e];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += y;
        }
        const int64_t t = r0 + 32 * e + lane;
        if (t < nblk) pre[t] = carry + inc - v[e];
        carry += __shfl_sync(0xffffffffu, inc, 31);
      }
    }
    if (lane == 0) pre[nblk] = carry;
  }
}

// k_span_scan: bin_start of the span (exclusive scan of bin_count), the list
// of bins in use (each thread appends its non-empty bins of 4) and the
// span's purity.
static __global__ void __launch_bounds__(256) k_span_scan(Batch b, Span sp) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t s_base;
  pdl_trigger();
  pdl_wait();
  scan_bins<SPAN_SCAN_TILE>(sp.bin_count, sp.bin_start, sp.scan_status, &sp.sc->scan_ticket, b.bs);
  // this block's SPAN_SCAN_TILE bins (scan_bins took a tile by ticket; any
  // split of the bins over the blocks will do here)
  constexpr int Q = SPAN_SCAN_TILE / 1024;
  const uint32_t b0 = blockIdx.x * SPAN_SCAN_TILE + threadIdx.x * 4 * Q;
  uint32_t c[4 * Q];
  uint32_t nz = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const uint4 v = *reinterpret_cast<const uint4*>(sp.bin_count + b0 + 4 * q);
    c[4 * q] = v.x; c[4 * q + 1] = v.y; c[4 * q + 2] = v.z; c[4 * q + 3] = v.w;
  }
#pragma unroll
  for (int e = 0; e < 4 * Q; ++e) nz += c[e] != 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // pure: the span's cells, widened by the sure / group-rule neighbours
    // (within n-2), map to distinct bins
    const int margin = 2 * max(sp.n - 2, 0);
    const long long* mn = sp.sc->cmin;
    const long long* mx = sp.sc->cmax;
    sp.sc->pure = sp.h == 1 ? box_pure<1>(mn, mx, margin)
                            : (sp.h == 2 ? box_pure<2>(mn, mx, margin) : box_pure<3>(mn, mx, margin));
  }
  uint32_t total;
  const uint32_t ex = block_exclusive_scan(nz, &total, sm);
  if (threadIdx.x == 0) s_base = total ? atomicAdd(&sp.sc->n_used, total) : 0u;
  __syncthreads();
  uint32_t o = s_base + ex;
#pragma unroll
  for (int e = 0; e < 4 * Q; ++e)
    if (c[e]) sp.used[o++] = b0 + e;
}

// ---------------------------------------------------------------------------
// k_span_scatter: the span in (bin, block) order. A block-local table
// aggregates the points of one chunk per (block, bin); each entry claims its
// positions with one atomicSub on cnt, which returns cnt to zero.
// ---------------------------------------------------------------------------
template <int D, typename T>
__global__ void __launch_bounds__(256) k_span_scatter(Batch b, Span sp) {
  constexpr int H = Hashed<D>::value;
  __shared__ uint32_t tkey[HIST_SLOTS];
  __shared__ uint32_t tcnt[HIST_SLOTS];
  __shared__ uint32_t tbase[HIST_SLOTS];
  pdl_trigger();
  pdl_wait();
  constexpr int U = 2;  // points per thread and step (measured: 2 beats 1 and 4)
  const int64_t lo0 = span_lo(b);
  const int64_t npts = sp.nblk * sp.S;
  if (blockIdx.x == 0 && threadIdx.x < SPAN_SCAN_TILES) sp.scan_status[threadIdx.x] = 0;
  for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
    tkey[t] = 0xffffffffu;
    tcnt[t] = 0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const uint32_t S32 = (uint32_t)sp.S;
  const int64_t chunk = (int64_t)blockDim.x * U;
  for (int64_t c0 = (int64_t)blockIdx.x * chunk; c0 < npts; c0 += (int64_t)gridDim.x * chunk) {
    const int64_t w0 = c0 + (int64_t)(threadIdx.x >> 5) * 32 * U;
    uint64_t key[U];
    uint32_t comp[U], goff[U];
    int slot[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = w0 + u * 32 + lane;
      key[u] = i < npts ? sp.keys[lo0 + i] : EMPTY_KEY;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = w0 + u * 32 + lane;
      const bool valid = key[u] != EMPTY_KEY;
      comp[u] = valid ? bin_of_key(key[u], H) * (uint32_t)sp.ts + (uint32_t)i / S32 : 0xffffffffu;
      const unsigned peers = __match_any_sync(0xffffffffu, comp[u]);
      const int leader = __ffs(peers) - 1;
      int sl_found = -1;
      uint32_t off = 0;
      if (valid && lane == leader) {
        const uint32_t c = (uint32_t)__popc(peers);
        uint32_t sl = (comp[u] * 2654435761u) >> (32 - HIST_BITS);
#pragma unroll 1
        for (int probe = 0; probe < 8; ++probe) {
          const uint32_t old = atomicCAS(&tkey[sl], 0xffffffffu, comp[u]);
          if (old == 0xffffffffu || old == comp[u]) {
            off = atomicAdd(&tcnt[sl], c);
            sl_found = (int)sl;
            break;
          }
          sl = (sl + 1) & (HIST_SLOTS - 1);
        }
        if (sl_found < 0) off = atomicSub(&sp.cnt[comp[u]], c) - c;  // table full: claim directly
      }
      slot[u] = __shfl_sync(0xffffffffu, sl_found, leader);
      goff[u] = __shfl_sync(0xffffffffu, off, leader) + __popc(peers & lt);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < HIST_SLOTS; t += blockDim.x) {
      const uint32_t k = tkey[t];
      if (k != 0xffffffffu) {
        const uint32_t c = tcnt[t];
        tbase[t] = atomicSub(&sp.cnt[k], c) - c;
        tkey[t] = 0xffffffffu;
        tcnt[t] = 0;
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (comp[u] != 0xffffffffu) {
        const int64_t i = w0 + u * 32 + lane;
        const uint32_t bin = comp[u] / (uint32_t)sp.ts;
        const uint32_t pos = sp.bin_start[bin] + sp.pre[comp[u]] + goff[u] + (slot[u] >= 0 ? tbase[slot[u]] : 0u);
        sp.s_off[pos] = (uint32_t)i;
#pragma unroll
        for (int d = 0; d < D; ++d)
          static_cast<T*>(sp.s_x)[(int64_t)d * sp.Wp + pos] = static_cast<const T*>(sp.pts)[(lo0 + i) * D + d];
      }
    }
  }
}

// 1-d group rule of the window engine over window counts of the span: the
// 2n-3 cells within n-2 of the cell of bin `bin` (all within R of every
// point of that cell), or some run of n-1 consecutive cells containing it
// (all within R of each other), hold more than K window points, every bin
// involved holding nothing in the window or only its expected cell over the
// whole span.
__device__ __forceinline__ bool span_group_safe(const Span& sp, const WinPre& wp, uint32_t bin, bool pure) {
  const int m = sp.n - 1;
  if (m < 2 || bin < (uint32_t)(m - 1) || bin + m > NB - 1) return false;
  constexpr int MMAX = 7;
  uint32_t wc[2 * MMAX - 1];
  bool ok[2 * MMAX - 1];
  const unsigned long long key = sp.kmin[bin];
#pragma unroll
  for (int t = 0; t < 2 * MMAX - 1; ++t) {
    wc[t] = 0;
    ok[t] = false;
    if (t < 2 * m - 1) {
      const uint32_t j = bin - m + 1 + t;
      const bool any = sp.bin_count[j] != 0;
      wc[t] = any ? wp.count(j) : 0u;
      const unsigned long long want = key + (unsigned long long)(t - (m - 1));
      ok[t] = pure || wc[t] == 0 || (sp.kmin[j] == want && sp.kmax[j] == want);
    }
  }
  {  // the whole neighbourhood of 2n-3 cells
    bool all = true;
    uint32_t sum = 0;
#pragma unroll
    for (int t = 0; t < 2 * MMAX - 1; ++t)
      if (t < 2 * m - 1) {
        all &= ok[t];
        sum += wc[t];
      }
    if (all && sum > (uint32_t)sp.K) return true;
  }
#pragma unroll
  for (int g = 0; g < MMAX; ++g) {
    if (g < m) {
      bool all = true;
      uint32_t sum = 0;
#pragma unroll
      for (int t = 0; t < MMAX; ++t)
        if (t < m) {
          all &= ok[g + t];
          sum += wc[g + t];
        }
      if (all && sum > (uint32_t)sp.K) return true;
    }
  }
  return false;
}

// ---------------------------------------------------------------------------
// Exact counts of the nq points of window j in bin `bin` (bin-ordered
// positions [p, p + nq)) by one warp (count_group): the candidates of
// stencil bin sb are its points in window j, positions [bin_start[sb] +
// pre[j][sb], bin_start[sb] + pre[j + W/S][sb]); sure slots are used in a
// pure span of up to 3 dimensions. Outliers set their bit in the slide's
// bitset row.
// ---------------------------------------------------------------------------
template <int D, int PRED, typename T>
__device__ __forceinline__ int span_count_group(const Batch& b, const Span& sp, uint32_t p, uint32_t nq,
                                                uint32_t bin, const WinPre& wp, bool pure,
                                                unsigned long long* made = nullptr) {
  const int j = wp.j;
  const Job& jb = b.jobs[j];
  const int64_t shift = (int64_t)j * sp.S;  // window offset = span offset - shift
  uint32_t* row = sp.bits + ((jb.ctr->lo - sp.S) / sp.S % sp.chunk) * sp.words;
  const GroupArgs ga{p, nq, bin, sp.n, sp.K, sp.R2f, sp.R, sp.R2, sp.Wp, pure && D <= 3, &b.bs->pair_tests};
  const int nout = count_group_ex<D, PRED, T>(
      static_cast<const T*>(sp.s_x), ga,
      [&](uint32_t sb, uint32_t& rs, uint32_t& len) {
        const uint32_t b0 = sp.bin_start[sb], b1 = sp.bin_start[sb + 1];
        if (b1 > b0) {
          const uint32_t* row = wp.pre + (int64_t)sb * wp.ts + wp.j;
          rs = b0 + row[0];
          len = row[wp.wblk] - row[0];
        }
      },
      [&](uint32_t pos) {
        const int64_t w2 = (int64_t)sp.s_off[pos] - shift;
        atomicOr(&row[w2 >> 5], 1u << (w2 & 31));
      },
      [&](uint32_t i) { return p + i; }, [](uint32_t, int, int) {}, made);
  if ((threadIdx.x & 31) == 0 && nout) atomicAdd(&jb.ctr->n_out, nout);
  return nout;
}

// ---------------------------------------------------------------------------
// Learned routing of the span engine's exact counts (rtod_config.router).
//
// Consecutive windows of a batch share all but two slide blocks, so a
// point's neighbour count in window j equals its count in window j-1 plus
// its neighbours in the block that window j adds, minus those in the block
// it drops. A "delta segment" is a run of up to SEG_LEN consecutive windows
// of one bin that all need counting, taken by one warp in window order: the
// first window is counted in full (count_group), and every later window
// only tests the points both windows share against the two changed blocks
// of the stencil (about 2/(W/S) of the candidates), keeping for each point
// bounds [lo, hi] of its count (exact after a full sweep; lo > K only after
// an early exit). A point whose bounds leave K inside after the update, and
// the window's new points, are counted in full again. The result is exact
// either way. A delta segment pays off when the bin's points would test many
// candidates (large stencils, outliers); an independent early-exit count
// when they test few, since it runs in parallel instead of window after
// window. The router's network predicts, from the cell occupancy of the
// run's first window (cheap to read at classification), whether an
// independent count is the cheaper (bucket 3), a label the count kernel
// derives from what it has just counted (the stencil's candidates and the
// outliers found, route_label); k_span_classify routes predicted bucket-3
// runs to independent counts and the rest to delta segments. The network is
// trained on the GPU on samples of those counts (k_train); the autotuner
// also times routing off and the threshold's extremes.
// ---------------------------------------------------------------------------
constexpr int SEG_LEN = 8;                // windows per delta segment at most
constexpr int SEG_CAP = 64;               // points of the bin in any window of a delta segment at most
                                          // (measured: 128 lets dense bins in, whose inliers exit
                                          // early, and the 3-d sensor-like gain fell from 27% to 5%)
constexpr int SEG_PPL = SEG_CAP / 32;     // shared points per lane in a delta step
constexpr int SEG_RING = 2 * SEG_CAP;     // per-warp bounds, indexed by position mod SEG_RING
constexpr uint32_t SAMPLE_THIN = 8;       // groups and segment windows sampled for training: one in 8

// Router features of (window j, bin): f0 = log2(1 + points of the bin) / 8,
// f1 = log2(1 + points of the bins b-1, b, b+1: the neighbouring cells along
// the last hashed dimension) / 8, f2 = points of the bin / (K + 1), at most 2.
__device__ __forceinline__ void span_features(const Span& sp, const WinPre& wp, uint32_t bin, uint32_t wc, float* f) {
  uint32_t row = 0;
#pragma unroll
  for (int d = -1; d <= 1; ++d) {
    const uint32_t nb = (bin + (uint32_t)d) & NB_MASK;
    if (sp.bin_start[nb + 1] > sp.bin_start[nb]) row += wp.count(nb);
  }
  f[0] = log2f(1.0f + (float)wc) * 0.125f;
  f[1] = log2f(1.0f + (float)row) * 0.125f;
  f[2] = fminf(2.0f, (float)wc / (float)(sp.K + 1));
}

// Candidates of (window j, bin) over its whole stencil (one warp; slots <= 32).
template <int H>
__device__ __forceinline__ uint32_t span_stencil_total(const Span& sp, uint32_t bin, uint32_t j) {
  const int lane = threadIdx.x & 31;
  const int w = 2 * sp.n + 1;
  const int slots = H == 1 ? w : (H == 2 ? w * w : w * w * w);
  uint32_t c = 0;
  if (lane < slots) {
    int d[3] = {0, 0, 0};
    const uint32_t sb = (bin + (uint32_t)slot_cell<H>(lane, sp.n, d)) & NB_MASK;
    if (sp.bin_start[sb + 1] > sp.bin_start[sb]) {
      const uint32_t* r = sp.pre + (int64_t)sb * sp.ts + j;
      c = r[sp.wblk] - r[0];
    }
  }
  return __reduce_add_sync(0xffffffffu, c);
}

// Label of a counted (window, bin) of wc points, nout of them outliers, C
// stencil candidates: 3 when an independent early-exit count costs less
// than a delta step, else 0: the work of each in distance tests plus a
// fixed cost per count. Independent: `made` tests when it ran that way (else
// outliers sweep all C candidates, inliers about half of them); a delta
// step: `made` tests when it ran that way (else the shared points against
// the two changed blocks, 2C/(W/S) each, and the new points, wc/(W/S), in
// full). The label measures work only; where the count stage is bound by
// latency rather than work (short 1-d candidate lists, whose delta segments
// lengthen the chain of dependent steps), the autotuner, which times routing
// off as well, turns routing off.
__device__ __forceinline__ int route_label(const Span& sp, uint32_t wc, int nout, uint32_t C, bool ran_indep,
                                           unsigned long long made) {
  const float f = (float)C, blk = (float)sp.wblk, n = (float)wc, o = (float)nout;
  const float ind = (ran_indep ? (float)made : o * f + (n - o) * 0.5f * f) + 256.0f;
  const float del = (ran_indep ? n * 2.0f * f / blk + n / blk * f : (float)made) + 256.0f;
  return ind <= del ? 3 : 0;
}

// One training sample (lane 0 of the warp) into the block's buffer.
__device__ __forceinline__ void span_sample(SampleBuf& sb, const float* f, int label, bool routed_early) {
  if ((label == 3) != routed_early) atomicAdd(&sb.misrouted, 1u);
  const uint32_t k = atomicAdd(&sb.n, 1u);
  if (k >= BLOCK_SAMPLES) return;
  sb.s[k][0] = f[0];
  sb.s[k][1] = f[1];
  sb.s[k][2] = f[2];
  sb.s[k][3] = (float)label;
}

__device__ __forceinline__ bool span_sampled(uint32_t bin, uint32_t j) {
  return ((bin * 2654435761u + j * 40503u) >> 16) % SAMPLE_THIN == 0;
}

struct SegWarp {
  int32_t lo[SEG_RING];
  int32_t hi[SEG_RING];
  uint32_t redo[SEG_CAP];
};

// Counts a delta segment: windows j0 .. j0 + len - 1 of bin `bin`, every one
// holding 1..SEG_CAP points of the bin. One warp; sw is its shared state.
template <int D, int PRED, typename T>
__device__ void span_count_segment(const Batch& b, const Span& sp, uint32_t bin, uint32_t j0, uint32_t len,
                                   bool pure, SegWarp& sw, SampleBuf& sbuf) {
  constexpr int H = Hashed<D>::value;
  const int lane = threadIdx.x & 31;
  const T* sx = static_cast<const T*>(sp.s_x);
  const uint32_t B0 = sp.bin_start[bin];
  const uint32_t* prow = sp.pre + (int64_t)bin * sp.ts;
  // this lane's stencil slot (at most 32 slots: checked by the host)
  const int w = 2 * sp.n + 1;
  const int slots = H == 1 ? w : (H == 2 ? w * w : w * w * w);
  uint32_t sbase = 0;
  const uint32_t* srow = nullptr;
  if (lane < slots) {
    int d[3] = {0, 0, 0};
    const uint32_t sb = (bin + (uint32_t)slot_cell<H>(lane, sp.n, d)) & NB_MASK;
    if (sp.bin_start[sb + 1] > sp.bin_start[sb]) {
      sbase = sp.bin_start[sb];
      srow = sp.pre + (int64_t)sb * sp.ts;
    }
  }
  unsigned long long tests = 0;
  uint32_t e_prev = 0;
  for (uint32_t t = 0; t < len; ++t) {
    const uint32_t j = j0 + t;
    const uint32_t s = B0 + prow[j], e = B0 + prow[j + sp.wblk];
    const Job& jb = b.jobs[j];
    uint32_t* row = sp.bits + ((jb.ctr->lo - sp.S) / sp.S % sp.chunk) * sp.words;
    const int64_t shift = (int64_t)j * sp.S;
    const WinPre wp{sp.pre, sp.ts, (int)j, sp.wblk};
    auto mark = [&](uint32_t pos) {
      const int64_t w2 = (int64_t)sp.s_off[pos] - shift;
      atomicOr(&row[w2 >> 5], 1u << (w2 & 31));
    };
    auto rec = [&](uint32_t pos, int lo, int hi) {
      sw.lo[pos & (SEG_RING - 1)] = lo;
      sw.hi[pos & (SEG_RING - 1)] = hi;
    };
    auto range = [&](uint32_t sb, uint32_t& rs, uint32_t& l) {
      const uint32_t b0 = sp.bin_start[sb], b1 = sp.bin_start[sb + 1];
      if (b1 > b0) {
        const uint32_t* r = wp.pre + (int64_t)sb * wp.ts + wp.j;
        rs = b0 + r[0];
        l = r[wp.wblk] - r[0];
      }
    };
    int nout = 0;
    uint32_t nredo = 0, first_new = s;
    unsigned long long made = 0;  // distance tests of this window
    if (t > 0) {
      // Points of both windows, positions [s, e_prev): their counts change by
      // their neighbours in block j - 1 + W/S (added) minus those in block
      // j - 1 (dropped). The lane's slot contributes its points of both blocks
      // to one virtual list of signed candidates.
      const uint32_t told = j - 1, tnew = j - 1 + (uint32_t)sp.wblk;
      uint32_t ds = 0, dn = 0, as = 0, an = 0;
      if (srow) {
        ds = sbase + srow[told];
        dn = srow[told + 1] - srow[told];
        as = sbase + srow[tnew];
        an = srow[tnew + 1] - srow[tnew];
      }
      const uint32_t mine = dn + an;
      uint32_t inc = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
      }
      const uint32_t off = inc - mine, nd = __shfl_sync(0xffffffffu, inc, 31);
      const uint32_t nc = e_prev - s;
      T xq[SEG_PPL][D];
#pragma unroll
      for (int h = 0; h < SEG_PPL; ++h)
#pragma unroll
        for (int d = 0; d < D; ++d)
          xq[h][d] = lane + 32 * h < (int)nc ? sx[(int64_t)d * sp.Wp + s + 32 * h + lane] : T(0);
      int acc[SEG_PPL];
#pragma unroll
      for (int h = 0; h < SEG_PPL; ++h) acc[h] = 0;
      for (uint32_t c0 = 0; c0 < nd; c0 += 32) {
        const uint32_t v = c0 + lane;
        int src = 0;  // lane holding v: the last lane whose offset is <= v
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int cand = src + step;
          if (__shfl_sync(0xffffffffu, off, cand & 31) <= v) src = cand;
        }
        const uint32_t o_off = __shfl_sync(0xffffffffu, off, src), o_ds = __shfl_sync(0xffffffffu, ds, src),
                       o_dn = __shfl_sync(0xffffffffu, dn, src), o_as = __shfl_sync(0xffffffffu, as, src);
        const uint32_t k = v - o_off;
        const bool valid = v < nd;
        const uint32_t pos = k < o_dn ? o_ds + k : o_as + (k - o_dn);
        const int sg = k < o_dn ? -1 : 1;
        T cx[D];
#pragma unroll
        for (int d = 0; d < D; ++d) cx[d] = valid ? sx[(int64_t)d * sp.Wp + pos] : T(0);
        const uint32_t m = min(32u, nd - c0);
        for (uint32_t c = 0; c < m; ++c) {
          T y[D];
#pragma unroll
          for (int d = 0; d < D; ++d) y[d] = __shfl_sync(0xffffffffu, cx[d], c);
          const int g = __shfl_sync(0xffffffffu, sg, c);
#pragma unroll
          for (int h = 0; h < SEG_PPL; ++h)
            if (lane + 32 * h < (int)nc && is_nbr<D, PRED, T>(xq[h], y, sp.R2f, sp.R, sp.R2)) acc[h] += g;
        }
      }
      tests += (unsigned long long)nc * nd;
      made += (unsigned long long)nc * nd;
#pragma unroll
      for (int h = 0; h < SEG_PPL; ++h) {
        const uint32_t idx = (uint32_t)lane + 32u * h;
        const uint32_t pos = s + idx;
        bool out = false, redo = false;
        if (idx < nc) {
          const int sl = pos & (SEG_RING - 1);
          const int lo = sw.lo[sl] + acc[h];
          const int hi = sw.hi[sl] >= CNT_INF ? CNT_INF : sw.hi[sl] + acc[h];
          sw.lo[sl] = lo;
          sw.hi[sl] = hi;
          if (lo <= sp.K) {
            if (hi <= sp.K) {
              out = true;
              mark(pos);
            } else {
              redo = true;
            }
          }
        }
        nout += __popc(__ballot_sync(0xffffffffu, out));
        const unsigned rm = __ballot_sync(0xffffffffu, redo);
        if (redo) sw.redo[nredo + __popc(rm & lanemask_lt())] = pos;
        nredo += __popc(rm);
      }
      __syncwarp();
      first_new = e_prev;
    }
    // Full counts: the window's new points [first_new, e) and the points
    // whose bounds still hold K.
    const uint32_t nnew = e - first_new;
    if (nnew + nredo) {
      const GroupArgs ga{first_new, nnew + nredo, bin, sp.n, sp.K, sp.R2f, sp.R, sp.R2, sp.Wp, pure && D <= 3,
                         &b.bs->pair_tests};
      unsigned long long m2 = 0;
      nout += count_group_ex<D, PRED, T>(
          sx, ga, range, mark, [&](uint32_t i) { return i < nnew ? first_new + i : sw.redo[i - nnew]; }, rec, &m2);
      made += m2;
    }
    __syncwarp();
    if (lane == 0 && nout) atomicAdd(&jb.ctr->n_out, nout);
    if (span_sampled(bin, j)) {
      const uint32_t C = span_stencil_total<H>(sp, bin, j);
      if (lane == 0) {
        float f[MLP_IN];
        span_features(sp, wp, bin, e - s, f);
        span_sample(sbuf, f, route_label(sp, e - s, nout, C, false, made), false);
      }
    }
    e_prev = e;
  }
  if (lane == 0 && tests) atomicAdd(&b.bs->pair_tests, tests);
}

// Clears the per-bin state of the span's bins in use (all blocks of the
// launch share the work; finish_batch then clears the count of bins).
__device__ __forceinline__ void span_clear_bins(const SpanCtr* c) {
  const int64_t nb = (int64_t)gridDim.x * gridDim.y;
  const int64_t f = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
  const uint32_t nu = c->n_used;
  for (int64_t u = f * blockDim.x + threadIdx.x; u < nu; u += nb * blockDim.x) {
    const uint32_t bin = c->used[u];
    c->bin_count[bin] = 0;
    c->kmin[bin] = EMPTY_KEY;
    c->kmax[bin] = 0;
  }
}

// ---------------------------------------------------------------------------
// k_span_classify: one thread per (window, bin in use): the window's count of
// the bin from pre; a bin that is not provably all-inlier in that window
// (more than K window points in its single cell, in the 1-d group rule's
// cells, or, in a pure span of 2-3 hashed dimensions, in the cells within R
// of every point of its cell) is appended to the batch's list of groups to
// count (first position, points, bin, window): one atomic per warp for the
// list, one per window present in the warp for its count of listed points.
// Pairs run bin-major (consecutive windows of a bin together), so the list
// holds a bin's windows side by side and neighbouring count warps read
// mostly the same candidates. With ROUTE (the learned router), runs of up to
// SEG_LEN consecutive windows of one bin, each with at most SEG_CAP points of
// the bin, are routed by the network (features of the run's first window):
// predicted mostly-inlier runs are listed window by window as above, the
// others as one delta segment each (from the back of the list: first
// position, windows, bin, first window).
// ---------------------------------------------------------------------------
template <bool ROUTE>
__global__ void __launch_bounds__(256) k_span_classify(Batch b, Span sp) {
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const uint32_t nu = sp.sc->n_used;
  const bool pure = sp.sc->pure;
  const int64_t pairs = (int64_t)nu * b.njobs;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t e_end = (pairs + 31) & ~31ll;  // whole warps stay in the loop together
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < e_end; e += stride) {
    int j = -1;
    uint32_t start = 0, wc = 0, bin = 0;
    bool need = false;
    if (e < pairs) {
      // bin-major pairs: a warp takes consecutive windows of one bin (one
      // contiguous row of pre), and consecutive groups share their stencil
      const int64_t u = e / b.njobs;
      j = (int)(e - u * b.njobs);
      bin = sp.used[u];
      const WinPre wp{sp.pre, sp.ts, j, sp.wblk};
      const uint32_t* row = sp.pre + (int64_t)bin * sp.ts + j;
      const uint32_t a = row[0];
      wc = row[sp.wblk] - a;
      if (wc) {
        bool safe = false;
        if (sp.filter) {
          const bool single = pure || sp.kmin[bin] == sp.kmax[bin];
          safe = single && wc > (uint32_t)sp.K;
          if (!safe && single && sp.h == 1 && sp.n >= 3) safe = span_group_safe(sp, wp, bin, pure);
          if (!safe && pure && sp.h > 1 && sp.n_sure > 1) {
            // the sure neighbourhood: cells within R of every point of this one
            uint32_t sum = 0;
            for (int t = 0; t < sp.n_sure; ++t) {
              const uint32_t nb = (bin + (uint32_t)sp.sure_delta[t]) & NB_MASK;
              if (sp.bin_count[nb]) sum += wp.count(nb);
            }
            safe = sum > (uint32_t)sp.K;
          }
        }
        need = !safe;
        start = sp.bin_start[bin] + a;
      }
    }
    const unsigned peers = __match_any_sync(0xffffffffu, need ? j : -1);
    if (need) {
      const uint32_t pts = __reduce_add_sync(peers, wc);
      if (lane == __ffs(peers) - 1) atomicAdd(&b.jobs[j].ctr->n_undet, (int)pts);
    }
    bool indep = need;  // listed as an independent group
    if constexpr (ROUTE) {
      // Runs of eligible windows of one bin inside the warp's 32 pairs, cut
      // into segments of SEG_LEN windows; each segment's first lane routes it.
      const bool el = need && wc <= (uint32_t)SEG_CAP;
      const uint32_t pbin = __shfl_up_sync(0xffffffffu, bin, 1);
      const bool pel = __shfl_up_sync(0xffffffffu, el ? 1 : 0, 1) != 0;
      const unsigned cont = __ballot_sync(0xffffffffu, lane > 0 && el && pel && pbin == bin);
      const unsigned elm = __ballot_sync(0xffffffffu, el);
      const unsigned le = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);  // lanes <= this one
      const unsigned heads = elm & ~cont;
      const int rhead = el ? 31 - __clz(heads & le) : lane;
      const bool shead = el && ((lane - rhead) % SEG_LEN) == 0;
      const unsigned sheads = __ballot_sync(0xffffffffu, shead);
      const int myhead = el ? 31 - __clz(sheads & le) : lane;
      bool delta = false;
      uint32_t slen = 0;
      if (shead) {
        float f[MLP_IN];
        span_features(sp, WinPre{sp.pre, sp.ts, j, sp.wblk}, bin, wc, f);
        delta = !route_early(b.router, f);
        const unsigned stop = (~cont | sheads) & ~le;  // lanes after this one that start a run or segment
        slen = (uint32_t)((stop ? __ffs(stop) - 1 : 32) - lane);
      }
      const bool my_delta = __shfl_sync(0xffffffffu, delta ? 1 : 0, myhead & 31) != 0;
      if (el && my_delta) indep = false;
      const unsigned dheads = __ballot_sync(0xffffffffu, shead && delta);
      uint32_t sbase = 0;
      if (lane == 0 && dheads) sbase = atomicAdd(&sp.sc->n_segs, (uint32_t)__popc(dheads));
      sbase = __shfl_sync(0xffffffffu, sbase, 0);
      if (shead && delta)
        sp.groups[sp.gcap - 1 - (sbase + __popc(dheads & lanemask_lt()))] = make_uint4(start, slen, bin, (uint32_t)j);
      const unsigned em = __ballot_sync(0xffffffffu, el);
      const unsigned dm = __ballot_sync(0xffffffffu, el && my_delta);
      if (lane == 0 && (em || dm)) {
        atomicAdd(&b.router->routed_early, (unsigned long long)__popc(em & ~dm));
        atomicAdd(&b.router->routed_sweep, (unsigned long long)__popc(dm));
      }
    }
    const unsigned nmask = __ballot_sync(0xffffffffu, indep);
    uint32_t gbase = 0;
    if (lane == 0 && nmask) gbase = atomicAdd(&sp.sc->n_groups, (uint32_t)__popc(nmask));
    gbase = __shfl_sync(0xffffffffu, gbase, 0);
    if (indep) sp.groups[gbase + __popc(nmask & lanemask_lt())] = make_uint4(start, wc, bin, (uint32_t)j);
  }
}

// ---------------------------------------------------------------------------
// k_span_count: one warp per listed group of the batch, warps striding over
// the list (measured against groups taken by ticket, one atomic per group or
// only for the last round: the static stride was as fast on the 3-d
// sensor-like stream and 20-40% faster on the 1-d streams, whose groups are
// too short to pay for the atomics). Outliers set their bit in the slide's
// bitset row. Then the blocks clear the per-bin state, and the block that
// finishes last ends the batch (records, window advance, counters).
// ---------------------------------------------------------------------------
// With ROUTE, the warps first take the delta segments by ticket (from the
// back of the list), and every sampled group or segment window leaves a
// training sample for the router.
template <int D, int PRED, typename T, bool ROUTE = false>
__global__ void __launch_bounds__(256) k_span_count(Batch b, Span sp) {
  __shared__ int s_last;
  __shared__ SegWarp s_seg[ROUTE ? 8 : 1];
  __shared__ SampleBuf s_samples;
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const uint32_t ng = sp.sc->n_groups;
  const bool pure = sp.sc->pure;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if constexpr (ROUTE) {
    if (threadIdx.x == 0) {
      s_samples.n = 0;
      s_samples.misrouted = 0;
    }
    __syncthreads();
    const uint32_t ns = sp.sc->n_segs;
    while (true) {
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(&sp.sc->seg_ticket, 1u);
      k = __shfl_sync(0xffffffffu, k, 0);
      if (k >= ns) break;
      const uint4 g = sp.groups[sp.gcap - 1 - k];
      span_count_segment<D, PRED, T>(b, sp, g.z, g.w, g.y, pure, s_seg[(threadIdx.x >> 5) & 7], s_samples);
    }
  }
  auto one = [&](uint32_t k) {
    const uint4 g = sp.groups[k];
    unsigned long long made = 0;
    const int nout = span_count_group<D, PRED, T>(b, sp, g.x, g.y, g.z, WinPre{sp.pre, sp.ts, (int)g.w, sp.wblk},
                                                  pure, ROUTE ? &made : nullptr);
    if constexpr (ROUTE) {
      if (span_sampled(g.z, g.w)) {
        const uint32_t C = span_stencil_total<Hashed<D>::value>(sp, g.z, g.w);
        if (lane == 0) {
          float f[MLP_IN];
          span_features(sp, WinPre{sp.pre, sp.ts, (int)g.w, sp.wblk}, g.z, g.y, f);
          span_sample(s_samples, f, route_label(sp, g.y, nout, C, true, made), true);
        }
      }
    }
  };
  bool ticketed = false;
  if constexpr (ROUTE) ticketed = sp.sc->n_segs > 0;
  if (ticketed) {
    // after the segments, the independent groups by ticket as well: warps
    // finish their segments at different times (3-d sensor-like stream: the
    // pass 3.5 -> 2.9 us per slide against a static stride here)
    while (true) {
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(&sp.sc->group_ticket, 1u);
      k = __shfl_sync(0xffffffffu, k, 0);
      if (k >= ng) break;
      one(k);
    }
  } else {
    for (uint32_t k = warp; k < ng; k += nw) one(k);
  }
  if constexpr (ROUTE) flush_samples(s_samples, b.router);
  // The per-bin state is no longer read in this batch: clear it, then the
  // block that finishes last ends the batch.
  span_clear_bins(sp.sc);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&b.bs->done, 1u) == gridDim.x * gridDim.y - 1;
  __syncthreads();
  if (s_last) finish_batch(b);
}

// ---------------------------------------------------------------------------
// Deferred compaction of a chunk of slides [s0, s0 + n): k_span_compact, one
// block per slide, turns the slide's bitset row into sorted global indices
// at the slide's output offset (recorded by finish_batch; 4 words per
// thread, one block scan per 4096 words) and clears the row. The IDs of a
// step are gathered in shared memory (up to SPAN_CMP_SMEM_IDS) and written
// by consecutive threads: outliers cluster (a stream's jumps fill whole
// bitset words), and a thread's run of single 8-byte stores held the
// window engine's compaction block about 9 us on B200.
// ---------------------------------------------------------------------------
constexpr uint32_t SPAN_CMP_SMEM_IDS = 4096;

struct SpanOut {
  uint32_t* bits;
  int64_t words, chunk, W, S;
  const int64_t* rec_base;  // per-slide output offsets
  int64_t* out_ids;
  int64_t out_cap;
  BatchState* bs;
};

static __global__ void __launch_bounds__(1024) k_span_compact(SpanOut o, int64_t s0) {
  __shared__ uint32_t sm[33];
  __shared__ int64_t s_ids[SPAN_CMP_SMEM_IDS];
  pdl_trigger();
  pdl_wait();
  constexpr int WPT = 4;  // bitset words per thread and step
  const int64_t s = s0 + blockIdx.x;
  uint32_t* row = o.bits + (s % o.chunk) * o.words;
  const int64_t lo = (s + 1) * o.S;
  int64_t out = o.rec_base[s];
  const int64_t step = (int64_t)blockDim.x * WPT;
  for (int64_t c = 0; c < o.words; c += step) {
    const int64_t w0 = c + (int64_t)threadIdx.x * WPT;
    uint32_t bits[WPT];
    uint32_t cnt = 0;
#pragma unroll
    for (int e = 0; e < WPT; ++e) {
      bits[e] = w0 + e < o.words ? row[w0 + e] : 0u;
      cnt += __popc(bits[e]);
    }
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(cnt, &total, sm);
    if (total <= SPAN_CMP_SMEM_IDS && out + total <= o.out_cap) {  // block-uniform
      uint32_t k = ex;
#pragma unroll
      for (int e = 0; e < WPT; ++e) {
        uint32_t b = bits[e];
        if (b) row[w0 + e] = 0;
        while (b) {
          const int f = __ffs(b) - 1;
          b &= b - 1;
          s_ids[k++] = lo + (w0 + e) * 32 + f;
        }
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) o.out_ids[out + i] = s_ids[i];
      __syncthreads();  // s_ids is refilled by the next step
    } else {
      int64_t q = out + ex;
#pragma unroll
      for (int e = 0; e < WPT; ++e) {
        uint32_t b = bits[e];
        if (b) row[w0 + e] = 0;
        while (b) {
          const int f = __ffs(b) - 1;
          b &= b - 1;
          if (q < o.out_cap) o.out_ids[q] = lo + (w0 + e) * 32 + f;
          else set_err(o.bs, DERR_CAPACITY);
          ++q;
        }
      }
    }
    out += total;
  }
}

}  // namespace rtod
