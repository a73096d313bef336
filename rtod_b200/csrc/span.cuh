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
__device__ __forceinline__ void span_count_group(const Batch& b, const Span& sp, uint32_t p, uint32_t nq,
                                                 uint32_t bin, const WinPre& wp, bool pure) {
  const int j = wp.j;
  const Job& jb = b.jobs[j];
  const int64_t shift = (int64_t)j * sp.S;  // window offset = span offset - shift
  uint32_t* row = sp.bits + ((jb.ctr->lo - sp.S) / sp.S % sp.chunk) * sp.words;
  const GroupArgs ga{p, nq, bin, sp.n, sp.K, sp.R2f, sp.R, sp.R2, sp.Wp, pure && D <= 3, &b.bs->pair_tests};
  const int nout = count_group<D, PRED, T>(
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
      });
  if ((threadIdx.x & 31) == 0 && nout) atomicAdd(&jb.ctr->n_out, nout);
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
// mostly the same candidates.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(256) k_span_classify(Batch b, Span sp) {
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
    const unsigned nmask = __ballot_sync(0xffffffffu, need);
    uint32_t gbase = 0;
    if (lane == 0 && nmask) gbase = atomicAdd(&sp.sc->n_groups, (uint32_t)__popc(nmask));
    gbase = __shfl_sync(0xffffffffu, gbase, 0);
    const unsigned peers = __match_any_sync(0xffffffffu, need ? j : -1);
    if (need) {
      sp.groups[gbase + __popc(nmask & lanemask_lt())] = make_uint4(start, wc, bin, (uint32_t)j);
      const uint32_t pts = __reduce_add_sync(peers, wc);
      if (lane == __ffs(peers) - 1) atomicAdd(&b.jobs[j].ctr->n_undet, (int)pts);
    }
  }
}

// ---------------------------------------------------------------------------
// k_span_count: one warp per listed group of the batch, groups taken in list
// order by ticket (one atomic per group), so that a warp that drew short
// groups takes more of them and no warp idles while long groups remain.
// Outliers set their bit in the slide's bitset row. Then the blocks clear the
// per-bin state, and the block that finishes last ends the batch (records,
// window advance, counters).
// ---------------------------------------------------------------------------
template <int D, int PRED, typename T>
__global__ void __launch_bounds__(256) k_span_count(Batch b, Span sp) {
  __shared__ int s_last;
  pdl_trigger();
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const uint32_t ng = sp.sc->n_groups;
  const bool pure = sp.sc->pure;
  while (true) {
    uint32_t k = 0;
    if (lane == 0) k = atomicAdd(&sp.sc->count_ticket, 1u);
    k = __shfl_sync(0xffffffffu, k, 0);
    if (k >= ng) break;
    const uint4 g = sp.groups[k];
    const int j = (int)g.w;
    span_count_group<D, PRED, T>(b, sp, g.x, g.y, g.z, WinPre{sp.pre, sp.ts, j, sp.wblk}, pure);
  }
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
// thread, one block scan per 4096 words) and clears the row.
// ---------------------------------------------------------------------------
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
    out += total;
  }
}

}  // namespace rtod
