// Exact counts of a group of points that share one stencil, by one warp.
//
// A group is a run of points of one bin in a bin-ordered SoA (positions
// [p, p + nq), coordinates in rows of stride Wp). Whatever cell k of the bin
// a point is in, its stencil cells k + d lie in bins bin + delta(d) (mod NB,
// the bin map being linear in the cell coordinates), so the candidates are
// the same for every point of the group: the (2n+1)^h stencil slots, one bin
// each, taken 32 slots per round; points of other cells sharing those bins
// are rejected by the distance test. This is the grid part of RTOD's range
// count (the ray of each undetermined point against the AABBs of its
// neighbourhood, src/ods/optixScan.cu:158-199): count including self,
// outlier iff count <= K.
//
// The warp keeps up to 32 undecided points (one per lane) and walks the
// candidate list in chunks of 32 * CPL (CPL candidates per lane, held in
// registers); every undecided point is tested against each chunk (CPL tests
// per lane and one warp reduction per point). A point is decided as soon as
// its count exceeds K (inlier), or once it has seen every chunk (outlier iff
// its count <= K). A decided point's lane takes the next point of the group
// at the next chunk boundary, and that point starts its walk at the current
// chunk and wraps around: the count does not depend on the order of the
// chunks, so the warp stays full until the group runs out of points instead
// of rescanning the list for every 32 points. Above 3 dimensions under the
// FP32 predicate the tests run on pairs of candidates with the paired FP32
// instructions (is_nbr_f32x2: the same sums bit for bit), two queries per
// step.
//
// "Sure" slots (can_sure: the bins hold exactly their cells, D <= 3) hold
// cells whose points all lie within R of every point of the group's cell:
// they are counted without tests into `given` (given > K: all inliers; given
// plus every other candidate <= K: all outliers).
#pragma once

#include "kernels.cuh"

namespace rtod {

// Stencil slot s of 2n+1 cells per hashed dimension: offsets d in [-n, n]^h
// (1-d: 0, -1, +1, -2, +2, ..., nearest first; otherwise row-major) and the
// bin offset of the cell k + d (bins are linear in the cell coordinates mod
// NB: d, d1 + 256 d0, d2 + 64 d1 + 4096 d0).
template <int H>
__device__ __forceinline__ int slot_cell(int s, int n, int* d) {
  if constexpr (H == 1) {
    d[0] = (s & 1) ? -((s + 1) >> 1) : (s >> 1);
    return d[0];
  } else {
    const int w = 2 * n + 1;
#pragma unroll
    for (int i = H - 1; i >= 0; --i) {
      d[i] = s % w - n;
      s /= w;
    }
    return H == 2 ? d[1] + 256 * d[0] : d[2] + 64 * d[1] + 4096 * d[0];
  }
}

// Whether every point of cell k + d lies within R of every point of cell k:
// sum of (|d_i| + 1)^2 < n^2 (cells of R(1+2^-12)/n; the margin is at least
// 1/n^2 - 2^-11 of R^2, far above the predicates' rounding).
template <int H>
__device__ __forceinline__ bool slot_sure(const int* d, int n) {
  int q = 0;
#pragma unroll
  for (int i = 0; i < H; ++i) {
    const int a = (d[i] < 0 ? -d[i] : d[i]) + 1;
    q += a * a;
  }
  return q < n * n;
}

// Candidates per lane and chunk, measured on B200: 2 in 1-d (short lists),
// 4 otherwise (3-d sensor-like stream: 3.98 -> 3.42 us per slide against 8;
// 8-d Gaussian blobs: 2 is 35% slower than 4).
template <int D>
struct GroupCpl {
  static constexpr int value = D == 1 ? 2 : 4;
};

struct GroupArgs {
  uint32_t p;      // first position of the group
  uint32_t nq;     // points in the group
  uint32_t bin;    // the group's bin
  int n;           // cells per R
  int K;
  float R2f;
  double R, R2;
  int64_t Wp;      // row stride of the coordinates
  bool can_sure;
  unsigned long long* tests;  // distance tests made, added once per group (may be null)
};

// Bounds of a count: [lo, hi], hi = CNT_INF when only a lower bound is known.
constexpr int32_t CNT_INF = 1 << 29;

// Counts the group; range(sb, rs, len) gives the candidate positions of
// stencil bin sb, mark(pos) records an outlier (called by one lane per
// outlier). pick(i) is the position of the group's i-th point (i < a.nq) and
// rec(pos, lo, hi) receives bounds of each point's count (exact when equal:
// the outliers; inliers get lo > K and hi = CNT_INF); *made (may be null)
// receives the distance tests made. Returns the number of outliers (the
// same on every lane).
template <int D, int PRED, typename T, class Range, class Mark, class Pick, class Rec>
__device__ __forceinline__ int count_group_ex(const T* sx, const GroupArgs& a, Range range, Mark mark, Pick pick,
                                              Rec rec, unsigned long long* made = nullptr) {
  if (made) *made = 0;
  constexpr int H = Hashed<D>::value;
  constexpr int CPL = GroupCpl<D>::value;
  constexpr uint32_t CHUNK = 32 * CPL;
  const int lane = threadIdx.x & 31;
  const int w = 2 * a.n + 1;
  const int slots = H == 1 ? w : (H == 2 ? w * w : w * w * w);
  const int rounds = (slots + 31) >> 5;
  auto slot = [&](int s, uint32_t& rs, uint32_t& len, bool& sure) {
    rs = 0;
    len = 0;
    sure = false;
    if (s >= slots) return;
    int d[3] = {0, 0, 0};
    const int delta = slot_cell<H>(s, a.n, d);
    sure = a.can_sure && slot_sure<H>(d, a.n);
    range((a.bin + (uint32_t)delta) & NB_MASK, rs, len);
  };
  // Pass over the rounds: sure count, all candidates, chunks of the others.
  uint32_t given = 0, total = 0, nchunks = 0, rs1 = 0, len1 = 0;
  for (int r = 0; r < rounds; ++r) {
    uint32_t rs, len;
    bool sure;
    slot(32 * r + lane, rs, len, sure);
    const uint32_t s_len = __reduce_add_sync(0xffffffffu, sure ? len : 0u);
    const uint32_t o_len = __reduce_add_sync(0xffffffffu, sure ? 0u : len);
    given += s_len;
    total += s_len + o_len;
    nchunks += (o_len + CHUNK - 1) / CHUNK;
    rs1 = rs;
    len1 = sure ? 0u : len;
  }
  if (given > (uint32_t)a.K) {  // every point of the group is an inlier
    for (uint32_t q = lane; q < a.nq; q += 32) rec(pick(q), (int)given, CNT_INF);
    return 0;
  }
  if (total <= (uint32_t)a.K) {  // every point of the group is an outlier
    for (uint32_t q = lane; q < a.nq; q += 32) {
      mark(pick(q));
      rec(pick(q), 1, (int)total);
    }
    return (int)a.nq;
  }
  // Current round: per-lane range, exclusive offset of the lane's range in
  // the round's virtual candidate list, and the list's length.
  uint32_t rs = rs1, len = len1, off = 0, ncand = 0;
  auto enter = [&](int r) {
    if (rounds > 1) {
      bool sure;
      slot(32 * r + lane, rs, len, sure);
      if (sure) len = 0;
    }
    uint32_t inc = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    off = inc - len;
    ncand = __shfl_sync(0xffffffffu, inc, 31);
  };
  int r = 0;
  enter(0);
  for (int t = 1; t < rounds && ncand == 0; ++t) {  // nchunks > 0: some round has candidates
    r = t;
    enter(r);
  }
  if (ncand == 0) return 0;
  uint32_t c0 = 0, next = 0, left = 0, mine = 0;
  bool has = false;
  int cnt = 0, nout = 0;
  unsigned long long tests = 0;  // warp-uniform: live points x candidates of each chunk
  T qx[D];
#pragma unroll
  for (int d = 0; d < D; ++d) qx[d] = T(0);
  while (true) {
    // idle lanes take the next points of the group
    const unsigned empty = __ballot_sync(0xffffffffu, !has);
    if (empty && next < a.nq) {
      const uint32_t rank = (uint32_t)__popc(empty & lanemask_lt());
      if (!has && next + rank < a.nq) {
        mine = pick(next + rank);
#pragma unroll
        for (int d = 0; d < D; ++d) qx[d] = sx[(int64_t)d * a.Wp + mine];
        cnt = (int)given;
        left = nchunks;
        has = true;
      }
      next = min(a.nq, next + (uint32_t)__popc(empty));
    }
    const unsigned live = __ballot_sync(0xffffffffu, has);
    if (!live) break;
    // the chunk [c0, c0 + CHUNK) of the round's list, CPL candidates per lane
    T cx[CPL][D];
    bool cv[CPL];
#pragma unroll
    for (int e = 0; e < CPL; ++e) {
      const uint32_t v = c0 + 32 * e + lane;
      // lane holding v's range: the last lane whose offset is <= v
      int s = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int cand = s + step;
        const uint32_t oc = __shfl_sync(0xffffffffu, off, cand & 31);
        if (oc <= v) s = cand;
      }
      const uint32_t base = __shfl_sync(0xffffffffu, rs, s);
      const uint32_t os = __shfl_sync(0xffffffffu, off, s);
      cv[e] = v < ncand;
      const uint32_t c = base + (v - os);
#pragma unroll
      for (int d = 0; d < D; ++d) cx[e][d] = cv[e] ? sx[(int64_t)d * a.Wp + c] : T(0);
    }
    tests += (unsigned long long)__popc(live) * min(CHUNK, ncand - c0);
    // Above 3 dimensions the FP32 test dominates: candidates in pairs for
    // the paired FP32 instructions (half the arithmetic instructions, the
    // same sums bit for bit).
    constexpr bool PAIRED = PRED == 0 && D > 3 && CPL % 2 == 0 && sizeof(T) == sizeof(float);
    unsigned long long cp[PAIRED ? CPL / 2 : 1][PAIRED ? D : 1];
    if constexpr (PAIRED) {
#pragma unroll
      for (int e = 0; e < CPL / 2; ++e)
#pragma unroll
        for (int d = 0; d < D; ++d) cp[e][d] = f2_pack((float)cx[2 * e][d], (float)cx[2 * e + 1][d]);
    }
    unsigned todo = live;
    if constexpr (PAIRED) {
      // two queries per step: four independent chains of paired
      // instructions per lane (a lone last query is tested twice, the second
      // result dropped)
      while (todo) {
        const int qa = __ffs(todo) - 1;
        todo &= todo - 1;
        const int qb = todo ? __ffs(todo) - 1 : -1;
        todo &= todo - 1;
        const int qs = qb >= 0 ? qb : qa;
        unsigned long long ya[D], yb[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const float va = (float)__shfl_sync(0xffffffffu, qx[d], qa);
          const float vb = (float)__shfl_sync(0xffffffffu, qx[d], qs);
          ya[d] = f2_pack(va, va);
          yb[d] = f2_pack(vb, vb);
        }
        unsigned ma = 0, mb = 0;
#pragma unroll
        for (int e = 0; e < CPL / 2; ++e) {
          bool a0, a1, b0, b1;
          is_nbr_f32x2<D>(ya, cp[e], a.R2f, a0, a1);
          is_nbr_f32x2<D>(yb, cp[e], a.R2f, b0, b1);
          ma += (cv[2 * e] && a0 ? 1u : 0u) + (cv[2 * e + 1] && a1 ? 1u : 0u);
          mb += (cv[2 * e] && b0 ? 1u : 0u) + (cv[2 * e + 1] && b1 ? 1u : 0u);
        }
        const unsigned ta = __reduce_add_sync(0xffffffffu, ma);
        const unsigned tb = __reduce_add_sync(0xffffffffu, mb);
        if (lane == qa) cnt += (int)ta;
        if (lane == qb) cnt += (int)tb;
      }
    } else {
      while (todo) {
        const int qq = __ffs(todo) - 1;
        todo &= todo - 1;
        T y[D];
#pragma unroll
        for (int d = 0; d < D; ++d) y[d] = __shfl_sync(0xffffffffu, qx[d], qq);
        unsigned m = 0;
#pragma unroll
        for (int e = 0; e < CPL; ++e) m += (cv[e] && is_nbr<D, PRED, T>(y, cx[e], a.R2f, a.R, a.R2)) ? 1u : 0u;
        const unsigned tot = __reduce_add_sync(0xffffffffu, m);
        if (lane == qq) cnt += (int)tot;
      }
    }
    bool out = false;
    if (has) {
      --left;
      if (cnt > a.K) {
        rec(mine, cnt, CNT_INF);
        has = false;
      } else if (left == 0) {
        rec(mine, cnt, cnt);
        out = true;
        has = false;
      }
    }
    if (out) mark(mine);
    nout += __popc(__ballot_sync(0xffffffffu, out));
    // next chunk, wrapping around the rounds
    c0 += CHUNK;
    if (c0 >= ncand) {
      c0 = 0;
      if (rounds > 1) {
        for (int t = 0; t < rounds; ++t) {  // the next round with candidates
          r = (r + 1) % rounds;
          enter(r);
          if (ncand) break;
        }
      }
    }
  }
  if (a.tests && lane == 0 && tests) atomicAdd(a.tests, tests);
  if (made) *made = tests;
  return nout;
}

// count_group_ex over the contiguous positions [a.p, a.p + a.nq), no bounds kept.
template <int D, int PRED, typename T, class Range, class Mark>
__device__ __forceinline__ int count_group(const T* sx, const GroupArgs& a, Range range, Mark mark) {
  return count_group_ex<D, PRED, T>(
      sx, a, range, mark, [&](uint32_t i) { return a.p + i; }, [](uint32_t, int, int) {});
}

}  // namespace rtod
