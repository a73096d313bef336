// CPU oracle for the sliding-window distance outlier detector.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: the test suite, the
// smoke check and bench.py's CPU-baseline / reference arm load it. The
// product library (rtod_b200/librtod.so) never links, loads or calls it.
//
// Parity status: pinned to RTOD's own code. RTOD ships no tests, golden
// vectors or data files, and its GPU path needs OptiX and RT cores; but its
// host code (src/ods/optixScan.cpp: the slide loop, FixQueue grid filter,
// outlier pick and the brute-force check_outlier) compiles unmodified here
// (oracle/ref/Makefile, with the OptiX programs and AABB kernel restated on
// the host in oracle/ref/ref_fakes.cpp). Its per-slide outliers on seeded
// 1-d and 3-d streams are committed as tests/golden/ref_*.npz, and this
// file's double mode (PRED_F64_LT on double storage) reproduces them on
// every slide (tests/test_reference_pin.py). Further pins: hand-derived
// known-answer cases and numpy brute-force fixtures in tests/golden/, and
// the agreement of this file's two engines with each other.
//
// What is restated, and from where (paths relative to the RTOD project):
//  * Slide schedule and ring order: src/ods/optixScan.cpp:1019-1126. The
//    first W points fill the window, each slide expires the oldest S and
//    inserts the next S, the first detected window is [S, W+S), slide j
//    detects [(j+1)S, W+(j+1)S), and the loop runs while at least S points
//    remain (at most 10000 slides by default, :1045).
//  * Outlier rule: src/ods/optixScan.cu:158-199 and
//    src/ods/optixScan.cpp:1095-1099. The neighbour count includes the
//    point itself and a point is an outlier iff count <= K; counting stops
//    once count > K (the `count > K` skip at optixScan.cu:161).
//  * Grid filter: src/ods/optixScan.cpp:947-1017 with FixQueue from
//    src/ods/state.h:15-57. Cells of side R/sqrt(D) keyed from the global
//    per-dimension minimum (:950-955, :960-965); expire S points then insert
//    S points (:969-981); cells holding more than K points are all-inlier,
//    the rest are "undetermined" (:987-993) and their points get an exact
//    count.
//  * Brute force: check_outlier, src/ods/optixScan.cpp:817-881.
//
// Deliberate differences (none changes a result):
//  * Predicate. PRED_FP32_LE (default): dx_i = fl32(p_i - q_i),
//    d2 = fl32(...fl32(fl32(dx_0^2) + fl32(dx_1^2))... + fl32(dx_{d-1}^2))
//    summed left to right without FMA, neighbour iff d2 <= fl32(Rf*Rf) with
//    Rf = fl32(R). PRED_F64_LT restates RTOD's own double test
//    (optixScan.cu:170-190): |dx| < R in 1-d, dx^2+dy^2+... < R*R otherwise.
//  * Cell side is R/sqrt(D)*(1-2^-16) instead of R/sqrt(D), so that "more
//    than K points in a cell" provably implies "inlier" under both
//    predicates (the unshrunk cell's diagonal equals R exactly and FP32
//    rounding can push a same-cell pair past R^2). Results do not depend on
//    the cell side; only the set of skipped points does.
//  * A cell keeps all of its live points (a FIFO), not only the newest MK,
//    because the exact count here walks neighbouring cells instead of a BVH.
//  * Dimensions beyond 3 (d = 8): cells are formed on the first three
//    dimensions and no cell is all-inlier (a 3-d cell does not bound the
//    other dimensions).
//  * Output: per slide the sorted global stream indices of the outliers
//    (RTOD prints ring slots; slot = index mod W).
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off, no fast-math).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

enum { PRED_FP32_LE = 0, PRED_F64_LT = 1 };
enum { ENGINE_BRUTE = 0, ENGINE_GRID = 1 };

struct Pred {
  int dim;
  int mode;
  double R;
  double R2;   // R*R in double (optixScan.cpp:714)
  float R2f;   // fl32(fl32(R)^2)

  Pred(int d, int m, double r) : dim(d), mode(m), R(r), R2(r * r) {
    float rf = (float)r;
    R2f = rf * rf;
  }

  // Neighbour test between two points stored point-major (d coordinates
  // each, float or double; the FP32 predicate is only used with float).
  template <typename T>
  inline bool operator()(const T* p, const T* q) const {
    if (mode == PRED_FP32_LE) {
      float s = 0.0f;
      for (int i = 0; i < dim; ++i) {
        float dx = (float)p[i] - (float)q[i];
        float t = dx * dx;
        s = (i == 0) ? t : s + t;
        if (s > R2f) return false;  // partial sums never decrease
      }
      return s <= R2f;
    } else {
      if (dim == 1) {
        double dx = (double)p[0] - (double)q[0];
        return std::fabs(dx) < R;
      }
      double s = 0.0;
      for (int i = 0; i < dim; ++i) {
        double dx = (double)p[i] - (double)q[i];
        double t = dx * dx;
        s = (i == 0) ? t : s + t;
      }
      return s < R2;
    }
  }
};

template <typename T>
struct Stream {
  const T* pts;
  int64_t n;
  int dim;
  int64_t W, S;
  int K;
  Pred pred;
  const T* at(int64_t g) const { return pts + g * dim; }
};

// Brute-force count of window [lo, lo+W) neighbours of point g, stopping once
// the count exceeds `cap` (check_outlier, optixScan.cpp:820-833).
template <typename T>
int count_brute(const Stream<T>& s, int64_t lo, int64_t g, int cap, uint64_t* tests) {
  int c = 0;
  const T* p = s.at(g);
  for (int64_t q = lo; q < lo + s.W; ++q) {
    ++*tests;
    if (s.pred(p, s.at(q))) {
      if (++c > cap) break;
    }
  }
  return c;
}

// Grid filter state: a restatement of ScanState::cell_queue plus FixQueue.
template <typename T>
struct Grid {
  const Stream<T>& s;
  int hd;                 // hashed dimensions (min(d, 3))
  double cell;            // cell side
  double mn[3];           // global per-dim minimum (read_data, optixScan.cpp:104-146)
  int64_t cnt[3];         // cells per dim (initialize_cell, optixScan.cpp:960-965)
  bool safe_enabled;      // "num > K means all inlier" (optixScan.cpp:988)
  int reach;              // neighbour-cell reach (cells) of the exact count
  std::unordered_map<int64_t, std::deque<int64_t>> cells;

  Grid(const Stream<T>& st, bool filter) : s(st) {
    hd = s.dim < 3 ? s.dim : 3;
    cell = s.pred.R / std::sqrt((double)hd) * (1.0 - std::ldexp(1.0, -16));
    double mx[3];
    for (int i = 0; i < hd; ++i) { mn[i] = INFINITY; mx[i] = -INFINITY; }
    for (int64_t g = 0; g < s.n; ++g)
      for (int i = 0; i < hd; ++i) {
        double v = s.at(g)[i];
        mn[i] = std::min(mn[i], v);
        mx[i] = std::max(mx[i], v);
      }
    for (int i = 0; i < hd; ++i) cnt[i] = (int64_t)((mx[i] - mn[i] + cell) / cell) + 1;
    safe_enabled = filter && s.dim <= 3;
    // Any neighbour pair differs by at most R*(1+2^-22) per dimension.
    reach = (int)std::ceil(s.pred.R * (1.0 + std::ldexp(1.0, -22)) / cell);
  }

  void coords(int64_t g, int64_t* c) const {
    for (int i = 0; i < hd; ++i) c[i] = (int64_t)std::floor(((double)s.at(g)[i] - mn[i]) / cell);
  }
  int64_t linear(const int64_t* c) const {
    int64_t id = 0;
    for (int i = 0; i < hd; ++i) id = id * cnt[i] + c[i];
    return id;
  }
  int64_t cell_of(int64_t g) const {
    int64_t c[3];
    coords(g, c);
    return linear(c);
  }
  void insert(int64_t g) { cells[cell_of(g)].push_back(g); }
  void expire(int64_t g) {
    auto it = cells.find(cell_of(g));
    // FIFO per cell: the expiring point is the oldest one of its cell.
    it->second.pop_front();
    if (it->second.empty()) cells.erase(it);
  }

  // Exact count of g's neighbours in the current window, capped at K+1.
  int count(int64_t g, uint64_t* tests) const {
    int64_t c[3], o[3] = {0, 0, 0};
    coords(g, c);
    const T* p = s.at(g);
    int n = 0;
    int span = 2 * reach + 1;
    int total = 1;
    for (int i = 0; i < hd; ++i) total *= span;
    for (int t = 0; t < total; ++t) {
      int r = t;
      bool ok = true;
      for (int i = hd - 1; i >= 0; --i) {
        o[i] = c[i] + (r % span) - reach;
        r /= span;
        if (o[i] < 0 || o[i] >= cnt[i]) ok = false;
      }
      if (!ok) continue;
      auto it = cells.find(linear(o));
      if (it == cells.end()) continue;
      for (int64_t q : it->second) {
        ++*tests;
        if (s.pred(p, s.at(q))) {
          if (++n > s.K) return n;
        }
      }
    }
    return n;
  }
};

struct SlideOut {
  std::vector<int64_t> ids;
  int64_t undetermined = 0;
};

template <typename T>
void run_brute(const Stream<T>& s, int64_t j0, int64_t j1, std::vector<SlideOut>& out, uint64_t* tests) {
  for (int64_t j = j0; j < j1; ++j) {
    int64_t lo = (j + 1) * s.S;
    SlideOut& so = out[j];
    so.undetermined = s.W;
    for (int64_t g = lo; g < lo + s.W; ++g)
      if (count_brute(s, lo, g, s.K, tests) <= s.K) so.ids.push_back(g);
  }
}

template <typename T>
void run_grid(const Stream<T>& s, bool filter, int64_t j0, int64_t j1, std::vector<SlideOut>& out,
              uint64_t* tests) {
  if (j0 >= j1) return;
  Grid<T> grid(s, filter);
  // Window before slide j0 (detect_outlier's initial fill, optixScan.cpp:1029-1033).
  for (int64_t g = j0 * s.S; g < j0 * s.S + s.W; ++g) grid.insert(g);
  std::vector<int64_t> undet;
  for (int64_t j = j0; j < j1; ++j) {
    int64_t left = j * s.S, right = s.W + j * s.S;
    for (int64_t g = left; g < left + s.S; ++g) grid.expire(g);    // :969-976
    for (int64_t g = right; g < right + s.S; ++g) grid.insert(g);  // :978-981
    undet.clear();
    for (auto& kv : grid.cells) {                                  // :987-993
      if (grid.safe_enabled && (int64_t)kv.second.size() > s.K) continue;
      for (int64_t g : kv.second) undet.push_back(g);
    }
    SlideOut& so = out[j];
    so.undetermined = (int64_t)undet.size();
    for (int64_t g : undet)
      if (grid.count(g, tests) <= s.K) so.ids.push_back(g);  // :1095-1099
    std::sort(so.ids.begin(), so.ids.end());
  }
}

template <typename T>
bool finite_all(const T* p, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// Processes a whole stream the way detect_outlier does and writes, per slide,
// the sorted global indices of the outliers in CSR form.
//   pts          n points, point-major (n * dim coordinates)
//   engine       0 brute force, 1 grid filter (opt >= 1) , 2 grid without the
//                all-inlier filter (opt 0)
//   threads      >= 1; slides are split into contiguous ranges, one per thread
//   out_offsets  [n_slides + 1]
//   stats        [3]: undetermined points (sum over slides), pair tests, slides
// Returns the number of slides (>= 0) or a negative error:
//   -1 bad config, -2 output capacity, -5 non-finite input.
template <typename T>
int64_t detect_impl(const T* pts, int64_t n, int32_t dim, int64_t W, int64_t S, double R, int32_t K,
                    int32_t pred, int32_t engine, int32_t threads, int64_t max_slides, int64_t* out_offsets,
                    int64_t* out_ids, int64_t ids_cap, int64_t* stats) {
  if (dim < 1 || dim > 8 || W < 1 || S < 1 || S > W || W % S != 0 || !(R > 0) || K < 0 ||
      (pred != PRED_FP32_LE && pred != PRED_F64_LT) || engine < 0 || engine > 2 || n < 0)
    return -1;
  if (!finite_all(pts, n * dim)) return -5;
  int64_t slides = n >= W ? (n - W) / S : 0;
  if (max_slides >= 0 && slides > max_slides) slides = max_slides;
  Stream<T> s{pts, n, dim, W, S, K, Pred(dim, pred, R)};
  std::vector<SlideOut> out((size_t)slides);
  if (threads < 1) threads = 1;
  if (threads > slides) threads = (int)std::max<int64_t>(1, slides);
  std::vector<uint64_t> tests((size_t)threads, 0);
  auto work = [&](int t) {
    int64_t j0 = slides * t / threads, j1 = slides * (t + 1) / threads;
    if (engine == ENGINE_BRUTE)
      run_brute(s, j0, j1, out, &tests[t]);
    else
      run_grid(s, engine == 1, j0, j1, out, &tests[t]);
  };
  if (threads == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  }
  int64_t total = 0, undet = 0;
  uint64_t nt = 0;
  for (auto v : tests) nt += v;
  out_offsets[0] = 0;
  for (int64_t j = 0; j < slides; ++j) {
    const auto& ids = out[j].ids;
    if (total + (int64_t)ids.size() > ids_cap) return -2;
    std::memcpy(out_ids + total, ids.data(), ids.size() * sizeof(int64_t));
    total += (int64_t)ids.size();
    out_offsets[j + 1] = total;
    undet += out[j].undetermined;
  }
  if (stats) {
    stats[0] = undet;
    stats[1] = (int64_t)nt;
    stats[2] = slides;
  }
  return slides;
}

}  // namespace

extern "C" {

// detect_impl on float coordinates.
int64_t oracle_detect(const float* pts, int64_t n, int32_t dim, int64_t W, int64_t S, double R,
                      int32_t K, int32_t pred, int32_t engine, int32_t threads, int64_t max_slides,
                      int64_t* out_offsets, int64_t* out_ids, int64_t ids_cap, int64_t* stats) {
  return detect_impl(pts, n, dim, W, S, R, K, pred, engine, threads, max_slides, out_offsets, out_ids, ids_cap,
                     stats);
}

// The same on double coordinates (RTOD stores double3 points,
// src/ods/optixScan.cpp:95-147), with RTOD's double predicate only
// (pred must be 1).
int64_t oracle_detect_f64(const double* pts, int64_t n, int32_t dim, int64_t W, int64_t S, double R,
                          int32_t K, int32_t pred, int32_t engine, int32_t threads, int64_t max_slides,
                          int64_t* out_offsets, int64_t* out_ids, int64_t ids_cap, int64_t* stats) {
  if (pred != PRED_F64_LT) return -1;
  return detect_impl(pts, n, dim, W, S, R, K, pred, engine, threads, max_slides, out_offsets, out_ids, ids_cap,
                     stats);
}

// Uncapped neighbour counts (self included) of every point of the window
// [lo, lo+W) against that window, by brute force. counts[i] is point lo+i.
int32_t oracle_window_counts(const float* pts, int64_t n, int32_t dim, int64_t lo, int64_t W,
                             double R, int32_t pred, int32_t* counts) {
  if (dim < 1 || dim > 8 || lo < 0 || W < 1 || lo + W > n || !(R > 0)) return -1;
  Stream<float> s{pts, n, dim, W, W, 0, Pred(dim, pred, R)};
  for (int64_t i = 0; i < W; ++i) {
    int c = 0;
    const float* p = s.at(lo + i);
    for (int64_t q = lo; q < lo + W; ++q) c += s.pred(p, s.at(q));
    counts[i] = c;
  }
  return 0;
}

// The predicate itself, for known-answer tests.
int32_t oracle_pred(const float* p, const float* q, int32_t dim, double R, int32_t pred) {
  return Pred(dim, pred, R)(p, q) ? 1 : 0;
}

// RTOD's double predicate on double coordinates.
int32_t oracle_pred_f64(const double* p, const double* q, int32_t dim, double R) {
  return Pred(dim, PRED_F64_LT, R)(p, q) ? 1 : 0;
}

}  // extern "C"
