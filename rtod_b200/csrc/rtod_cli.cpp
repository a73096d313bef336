// rtod: native command line with the run surface of RTOD's optixScan,
// calling the detector only through the C ABI of include/rtod.h.
//
//   rtod --n 1048572 --R 0.45 --K 50 --window 100000 --slide 5000 -f stock.txt
//
// Flags follow RTOD's parse_args (src/ods/optixScan.cpp:149-212): --file/-f,
// --n, --window, --slide, --R, --K, --start_copy_pos, --launch_ray_num
// (accepted; it only sizes RTOD's OPTIMIZATION=0 ray launch). RTOD's
// compile-time switches are flags: --dim (DIMENSION, optixScan.h:10-12) and
// --opt (OPTIMIZATION, optixScan.h:22-24). Further flags: --coord f32|f64
// (f64 keeps RTOD's doubles and its double predicate end to end), --pred
// fp32_le|f64_lt, --router, --tuner, --no-graph, --warmup N (RTOD: 10),
// --max-slides N, --device N, --print-outliers, --engine auto|window|grid,
// and --streaming: RTOD's own per-slide loop (detect_outlier,
// optixScan.cpp:1045-1121) through rtod_push_slide + rtod_detect, one
// window per call, timed on the host clock per slide (the last warm-up
// slides excluded); the report then gives the median and mean wall time of a
// slide and the device stage split of the timed slides.
//
// Input is read like read_data (optixScan.cpp:95-147): %lf per line in 1-d,
// comma-separated values otherwise, parsed as doubles. Timing follows main()
// (optixScan.cpp:1159-1168): warm-up passes over the whole stream, then one
// timed pass. The report mirrors RTOD's stdout: DIM[i] lines, the common info
// block (:934-945), the [Time] block (src/ods/timer.h:102-117), [Mem] lines
// and "BVH Node / slide" (:1168-1186). The stage split of a graph-replayed
// pass comes from rtod_profile_run on the same handle (every kernel
// launched on its own with events) and is labelled as such.
//
// Exit status: 0 on success, 1 on bad usage or input, 2 when a library call
// fails (its message from rtod_last_error on stderr).
#include <sys/resource.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rtod.h"

namespace {

struct Args {
  std::string file;
  int64_t n = 100000000;
  int64_t window = -1, slide = -1;
  double R = -1;
  int K = -1;
  int64_t start_copy_pos = 0;
  int dim = 1, opt = 2, warmup = 10, device = 0;
  int64_t max_slides = 10000;
  bool f64 = false, router = false, tuner = false, graph = true, print = false, streaming = false;
  int pred = -1;
  int engine = RTOD_ENGINE_AUTO;
};

void usage(const char* argv0) {
  std::fprintf(stderr,
               "Usage  : %s [options]\n"
               "Options: --file | -f <filename>      Specify file for data input\n"
               "         --n <int>                   Set data num; defaults to 1e8\n"
               "         --window <int> --slide <int> --R <float> --K <int>\n"
               "         --start_copy_pos <int> --launch_ray_num <int>\n"
               "         --dim <1..8> --opt <0|1|2> --coord <f32|f64> --pred <fp32_le|f64_lt>\n"
               "         --router --tuner --no-graph --warmup <int> --max-slides <int> --device <int>\n"
               "         --print-outliers --streaming --engine <auto|window|grid>\n",
               argv0);
  std::exit(1);
}

bool parse(int argc, char** argv, Args* a) {
  for (int i = 1; i < argc; ++i) {
    const std::string s = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) usage(argv[0]);
      return argv[++i];
    };
    if (s == "--help" || s == "-h") usage(argv[0]);
    else if (s == "--file" || s == "-f") a->file = next();
    else if (s == "--n") a->n = std::atoll(next());
    else if (s == "--window") a->window = std::atoll(next());
    else if (s == "--slide") a->slide = std::atoll(next());
    else if (s == "--R") a->R = std::atof(next());
    else if (s == "--K") a->K = std::atoi(next());
    else if (s == "--start_copy_pos") a->start_copy_pos = std::atoll(next());
    else if (s == "--launch_ray_num") (void)next();
    else if (s == "--dim") a->dim = std::atoi(next());
    else if (s == "--opt") a->opt = std::atoi(next());
    else if (s == "--coord") {
      const std::string v = next();
      if (v != "f32" && v != "f64") usage(argv[0]);
      a->f64 = v == "f64";
    } else if (s == "--pred") {
      const std::string v = next();
      if (v == "fp32_le") a->pred = RTOD_PRED_FP32_LE;
      else if (v == "f64_lt") a->pred = RTOD_PRED_F64_LT;
      else usage(argv[0]);
    } else if (s == "--router") a->router = true;
    else if (s == "--tuner") a->tuner = true;
    else if (s == "--no-graph") a->graph = false;
    else if (s == "--warmup") a->warmup = std::atoi(next());
    else if (s == "--max-slides") a->max_slides = std::atoll(next());
    else if (s == "--device") a->device = std::atoi(next());
    else if (s == "--print-outliers") a->print = true;
    else if (s == "--streaming") a->streaming = true;
    else if (s == "--engine") {
      const std::string v = next();
      if (v == "auto") a->engine = RTOD_ENGINE_AUTO;
      else if (v == "window") a->engine = RTOD_ENGINE_WINDOW;
      else if (v == "grid") a->engine = RTOD_ENGINE_GRID;
      else usage(argv[0]);
    }
    else {
      std::fprintf(stderr, "Unknown option '%s'\n", s.c_str());
      usage(argv[0]);
    }
  }
  if (a->file.empty() || a->window < 1 || a->slide < 1 || !(a->R > 0) || a->K < 0) {
    std::fprintf(stderr, "need --file, --window, --slide, --R and --K\n");
    return false;
  }
  if (a->pred < 0) a->pred = a->f64 ? RTOD_PRED_F64_LT : RTOD_PRED_FP32_LE;
  return true;
}

// Up to n rows of `dim` doubles: one value per line in 1-d, comma-separated
// otherwise (RTOD's %lf / %lf,%lf,%lf).
bool read_text(const std::string& path, int64_t n, int dim, std::vector<double>* out) {
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) {
    std::fprintf(stderr, "Fail to open [%s]!\n", path.c_str());
    return false;
  }
  char line[4096];
  out->clear();
  for (int64_t r = 0; r < n && std::fgets(line, sizeof line, f); ++r) {
    char* p = line;
    for (int d = 0; d < dim; ++d) {
      char* end = nullptr;
      const double v = std::strtod(p, &end);
      if (end == p) {
        std::fprintf(stderr, "%s: row %lld has fewer than %d values\n", path.c_str(), (long long)r, dim);
        std::fclose(f);
        return false;
      }
      out->push_back(v);
      p = end;
      while (*p == ',' || *p == ' ' || *p == '\t') ++p;
    }
  }
  std::fclose(f);
  return true;
}

int lib_fail(const char* what) {
  std::fprintf(stderr, "%s failed: %s\n", what, rtod_last_error());
  return 2;
}

long rss_kb() {
  struct rusage u;
  getrusage(RUSAGE_SELF, &u);
  return u.ru_maxrss;
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  if (!parse(argc, argv, &a)) return 1;
  std::vector<double> rows;
  if (!read_text(a.file, a.n, a.dim, &rows)) return 1;
  const int D = a.dim;
  int64_t n = (int64_t)rows.size() / D;
  for (int d = 0; d < D; ++d) {
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t i = 0; i < n; ++i) {
      lo = std::fmin(lo, rows[(size_t)(i * D + d)]);
      hi = std::fmax(hi, rows[(size_t)(i * D + d)]);
    }
    std::printf("DIM[%d]: %g, %g\n", d, lo, hi);
  }
  const int64_t skip = std::min<int64_t>(n, a.start_copy_pos * a.slide);
  n -= skip;
  std::vector<float> rows32;
  if (!a.f64) {
    rows32.resize((size_t)(n * D));
    for (int64_t i = 0; i < n * D; ++i) rows32[(size_t)i] = (float)rows[(size_t)(skip * D + i)];
  }
  const double* p64 = rows.data() + skip * D;

  rtod_config cfg;
  rtod_config_init(&cfg);
  cfg.window = a.window;
  cfg.slide = a.slide;
  cfg.R = a.R;
  cfg.K = a.K;
  cfg.dim = D;
  cfg.opt = a.opt;
  cfg.pred = a.pred;
  cfg.coord = a.f64 ? RTOD_COORD_F64 : RTOD_COORD_F32;
  cfg.router = a.router;
  cfg.tuner = a.tuner;
  cfg.use_graph = a.graph;
  cfg.device = a.device;
  cfg.engine = a.engine;
  const long rss0 = rss_kb();
  rtod_handle* h = nullptr;
  if (rtod_create(&cfg, &h) != RTOD_OK) return lib_fail("rtod_create");

  std::printf("Dimension: %d\n", D);
  std::printf("data num: %lld\n", (long long)n);
  std::printf("R: %g, R2: %g\n", a.R, a.R * a.R);
  std::printf("K: %d\n", a.K);
  std::printf("Window size: %lld\n", (long long)a.window);
  std::printf("Slide size: %lld\n", (long long)a.slide);
  std::printf("Input file: %s\n", a.file.c_str());
  std::printf("Optimization: %d\n", a.opt);

  const int64_t slides_max = n >= a.window ? std::min<int64_t>((n - a.window) / a.slide, a.max_slides) : 0;
  std::vector<int64_t> offsets((size_t)slides_max + 1, 0), ids((size_t)std::max<int64_t>(1, slides_max * a.window));
  int64_t slides = 0;
  rtod_times t{};
  auto pass = [&](rtod_times* tp) -> int {
    if (rtod_reset(h) != RTOD_OK) return lib_fail("rtod_reset");
    const int rc = a.f64 ? rtod_run_f64(h, p64, n, a.max_slides, offsets.data(), ids.data(), (int64_t)ids.size(),
                                        &slides, tp)
                         : rtod_run(h, rows32.data(), n, a.max_slides, offsets.data(), ids.data(),
                                    (int64_t)ids.size(), &slides, tp);
    return rc == RTOD_OK ? 0 : lib_fail("rtod_run");
  };
  // RTOD's per-slide loop: W points, then one push and one detection per
  // slide; wall time per slide after `warmup` slides.
  std::vector<double> wall_us;
  auto stream_pass = [&]() -> int {
    if (rtod_reset(h) != RTOD_OK) return lib_fail("rtod_reset");
    auto push = [&](int64_t first, int64_t cnt) {
      return a.f64 ? rtod_push_slide_f64(h, p64 + first * D, cnt) : rtod_push_slide(h, rows32.data() + first * D, cnt);
    };
    if (push(0, a.window) != RTOD_OK) return lib_fail("rtod_push_slide");
    for (int64_t j = 0; j < slides_max; ++j) {
      const bool timing = j >= a.warmup;
      const auto t0 = std::chrono::steady_clock::now();
      if (push(a.window + j * a.slide, a.slide) != RTOD_OK) return lib_fail("rtod_push_slide");
      int64_t nout = 0;
      if (rtod_detect(h, ids.data() + offsets[(size_t)j], (int64_t)ids.size() - offsets[(size_t)j], &nout, nullptr) !=
          RTOD_OK)
        return lib_fail("rtod_detect");
      const auto t1 = std::chrono::steady_clock::now();
      offsets[(size_t)j + 1] = offsets[(size_t)j] + nout;
      if (timing) wall_us.push_back(std::chrono::duration<double, std::micro>(t1 - t0).count());
    }
    slides = slides_max;
    return 0;
  };
  if (a.streaming) {
    if (int rc = stream_pass()) return rc;
    // stage split: a second pass with per-detection stage times
    if (rtod_reset(h) != RTOD_OK) return lib_fail("rtod_reset");
    auto push = [&](int64_t first, int64_t cnt) {
      return a.f64 ? rtod_push_slide_f64(h, p64 + first * D, cnt) : rtod_push_slide(h, rows32.data() + first * D, cnt);
    };
    if (push(0, a.window) != RTOD_OK) return lib_fail("rtod_push_slide");
    std::vector<int64_t> tmp((size_t)a.window);
    int64_t timed = 0;
    for (int64_t j = 0; j < slides_max; ++j) {
      rtod_times st{};
      int64_t nout = 0;
      if (push(a.window + j * a.slide, a.slide) != RTOD_OK) return lib_fail("rtod_push_slide");
      if (rtod_detect(h, tmp.data(), (int64_t)tmp.size(), &nout, j >= a.warmup ? &st : nullptr) != RTOD_OK)
        return lib_fail("rtod_detect");
      if (j < a.warmup) continue;
      t.copy_new_points_h2d += st.copy_new_points_h2d;
      t.copy_outlier_d2h += st.copy_outlier_d2h;
      t.prepare_cell += st.prepare_cell;
      t.build_bvh += st.build_bvh;
      t.detect_outlier += st.detect_outlier;
      t.total += st.total;
      t.undetermined_per_slide += st.undetermined_per_slide;
      ++timed;
    }
    if (timed) {
      const double k = 1.0 / (double)timed;
      t.copy_new_points_h2d *= k;
      t.copy_outlier_d2h *= k;
      t.prepare_cell *= k;
      t.build_bvh *= k;
      t.detect_outlier *= k;
      t.total *= k;
      t.undetermined_per_slide *= k;
    }
  } else {
    for (int w = 0; w < a.warmup; ++w)
      if (int rc = pass(nullptr)) return rc;
    if (int rc = pass(&t)) return rc;
  }

  // A graph-replayed pass gives the total only: the stage split comes from
  // one diagnostic pass on the same handle (kernels launched one by one).
  bool split_from_profile = false;
  if (a.graph && !a.f64 && !a.streaming) {
    double ms[8] = {0};
    if (rtod_reset(h) == RTOD_OK && rtod_profile_run(h, rows32.data(), n, a.max_slides, ms, 8) == RTOD_OK) {
      // stage slots: keys, hist, scan, scatter, count, compact, train
      t.prepare_cell = ms[0] + ms[1];
      t.build_bvh = ms[2] + ms[3];
      t.detect_outlier = ms[4] + ms[5] + ms[6];
      split_from_profile = true;
    }
  }
  std::printf("\n###########   Time  ##########\n");
  std::printf("[Time] copy new points h2d: %g ms\n", t.copy_new_points_h2d);
  std::printf("[Time] copy filtered points h2d: %g ms\n", t.copy_filtered_points_h2d);
  std::printf("[Time] copy outlier d2h: %g ms\n", t.copy_outlier_d2h);
  std::printf("[Time] prepare cell: %g ms\n", t.prepare_cell);
  std::printf("[Time] build BVH: %g ms\n", t.build_bvh);
  std::printf("[Time] detect outlier: %g ms\n", t.detect_outlier);
  std::printf("[Time] total time for a slide: %g ms\n", t.total);
  std::printf("##############################\n");
  if (a.streaming && !wall_us.empty()) {
    std::vector<double> w = wall_us;
    std::sort(w.begin(), w.end());
    double mean = 0;
    for (double v : w) mean += v;
    mean /= (double)w.size();
    int64_t eng[4] = {0};
    rtod_get_stream_engine(h, eng);
    std::printf("(per-slide loop: rtod_push_slide + rtod_detect, %s engine; [Time] figures are the device\n"
                " stage times of a second pass, averaged over its slides after the warm-up)\n",
                eng[0] == RTOD_ENGINE_GRID ? "grid" : "window");
    std::printf("[Wall] slide (push + detect), median: %.3f us, mean: %.3f us, over %zu slides\n",
                w[w.size() / 2], mean, w.size());
  }
  if (split_from_profile)
    std::printf("(stage split: device time per slide of a diagnostic pass on the same handle, kernels launched "
                "one by one; total: the graph-replayed pass)\n");
  std::printf("\n");
  int64_t stats[5] = {0};
  rtod_get_stats(h, stats);
  std::printf("[Mem] Host cpu memory used(MB): %g\n", (double)(rss_kb() - rss0) / 1024.0);
  std::printf("[Mem] Device memory used for data(MB): %g\n", (double)stats[4] / (1 << 20));
  std::printf("BVH Node / slide: %lld\n", (long long)t.undetermined_per_slide);
  std::printf("Outliers / slide: %g\n", slides ? (double)offsets[(size_t)slides] / (double)slides : 0.0);
  if (a.print) {
    for (int64_t j = 0; j < slides; ++j) {
      std::printf("slide %lld:", (long long)j);
      for (int64_t k = offsets[(size_t)j]; k < offsets[(size_t)j + 1]; ++k) std::printf(" %lld", (long long)ids[(size_t)k]);
      std::printf("\n");
    }
  }
  rtod_destroy(h);
  return 0;
}
