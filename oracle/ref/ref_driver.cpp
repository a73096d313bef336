// Runs RTOD's own detection code on the CPU and returns its per-slide
// outlier sets (TEST INFRASTRUCTURE ONLY: it produces the reference-run
// fixtures under tests/golden/; the product library never links or loads it).
//
// RTOD's host code is compiled unmodified from src/ods/optixScan.cpp
// (oracle/ref/Makefile), with the device side replaced by the host
// stand-ins of ref_fakes.cpp. rtod_ref_detect calls RTOD's functions in the
// order of its main() (src/ods/optixScan.cpp:1128-1168), skipping the OptiX
// context, module, program-group, pipeline and SBT setup that only the GPU
// launch needs:
//   read_data          the stream, read from RTOD's text format (%lf per
//                      line, %lf,%lf,%lf in 3-d) with its global min / max
//   data_h2d, make_gas, initialize_params, initialize_cell
//   detect_outlier(state, false)   the whole slide loop (:1019-1126): ring
//                      update, FixQueue grid filter, AABB build, launch,
//                      outlier pick from the counts (:1094-1099)
// The pick of each slide is read from state.h_outlier_list (ring slots; the
// list is refilled with -1 before every slide so that its length is visible).
//
// Optionally every slide is also checked by RTOD's own brute force,
// check_outlier (:817-881), in a child process: given a list one longer than
// its own count, check_outlier prints its complete outlier list (window
// offsets) and exits; the parent parses that listing.
#include <fcntl.h>
#include <sys/wait.h>
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "state.h"
#include "timer.h"

// Definitions in src/ods/optixScan.cpp.
extern int data_num;
extern double3* vertices;
extern Timer timer;
void read_data(std::string& outfile, ScanState& state);
void data_h2d(ScanState& state);
void make_gas(ScanState& state);
void initialize_params(ScanState& state);
void initialize_cell(ScanState& state);
void detect_outlier(ScanState& state, bool warmup);
void check_outlier(int* outlier_list, int outlier_num, double3* vertices_window, int window_id, int unit_num,
                   ScanState& state);

namespace rtod_ref {
extern void* slide_marker;
extern void (*on_slide_start)();
extern int64_t margin_events;
void install_optix_fakes();
}  // namespace rtod_ref

namespace {

ScanState* g_state = nullptr;
std::vector<std::vector<int>> g_picks;  // per slide: ring slots picked by RTOD
int64_t g_undetermined = 0;
bool g_started = false;

void capture_pick() {
  ScanState& st = *g_state;
  std::vector<int> slots;
  for (int i = 0; i < st.window && st.h_outlier_list[i] >= 0; ++i) slots.push_back(st.h_outlier_list[i]);
  g_picks.push_back(slots);
  g_undetermined += st.params.ray_origin_num;
}

void slide_start() {
  if (g_started) capture_pick();
  g_started = true;
  for (int i = 0; i < g_state->window; ++i) g_state->h_outlier_list[i] = -1;
}

// Silences RTOD's progress output on stdout for the duration of a call.
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    std::fflush(stdout);
    std::cout.flush();
    saved = dup(1);
    int null_fd = open("/dev/null", O_WRONLY);
    if (null_fd >= 0) {
      dup2(null_fd, 1);
      close(null_fd);
    }
  }
  ~QuietStdout() {
    std::fflush(stdout);
    std::cout.flush();
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

// RTOD's brute force for window `window_id` (1-based slide number), run in a
// child whose stdout goes to a file; returns the window offsets it lists, or
// false when its output could not be read.
bool brute_force(ScanState& st, int window_id, int unit_num, const std::string& path, std::vector<int>* out) {
  std::fflush(stdout);
  std::cout.flush();
  pid_t pid = fork();
  if (pid < 0) return false;
  if (pid == 0) {
    int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0600);
    if (fd < 0) _exit(3);
    dup2(fd, 1);
    dup2(fd, 2);
    close(fd);
    // one entry more than any window can have outliers: the counts differ, so
    // check_outlier prints its own list and exits
    std::vector<int> dummy((size_t)st.window + 1, -1);
    check_outlier(dummy.data(), st.window + 1, vertices + (int64_t)window_id * st.slide, window_id, unit_num, st);
    std::cout.flush();
    _exit(2);  // not reached: check_outlier exits on a count mismatch
  }
  int status = 0;
  waitpid(pid, &status, 0);
  if (!WIFEXITED(status) || WEXITSTATUS(status) != 1) return false;
  std::ifstream in(path);
  std::string line;
  bool inside = false, seen = false;
  out->clear();
  while (std::getline(in, line)) {
    if (line == "Naive outliers:") {
      inside = seen = true;
      continue;
    }
    if (!inside) continue;
    if (line == "BVH node index:") break;
    const size_t colon = line.find(": ");
    if (colon == std::string::npos) break;
    out->push_back(std::atoi(line.c_str() + colon + 2));
  }
  return seen;
}

}  // namespace

// Runs RTOD on n points (point-major, DIMENSION doubles each) with window W,
// slide S, radius R, K neighbours. offsets (slides + 1) and ids receive the
// sorted global indices of RTOD's picked outliers per slide (CSR);
// with brute != 0, b_offsets / b_ids receive check_outlier's sets the same
// way. stats: [0] undetermined points summed over slides ("BVH Node"),
// [1] margin events, [2] slides. Returns the number of slides, or < 0.
extern "C" __attribute__((visibility("default"))) int64_t rtod_ref_detect(
    const double* pts, int64_t n, int32_t W, int32_t S, double R, int32_t K, int32_t brute, int64_t* offsets,
    int64_t* ids, int64_t ids_cap, int64_t* b_offsets, int64_t* b_ids, int64_t b_cap, int64_t* stats,
    const char* tmp_dir) {
  if (n < W || W <= 0 || S <= 0 || W % S != 0) return -1;
  const std::string dir = tmp_dir ? tmp_dir : "/tmp";
  const std::string data_path = dir + "/rtod_ref_stream_" + std::to_string(getpid()) + ".txt";
  const std::string out_path = dir + "/rtod_ref_check_" + std::to_string(getpid()) + ".txt";
  {
    FILE* f = std::fopen(data_path.c_str(), "w");
    if (!f) return -2;
    for (int64_t i = 0; i < n; ++i) {
#if DIMENSION == 1
      std::fprintf(f, "%.17g\n", pts[i]);
#else
      std::fprintf(f, "%.17g,%.17g,%.17g\n", pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
#endif
    }
    std::fclose(f);
  }
  ScanState* st = new ScanState();
  st->infile = data_path;
  st->window = W;
  st->slide = S;
  st->R = R;
  st->K = K;
  data_num = (int)n;
  rtod_ref::install_optix_fakes();
  g_state = st;
  g_picks.clear();
  g_undetermined = 0;
  g_started = false;
  rtod_ref::margin_events = 0;
  try {
    QuietStdout quiet;
    read_data(st->infile, *st);
    data_h2d(*st);
    make_gas(*st);
    initialize_params(*st);
    initialize_cell(*st);
    timer.clearNew();
    rtod_ref::slide_marker = st->params.outlier_num;
    rtod_ref::on_slide_start = slide_start;
    detect_outlier(*st, false);
    if (g_started) capture_pick();
    rtod_ref::on_slide_start = nullptr;
    rtod_ref::slide_marker = nullptr;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "rtod_ref_detect: %s\n", e.what());
    std::remove(data_path.c_str());
    return -3;
  }
  std::remove(data_path.c_str());
  const int64_t slides = (int64_t)g_picks.size();
  int64_t pos = 0;
  offsets[0] = 0;
  for (int64_t j = 0; j < slides; ++j) {
    // slide j (0-based) detects the window [(j+1)S, W+(j+1)S); ring slot = index % W
    const int64_t lo = (j + 1) * (int64_t)S;
    std::vector<int64_t> g;
    for (int slot : g_picks[j]) {
      const int64_t base = lo - lo % W;
      int64_t idx = base + slot;
      if (idx < lo) idx += W;
      g.push_back(idx);
    }
    std::sort(g.begin(), g.end());
    for (int64_t v : g) {
      if (pos >= ids_cap) return -4;
      ids[pos++] = v;
    }
    offsets[j + 1] = pos;
  }
  if (brute) {
    const int unit_num = W / S;
    int64_t bpos = 0;
    b_offsets[0] = 0;
    std::vector<int> lst;
    for (int64_t j = 0; j < slides; ++j) {
      if (!brute_force(*st, (int)(j + 1), unit_num, out_path, &lst)) {
        std::remove(out_path.c_str());
        return -5;
      }
      std::sort(lst.begin(), lst.end());
      for (int v : lst) {
        if (bpos >= b_cap) return -4;
        b_ids[bpos++] = (j + 1) * (int64_t)S + v;
      }
      b_offsets[j + 1] = bpos;
    }
    std::remove(out_path.c_str());
  }
  stats[0] = g_undetermined;
  stats[1] = rtod_ref::margin_events;
  stats[2] = slides;
  free(vertices);
  vertices = nullptr;
  // RTOD's fake device buffers and host arrays of this run are left to the
  // process (its cleanup() also tears down OptiX objects never created here).
  delete st;
  g_state = nullptr;
  return slides;
}
