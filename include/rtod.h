/*
 * rtod.h - C ABI of the B200 sliding-window distance outlier detector.
 *
 * A point of the current window is an outlier when at most K window points
 * (itself included) lie within distance R of it, i.e. when fewer than K
 * other points do. The window holds the last W points of a stream and
 * advances by S points per slide (W % S == 0).
 *
 * This ABI replaces RTOD's per-slide detector, stages 2-8 of its slide loop
 * (src/ods/optixScan.cpp:1045-1121): the slide H2D copy, the host grid
 * filter, the AABB kernel and BVH rebuild, the ray launch and the outlier
 * read-back. RTOD has no plugin/FFI interface of its own; its boundary is
 * the optixScan command line and compile-time macros, which rtod_config
 * mirrors field by field (each field names the flag or macro it replaces).
 * Its only C-ABI seam, `extern "C" void kGenAABB(double3*, double, unsigned,
 * OptixAabb*)` (src/ods/optixScan.cpp:49, src/ods/aabb.cu:35-45), has no
 * counterpart here: the grid build supersedes AABB generation.
 *
 * Conventions: every call returns RTOD_OK (0) or a negative RTOD_ERR_*;
 * no C++ exception crosses the ABI (RTOD's CUDA_CHECK/OPTIX_CHECK throw
 * sutil::Exception, src/sutil/Exception.h:80-113); rtod_last_error() gives
 * the message of the calling thread's last failure. A handle owns its CUDA
 * stream and graphs and must be used by one host thread at a time. Points
 * are float32, point-major (n rows of `dim` values: the layout of RTOD's
 * double3 vertices[], src/ods/optixScan.cpp:96), in host or device memory;
 * the caller keeps ownership. Outlier IDs are global stream indices
 * (0-based position of the point in the stream), sorted ascending; RTOD's
 * ring-slot IDs are index % W (src/ods/optixScan.cpp:1097).
 */
#ifndef RTOD_H
#define RTOD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTOD_OK 0
#define RTOD_ERR_CONFIG (-1)   /* invalid rtod_config */
#define RTOD_ERR_ARG (-2)      /* invalid argument (null pointer, bad size) */
#define RTOD_ERR_CUDA (-3)     /* a CUDA runtime call failed */
#define RTOD_ERR_CAPACITY (-4) /* output buffer too small */
#define RTOD_ERR_INPUT (-5)    /* non-finite coordinate, or |x|/R too large for the grid */
#define RTOD_ERR_STATE (-6)    /* call out of order (e.g. detect before the window is full) */
#define RTOD_ERR_TIMEOUT (-7)  /* a bounded device-side wait ran out */
#define RTOD_ERR_NODEV (-8)    /* no CUDA device, or not sm_100 */

/* Neighbour predicates. */
#define RTOD_PRED_FP32_LE 0 /* fl32 d^2, summed left to right without FMA, d^2 <= fl32(fl32(R)^2) */
#define RTOD_PRED_F64_LT 1  /* RTOD's double test: |dx| < R in 1-d, d^2 < R*R otherwise
                               (src/ods/optixScan.cu:170-190) */

/* rtod_config.coord: how coordinates are passed and stored. */
#define RTOD_COORD_F32 0 /* float (default) */
#define RTOD_COORD_F64 1 /* double, as RTOD stores them (double3 read with %lf, src/ods/optixScan.cpp:95-147);
                            needs RTOD_PRED_F64_LT; pass points to the _f64 entry points */

/* rtod_config.engine */
#define RTOD_ENGINE_AUTO 0
#define RTOD_ENGINE_WINDOW 1
#define RTOD_ENGINE_SPAN 2
#define RTOD_ENGINE_GRID 3 /* push/detect: the streaming grid engine (a persistent cell grid of the
                              window, updated by each slide's points); rtod_run: the span engine */

/* rtod_config.count: how the window engine counts the points of a cell
   that are not provably inliers (the range count of RTOD's intersection
   program, src/ods/optixScan.cu:158-199). Results are identical. */
#define RTOD_COUNT_AUTO 0  /* group counts in more than 3 dimensions (no cell is ever all-inlier
                              there) with the router off when a window (in the multi-stream API:
                              the windows of the streams of that dimension and predicate) holds
                              at least 4096 points per SM, point counts otherwise; the tuner
                              may choose either */
#define RTOD_COUNT_POINT 1 /* one warp per point, early exit at K+1 (with the router: early-exit
                              and full-sweep queues) */
#define RTOD_COUNT_GROUP 2 /* one warp per part of a cell bin (32 to 1024 points, longer for larger
                              launches): they share the stencil's candidates, read once per part;
                              the router is not used */

typedef struct rtod_config {
  int64_t window;      /* W  (--window, src/ods/optixScan.cpp:166-171) */
  int64_t slide;       /* S  (--slide, :172-177); W % S == 0 (:1037) */
  double R;            /* R  (--R, :179-185); > 0 */
  int32_t K;           /* K  (--K, :186-192); >= 0 */
  int32_t dim;         /* DIMENSION macro (src/ods/optixScan.h:10-12); 1..8 */
  int32_t opt;         /* OPTIMIZATION macro (optixScan.h:22-24): 0 = no grid filter,
                          1 and 2 = grid filter (identical results) */
  int32_t pred;        /* RTOD_PRED_*; default RTOD_PRED_FP32_LE */
  int32_t router;      /* 1 = learned router on: in the span engine it routes each bin's
                          counts to independent early-exit counts or to delta segments
                          (windows counted from the previous window's counts and the two
                          changed slide blocks); in the window engine it routes counted
                          points into an early-exit and a full-sweep queue. Results are
                          identical either way */
  int32_t tuner;       /* 1 = autotune cell width and block shape on the first slides */
  int32_t cells_per_r; /* grid cells per R along each hashed dimension (1..3, 1..8 in 1-d;
                          0 = auto) */
  int32_t block_warps; /* warps per block of the range-count kernel (1, 2, 4, 8; 0 = auto) */
  int32_t use_graph;   /* 1 = replay each launch sequence as a captured CUDA graph */
  int32_t device;      /* CUDA device ordinal */
  int32_t batch;       /* rtod_run: windows detected per launch (0 = auto); each window is
                          processed on its own, so results do not depend on it */
  int32_t engine;      /* rtod_run engine: RTOD_ENGINE_AUTO (span engine; the tuner may
                          choose either),
                          RTOD_ENGINE_WINDOW (one counting sort per window) or
                          RTOD_ENGINE_SPAN (one counting sort per batch of windows;
                          falls back to the window engine when W/S > 2047).
                          push/detect: RTOD_ENGINE_GRID runs the streaming grid engine
                          (each bin of the cell grid keeps its window points as a FIFO
                          that a slide's expiry and insertion update in place, three
                          launches per slide) for dim <= 3, W <= 262144 and W/S <= 4096;
                          every other case runs the window engine (measured as fast or
                          faster per slide on the stock-like, sensor-like and Gaussian-
                          mixture streams). Results are identical. */
  int32_t coord;       /* RTOD_COORD_F32 or RTOD_COORD_F64 */
  int32_t count;       /* RTOD_COUNT_*: window-engine count (push/detect, the multi-stream
                          API, rtod_run with the window engine) */
  int32_t pipeline;    /* RTOD_PIPELINE_*: how push/detect and the multi-stream API launch
                          the window engine. Results are identical. */
} rtod_config;

/* rtod_config.pipeline */
#define RTOD_PIPELINE_STAGED 0 /* default: one launch per stage (ingest, hist, scan, scatter,
                                  count, compact, output), PDL-chained, replayed as a graph */
#define RTOD_PIPELINE_FUSED 1  /* one persistent cooperative launch per detection (per group of
                                  streams in the multi-stream API) running every stage, the
                                  stages separated by bounded grid barriers. Measured on B200:
                                  no faster per window than the staged launches (the stages'
                                  own dependent memory round trips dominate, not the launches),
                                  and slower on 8-d multi-stream steps (one register budget for
                                  every stage lowers the count stage's occupancy) */

/* Per-slide stage times in ms, averaged over the slides of the last call,
   under the names of RTOD's Timer (src/ods/timer.h:16-24, :102-117). */
typedef struct rtod_times {
  double copy_new_points_h2d;      /* slide points host -> device */
  double copy_filtered_points_h2d; /* always 0: nothing is gathered on the host */
  double copy_outlier_d2h;         /* outlier IDs device -> host */
  double prepare_cell;             /* ring update + cell hashing + cell occupancy */
  double build_bvh;                /* scan + scatter into the cell-ordered SoA */
  double detect_outlier;           /* range count + outlier compaction */
  double total;                    /* whole slide */
  double undetermined_per_slide;   /* points that needed an exact count ("BVH Node / slide",
                                      src/ods/optixScan.cpp:1179) */
  int64_t slides;
} rtod_times;

typedef struct rtod_handle rtod_handle;

/* Fills *cfg with defaults: W=100000 S=5000 R=0.45 K=50 dim=1 opt=2,
   FP32 predicate, router off, tuner off, auto grid, graphs on, device 0. */
int rtod_config_init(rtod_config* cfg);

/* Validates cfg and allocates all device state (replaces data_h2d, make_gas,
   initialize_params and initialize_cell, src/ods/optixScan.cpp:232-426,
   :674-724, :960-965). */
int rtod_create(const rtod_config* cfg, rtod_handle** out);

/* Appends n points to the stream. The first push must be exactly W points
   (the initial window, src/ods/optixScan.cpp:1020-1034); every later push
   must be exactly S points (one slide, :1051-1064) and must be followed by
   rtod_detect before the next push. The caller may reuse pts at once. When
   the last rtod_detect was called with times = NULL, a slide push also
   launches the slide's detection on the handle's stream right behind the
   copy, and the next rtod_detect only waits for it and delivers the IDs. */
int rtod_push_slide(rtod_handle* h, const float* pts, int64_t n);

/* rtod_push_slide for a handle created with coord = RTOD_COORD_F64: n * dim
   doubles, stored and compared as doubles (RTOD keeps double3 points and
   tests them in double, src/ods/optixScan.cu:170-190). Each entry point
   rejects a handle of the other coordinate type (RTOD_ERR_ARG). */
int rtod_push_slide_f64(rtod_handle* h, const double* pts, int64_t n);

/* Detects the outliers of the window produced by the last push and copies
   their sorted global indices to out_ids (host or device memory, room for
   cap entries); *n_out receives the count even when it exceeds cap (then
   RTOD_ERR_CAPACITY is returned). times may be NULL; with times, the
   detection launched by the push before it (see rtod_push_slide) reports its
   copy and total times without the stage split, and the next push leaves the
   launch to rtod_detect, so that per-stage times are measured again. */
int rtod_detect(rtod_handle* h, int64_t* out_ids, int64_t cap, int64_t* n_out, rtod_times* times);

/* Runs a whole stream the way RTOD's detect_outlier does
   (src/ods/optixScan.cpp:1019-1126): the first W points fill the window,
   then up to max_slides slides (max_slides < 0: all) of S points each are
   detected, slide j covering points [(j+1)S, W+(j+1)S). The handle must be
   fresh (nothing pushed). out_offsets receives slides+1 CSR offsets into
   out_ids; *slides_out the number of slides. pts may be host or device
   memory (n * dim floats); so may out_ids (device memory and page-locked
   host memory are written during the pass, other host memory by one copy
   after it). times may be NULL. */
int rtod_run(rtod_handle* h, const float* pts, int64_t n, int64_t max_slides,
             int64_t* out_offsets, int64_t* out_ids, int64_t ids_cap, int64_t* slides_out,
             rtod_times* times);

/* rtod_run for a handle created with coord = RTOD_COORD_F64 (n * dim
   doubles). */
int rtod_run_f64(rtod_handle* h, const double* pts, int64_t n, int64_t max_slides,
                 int64_t* out_offsets, int64_t* out_ids, int64_t ids_cap, int64_t* slides_out,
                 rtod_times* times);

/* Clears the stream so that the handle can take a new first window. */
int rtod_reset(rtod_handle* h);

/* Number of slides detected since create/reset. */
int64_t rtod_slides_done(const rtod_handle* h);

/* The resolved grid and launch parameters (after autotuning, if on):
   out[0] cells per R, out[1] warps per block of the range count,
   out[2] hashed dimensions, out[3] windows per rtod_run launch, out[4] engine
   of rtod_run (RTOD_ENGINE_WINDOW or RTOD_ENGINE_SPAN). The window engine's
   count mode is read with rtod_get_count_mode.
   With rtod_config.tuner = 1 the first rtod_run times candidate settings
   (with engine = AUTO both engines, cells per R 1..3 or up to 6 in 1-d,
   2/4/8 warps per block, 8..256 windows per launch (up to 32 with the
   window engine), with the window engine and count = AUTO both count
   modes, and with the router on and point counts its routing threshold and
   full-sweep size limit) on the first 256 slides of the stream and keeps
   the fastest; the choice is cached per configuration (including engine,
   coordinate type and count mode) for the rest of the process. Results do
   not depend on it. */
int rtod_get_tuning(const rtod_handle* h, int32_t out[5]);

/* The resolved window-engine count (RTOD_COUNT_POINT or RTOD_COUNT_GROUP). */
int rtod_get_count_mode(const rtod_handle* h, int32_t* mode);

/* Self-check of the device-side failure detection: runs the look-back wait
   of the library's scans (k_scan, k_compact, k_span_scan) for a tile whose
   predecessor never publishes, on `device`. The wait gives up after its
   bound (a few hundred milliseconds), records RTOD_ERR_TIMEOUT's device code
   and returns; *timed_out = 1 when that was recorded, *ms = the kernel's
   time. Nothing faults or hangs, and the device stays usable. No
   counterpart in RTOD, which has no device-side waits. */
int rtod_check_bounded_wait(int32_t device, int32_t* timed_out, double* ms);

/* Counters since create: out[0] kernel launches issued by the library (a
   graph replay counts each of its kernels), out[1] graph replays, out[2]
   slides detected, out[3] points that needed an exact count, out[4] device
   bytes currently allocated by the handle (RTOD's "[Mem] Device memory used
   for data", src/ods/optixScan.cpp:1172-1174). */
int rtod_get_stats(const rtod_handle* h, int64_t out[5]);

/* Engine of push/detect: out[0] RTOD_ENGINE_GRID or RTOD_ENGINE_WINDOW,
   out[1] builds of the streaming grid from the ring (its first window, and
   rebuilds after its pool ran out), out[2] pool slots of the grid, out[3]
   the largest bin occupancy of the last counted window. The grid engine has
   no counterpart in RTOD, which rebuilds or refits its BVH every slide
   (src/ods/optixScan.cpp:335-426). */
int rtod_get_stream_engine(const rtod_handle* h, int64_t out[4]);

/* Pool size of the streaming grid (slots of D coordinates and a 32-bit ring
   slot each; default 16 W + 2^22, at most 2^31): the grid's first build
   starts from it and doubles it while the bins' regions do not fit. For
   callers that bound the library's device memory, and for tests of the
   rebuild path. Call before the first push (or after rtod_reset). */
int rtod_set_grid_pool(rtod_handle* h, int64_t slots);

/* Diagnostic run: like rtod_run on a fresh handle but launches every kernel
   individually with a CUDA event after each, and writes the average device
   time per slide of each pipeline stage, in order (keys, hist, scan,
   scatter, count, compact, and the router's training step), to
   kernel_ms[0..n_kernels). A batch of B windows shares one launch of each
   kernel; its time is divided by B. With the span engine the seven slots
   hold its kernels: keys (none: k_span_hist computes them), k_span_hist,
   k_span_scan + k_span_prefix, k_span_scatter, k_span_classify,
   k_span_count, and the compaction of each chunk of slides
   (k_span_compact).
   The stage names are given by rtod_kernel_name(i). Results are discarded.
   No counterpart in RTOD (it times stages with gettimeofday, src/ods/timer.h). */
int rtod_profile_run(rtod_handle* h, const float* pts, int64_t n, int64_t max_slides,
                     double* kernel_ms, int32_t n_kernels);

/* Name of pipeline kernel i (0-based) as used by rtod_profile_run, or NULL. */
const char* rtod_kernel_name(int32_t i);

/* ------------------------------------------------------------------------
   Batched streams: many independent streams, each with its own window,
   slide, R, K and dimension, advanced together one slide per step. A step
   detects the pushed slide of every stream in one replay of a captured CUDA
   graph (streams grouped by dimension, predicate and count mode, at most 256
   streams per group, one launch sequence per group, all groups in the
   graph, side by side with staged launches (the routed groups, which share
   the router, one after another);
   the count work of a group's streams is shared by all warps of its count
   launch). n_streams is at most 4096. No counterpart in RTOD (one
   stream per process). The learned router, when on, is shared by all
   streams (cfgs[0].router decides for all) and routes the streams counted
   point by point; streams above 3 dimensions on group counts run unrouted.
   ------------------------------------------------------------------------ */
typedef struct rtod_batch rtod_batch;

int rtod_batch_create(const rtod_config* cfgs, int32_t n_streams, rtod_batch** out);

/* Stream s: first push W points, then S points before each step (a stream
   without a pushed slide sits the step out). */
int rtod_batch_push(rtod_batch* b, int32_t s, const float* pts, int64_t n);

/* Detects the pushed slide of every stream that has one. out_offsets
   (n_streams + 1 entries) receives CSR offsets into out_ids by stream (a
   stream that sat out gets an empty range); *n_total the number of IDs. */
int rtod_batch_step(rtod_batch* b, int64_t* out_offsets, int64_t* out_ids, int64_t cap, int64_t* n_total);

/* out[0] steps, out[1] kernel launches (graph replays count their kernels),
   out[2] window detections summed over streams, out[3] groups, out[4]
   distance tests made by group counts (RTOD_COUNT_GROUP streams) since
   create: the work of the compute-bound count, for its roofline. */
int rtod_batch_stats(const rtod_batch* b, int64_t out[5]);

/* Settings of each group of streams (one per dimension, predicate and
   count mode): out[6 * i + 0..5] = dimension, predicate, cells per R, count
   block warps, count mode (RTOD_COUNT_POINT or RTOD_COUNT_GROUP), and 1 once
   the autotuner has settled that group (always 1 without the tuner).
   Returns the number of groups (fills at most cap of them).
   Autotuner: when any stream's rtod_config.tuner is 1, every group tries
   its candidate settings over the first steps, one setting per step, each
   timed on the device around the group's launches (two rounds), then keeps
   the fastest: cells per R (2..4 in 1-d, 1..3 up to 3-d, 1..2 beyond,
   unless the stream's config fixes it; the streams' ring keys are recomputed
   when it changes) x count block warps (2, 4, 8; 4, 8 beyond 3-d) x, beyond
   3 dimensions and with the router off, both count modes. Steps run without
   the captured graph while tuning. Results do not depend on any setting. */
int rtod_batch_get_tuning(const rtod_batch* b, int32_t* out, int32_t cap);

void rtod_batch_destroy(rtod_batch* b);

/* ------------------------------------------------------------------------
   Allocation-free detection of one window (no counterpart in RTOD).

   For callers that must not allocate device memory at detection time: code
   running inside a memory pool or allocator it does not own, real-time loops
   where cudaMalloc's implicit synchronisation and latency are not allowed,
   and hosts that only lend the library their own device buffers. All scratch
   lives in one file-scope device array of RTOD_STATIC_SCRATCH_BYTES that
   every GPU loading the library holds until the process exits; this call
   performs no cudaMalloc, cudaFree or other allocating call.

   pts      device pointer, n points point-major (n * dim floats): the window
   out_ids  device pointer with room for n entries: the sorted offsets
            (0 .. n-1) of the window's outliers
   n_out    host pointer: number of outliers written
   stream   the cudaStream_t to run on (NULL: the legacy default stream)
   Predicate, grid and filter as rtod_create with opt = 2, cells_per_r = 2,
   router and tuner off. n must be 1..RTOD_STATIC_MAX_POINTS and dim
   1..RTOD_STATIC_MAX_DIM (RTOD_ERR_CAPACITY otherwise). The call returns
   after its work on `stream` has finished.

   The first call on a device looks up the device address of the scratch
   array (cudaGetSymbolAddress, with that device current); make that first
   call before any stream capture. All calls share the one array and it keeps
   the previous call's contents (each call clears what must start at zero):
   calls that overlap on the GPU, from several host threads or streams, race
   and must not be issued. */
#define RTOD_STATIC_MAX_POINTS 65536
#define RTOD_STATIC_MAX_DIM 3
#define RTOD_STATIC_SCRATCH_BYTES (4608u * 1024u)
int rtod_detect_window_static(const float* pts, int64_t n, int32_t dim, double R, int32_t K, int32_t pred,
                              int64_t* out_ids, int64_t* n_out, void* stream);

/* Learned router state (rtod_config.router = 1). params (may be NULL)
   receives the network's rtod_mlp_param_count() parameters; info receives
   [0] training steps, [1] last training loss, [2] points routed to the
   early-exit queue, [3] to the full-sweep queue, [4] misroutes (predicted
   inlier but outlier, or the reverse), [5] routing threshold. No counterpart
   in RTOD (it has no learned component). */
int rtod_router_info(rtod_handle* h, float* params, double info[6]);

/* Sets the router's threshold: a count (span engine: a bin's run of windows;
   window engine: a point) goes to the early-exit path when the network's
   probability of "mostly inliers" is at least the threshold, else to the
   delta segments / full-sweep queue. 0 sends everything to early exit, any
   value above 1 sends everything eligible to the other path. The tuner sets
   it when on. Results do not depend on it. No counterpart in RTOD. */
int rtod_router_set_threshold(rtod_handle* h, float threshold);

/* Router network test entry points (no counterpart in RTOD), run on the
   given device with host buffers: parameter count; forward logits
   (n x 4) of n feature rows (n x 3); mean cross-entropy loss and its
   gradient for labels y in 0..3; one Adam step (step number t >= 1,
   beta1 0.9, beta2 0.999, eps 1e-8) updating params, m and v in place. */
int rtod_mlp_param_count(void);
int rtod_mlp_forward(int32_t device, const float* params, const float* x, int64_t n, float* logits);
int rtod_mlp_grad(int32_t device, const float* params, const float* x, const int32_t* y, int64_t n,
                  float* grad, float* loss);
int rtod_mlp_adam(int32_t device, float* params, float* m, float* v, int32_t t, const float* x,
                  const int32_t* y, int64_t n, float lr, float* loss);

void rtod_destroy(rtod_handle* h);

/* Message of the calling thread's last failed call ("" if none). */
const char* rtod_last_error(void);

/* Library version string. */
const char* rtod_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RTOD_H */
