// Launches of the streaming grid engine (grid.cuh), compiled as its own
// translation unit.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>

#include "grid.cuh"

namespace rtod {
namespace {

// Programmatic dependent launch: the kernel may be scheduled while its
// predecessor in the stream finishes (each kernel waits before reading).
template <typename... KArgs, typename... Args>
cudaError_t pdl_launch(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

unsigned point_blocks(int64_t n, int sm_count) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + GRID_INGEST_THREADS - 1) / GRID_INGEST_THREADS,
                                                          (int64_t)sm_count * 8));
}

template <int D>
cudaError_t ingest_d(const GridKind& k, const Batch& b, const Grid& g, unsigned nb, cudaStream_t st) {
  return k.f64 ? pdl_launch(k_grid_ingest<D, double>, nb, GRID_INGEST_THREADS, st, b, g, 1)
               : pdl_launch(k_grid_ingest<D, float>, nb, GRID_INGEST_THREADS, st, b, g, 1);
}

template <int D>
cudaError_t count_d(const GridKind& k, const Batch& b, const Grid& g, int sm_count, cudaStream_t st) {
  constexpr unsigned cls_blocks = NB / 32 / (GRID_COUNT_THREADS / 32);
  cudaError_t e = pdl_launch(k_grid_classify<D>, cls_blocks, GRID_COUNT_THREADS, st, b, g);
  if (e != cudaSuccess) return e;
  const unsigned blocks = (unsigned)sm_count * 4;
  if (k.f64) return pdl_launch(k_grid_count<D, 1, double>, blocks, GRID_COUNT_THREADS, st, b, g);
  return k.pred == 0 ? pdl_launch(k_grid_count<D, 0, float>, blocks, GRID_COUNT_THREADS, st, b, g)
                     : pdl_launch(k_grid_count<D, 1, float>, blocks, GRID_COUNT_THREADS, st, b, g);
}

template <int D>
cudaError_t build_d(const GridKind& k, const Batch& b, const Grid& g, int64_t lo, int64_t W, int64_t S,
                    int sm_count, cudaStream_t st) {
  cudaError_t e = pdl_launch(k_grid_reset, (NB + 255) / 256, 256, st, g);
  if (e != cudaSuccess) return e;
  e = pdl_launch(k_grid_occ<D>, point_blocks(W, sm_count), 256, st, b, g, lo);
  if (e != cudaSuccess) return e;
  e = pdl_launch(k_grid_alloc, (NB + 255) / 256, 256, st, g, b.bs);
  if (e != cudaSuccess) return e;
  const unsigned nb = point_blocks(S, sm_count);
  for (int64_t t = lo / S; t < (lo + W) / S; ++t) {
    e = k.f64 ? pdl_launch(k_grid_insert<D, double>, nb, GRID_INGEST_THREADS, st, b, g, t)
              : pdl_launch(k_grid_insert<D, float>, nb, GRID_INGEST_THREADS, st, b, g, t);
    if (e != cudaSuccess) return e;
  }
  return pdl_launch(k_grid_purity<D>, 1, 32, st, b, g, (lo + W) / S - 1);
}

// The engine serves 1 to 3 dimensions (beyond, no cell is all-inlier and the
// window engine's group counts are the better choice).
#define GRID_DIMS(D_, CALL)           \
  switch (D_) {                       \
    case 1: return CALL(1);           \
    case 2: return CALL(2);           \
    case 3: return CALL(3);           \
    default: return cudaErrorInvalidValue; \
  }

}  // namespace

cudaError_t grid_launch_ingest(const GridKind& k, const Batch& b, const Grid& g, int64_t S, int sm_count,
                               cudaStream_t st) {
  const unsigned nb = point_blocks(S, sm_count);
#define CALL(d) ingest_d<d>(k, b, g, nb, st)
  GRID_DIMS(k.D, CALL)
#undef CALL
}

cudaError_t grid_launch_count(const GridKind& k, const Batch& b, const Grid& g, int sm_count, cudaStream_t st) {
#define CALL(d) count_d<d>(k, b, g, sm_count, st)
  GRID_DIMS(k.D, CALL)
#undef CALL
}

cudaError_t grid_launch_build(const GridKind& k, const Batch& b, const Grid& g, int64_t lo, int64_t W, int64_t S,
                              int sm_count, cudaStream_t st) {
#define CALL(d) build_d<d>(k, b, g, lo, W, S, sm_count, st)
  GRID_DIMS(k.D, CALL)
#undef CALL
}

}  // namespace rtod
