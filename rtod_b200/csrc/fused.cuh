// Fused window-engine pipeline: every stage of a batch of window jobs in one
// cooperative launch, the stages separated by grid-wide barriers.
//
// The staged pipeline (kernels.cuh) runs k_ingest, k_hist, k_scan,
// k_scatter, k_count, k_compact and k_run_out as seven dependent launches;
// for one window of a stream (push/detect) the work of each is a few
// microseconds and the launches themselves dominate. k_fused runs the same
// stage bodies over virtual grids of blocks inside one resident grid:
//
//   hist (+ ingest of the staged slide) | scan | scatter | count | compact
//
// with a grid barrier after each of the first four (the ingest is folded
// into the histogram: the S newest window points are read from the staged
// slide, keyed and written into the ring there). The block that finishes
// the compaction ends the batch (finish_batch) and, for a streaming
// detection, writes the window's IDs and the batch state into the caller's
// mapped page-locked buffers, so the host waits once and copies nothing.
// The same kernel serves the multi-stream API: one launch per
// (dimension, predicate, count mode) group of streams, each stream a job.
//
// Every grid-barrier wait is bounded: after SPIN_LIMIT polls the block
// records DERR_TIMEOUT and goes on (the handle is then poisoned and scrubbed
// by rtod_reset), so no launch can hang. The launch is cooperative, which
// guarantees that all blocks are resident at once.
#pragma once

#include "kernels.cuh"

namespace rtod {

// Grid barrier state: arrivals of the current barrier and its generation,
// alone in a 128-byte line. count is back at zero after every barrier.
struct GridBar {
  unsigned int count;
  unsigned int gen;
  unsigned int pad[30];
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* a) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

// All blocks of the grid arrive before any leaves; writes before the
// barrier are visible after it. Bounded wait (DERR_TIMEOUT).
__device__ __forceinline__ void grid_sync(GridBar* gb, BatchState* bs) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int g = ld_acquire_u32(&gb->gen);
    __threadfence();
    if (atomicAdd(&gb->count, 1u) == gridDim.x - 1) {
      gb->count = 0;
      __threadfence();
      atomicAdd(&gb->gen, 1u);
    } else {
      int it = 0;
      while (ld_acquire_u32(&gb->gen) == g) {
        if (++it > SPIN_LIMIT) {
          set_err(bs, DERR_TIMEOUT);
          break;
        }
        __nanosleep(20);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

struct Fused {
  GridBar* bar;
  uint32_t hx;       // virtual blocks per job of the histogram and the scatter
  uint32_t cx;       // virtual blocks per job of the count
  uint32_t tx;       // compaction tiles of the largest job
  int32_t reset_out; // 1: this launch's IDs start at the beginning of the output (streaming)
  int64_t* ids_host;       // streaming: device view of the page-locked ID landing buffer, or null
  int64_t ids_host_cap;
  BatchState* mirror;      // device view of the page-locked copy of the batch state, or null
};

template <int D, int PRED, bool ROUTE, typename T, bool GROUP, bool INGEST>
__global__ void __launch_bounds__(256) k_fused(Batch b, Fused f) {
  const uint32_t nj = (uint32_t)b.njobs;
  if (f.reset_out && blockIdx.x == 0 && threadIdx.x == 0) b.bs->out_total = 0;  // read by the compaction
  for (uint32_t t = blockIdx.x; t < f.hx * nj; t += gridDim.x) {
    __syncthreads();
    hist_body<D, T, INGEST>(b, VB{t % f.hx, t / f.hx, f.hx});
  }
  grid_sync(f.bar, b.bs);
  for (uint32_t t = blockIdx.x; t < (uint32_t)SCAN_TILES * nj; t += gridDim.x) {
    __syncthreads();
    scan_body(b, VB{t % SCAN_TILES, t / SCAN_TILES, (uint32_t)SCAN_TILES});
  }
  grid_sync(f.bar, b.bs);
  for (uint32_t t = blockIdx.x; t < f.hx * nj; t += gridDim.x) {
    __syncthreads();
    scatter_body<D, ROUTE, T, GROUP>(b, VB{t % f.hx, t / f.hx, f.hx});
  }
  grid_sync(f.bar, b.bs);
  for (uint32_t t = blockIdx.x; t < f.cx * nj; t += gridDim.x) {
    __syncthreads();
    count_body<D, PRED, ROUTE, T, GROUP>(b, VB{t % f.cx, t / f.cx, f.cx});
  }
  grid_sync(f.bar, b.bs);
  for (uint32_t t = blockIdx.x; t < f.tx * nj; t += gridDim.x) {
    __syncthreads();
    if (compact_body(b, VB{t % f.tx, t / f.tx, f.tx})) {
      // this block ended the batch: deliver the IDs and the batch state
      __syncthreads();
      __threadfence();
      if (f.ids_host) {
        const int64_t n = min(b.bs->out_total, f.ids_host_cap);
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) f.ids_host[i] = b.out_ids[i];
      }
      __syncthreads();
      if (f.mirror && threadIdx.x == 0) *f.mirror = *b.bs;  // read by the host after its stream wait
    }
  }
}

// Which k_fused instantiation a launch needs.
struct FusedKind {
  int D;      // dimensions
  int pred;   // RTOD_PRED_* (double coordinates: the double predicate)
  int route;  // learned router on (point counts with two queues)
  int group;  // group counts
};

// Launches k_fused<...> for coordinate type T as a cooperative grid of
// `grid` blocks of 256 threads on st (grid 0: only report the blocks per SM
// that can be resident, in *per_sm). Defined in fused_f32.cu / fused_f64.cu.
template <typename T>
cudaError_t fused_dispatch(const FusedKind& k, const Batch& b, const Fused& f, int grid, cudaStream_t st,
                           int* per_sm);

}  // namespace rtod
