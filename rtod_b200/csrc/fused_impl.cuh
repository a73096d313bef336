// Instantiations of the fused pipeline for one coordinate type (included by
// fused_f32.cu and fused_f64.cu, which nvcc compiles in parallel with the
// rest of the library).
#pragma once

#include "fused.cuh"

namespace rtod {

template <typename Kern>
cudaError_t fused_launch_one(Kern kernel, const Batch& b, const Fused& f, int grid, cudaStream_t st, int* per_sm) {
  if (grid <= 0) {
    int nb = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, 256, 0);
    *per_sm = e == cudaSuccess ? nb : 0;
    return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, b, f);
}

template <int D, int PRED, typename T>
cudaError_t fused_modes(const FusedKind& k, const Batch& b, const Fused& f, int grid, cudaStream_t st, int* per_sm) {
  if (k.route) return fused_launch_one(k_fused<D, PRED, true, T, false, true>, b, f, grid, st, per_sm);
  if (k.group) return fused_launch_one(k_fused<D, PRED, false, T, true, true>, b, f, grid, st, per_sm);
  return fused_launch_one(k_fused<D, PRED, false, T, false, true>, b, f, grid, st, per_sm);
}

template <int PRED, typename T>
cudaError_t fused_dims(const FusedKind& k, const Batch& b, const Fused& f, int grid, cudaStream_t st, int* per_sm) {
  switch (k.D) {
    case 1: return fused_modes<1, PRED, T>(k, b, f, grid, st, per_sm);
    case 2: return fused_modes<2, PRED, T>(k, b, f, grid, st, per_sm);
    case 3: return fused_modes<3, PRED, T>(k, b, f, grid, st, per_sm);
    case 4: return fused_modes<4, PRED, T>(k, b, f, grid, st, per_sm);
    case 5: return fused_modes<5, PRED, T>(k, b, f, grid, st, per_sm);
    case 6: return fused_modes<6, PRED, T>(k, b, f, grid, st, per_sm);
    case 7: return fused_modes<7, PRED, T>(k, b, f, grid, st, per_sm);
    case 8: return fused_modes<8, PRED, T>(k, b, f, grid, st, per_sm);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace rtod
