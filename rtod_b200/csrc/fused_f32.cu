// Fused window-engine pipeline, float coordinates (both predicates).
#include "fused_impl.cuh"

namespace rtod {

template <>
cudaError_t fused_dispatch<float>(const FusedKind& k, const Batch& b, const Fused& f, int grid, cudaStream_t st,
                                  int* per_sm) {
  return k.pred == 0 ? fused_dims<0, float>(k, b, f, grid, st, per_sm) : fused_dims<1, float>(k, b, f, grid, st, per_sm);
}

}  // namespace rtod
