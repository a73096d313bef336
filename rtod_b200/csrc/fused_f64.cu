// Fused window-engine pipeline, double coordinates (RTOD's double predicate).
#include "fused_impl.cuh"

namespace rtod {

template <>
cudaError_t fused_dispatch<double>(const FusedKind& k, const Batch& b, const Fused& f, int grid, cudaStream_t st,
                                   int* per_sm) {
  return fused_dims<1, double>(k, b, f, grid, st, per_sm);
}

}  // namespace rtod
