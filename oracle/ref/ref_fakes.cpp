// Host stand-ins for the device side of RTOD's detector, so that RTOD's own
// host code (src/ods/optixScan.cpp, compiled unmodified from the RTOD
// sources beside this file by oracle/ref/Makefile) runs on the CPU.
//
// TEST INFRASTRUCTURE ONLY: used to produce reference-run fixtures; the
// product library never links or loads it.
//
// What is replaced, and how:
//  * The seven CUDA runtime calls optixScan.cpp makes (cudaMalloc, cudaFree,
//    cudaMemcpy, cudaMemset, cudaMemGetInfo, cudaDeviceSynchronize,
//    cudaGetLastError): "device memory" is host memory, copies are memcpy.
//  * kGenAABB (src/ods/aabb.cu:5-45): float AABBs of half-width R around
//    double points, the double -> float conversion of each bound rounding
//    to nearest as the kernel's assignments do.
//  * The OptiX entry points reached from detect_outlier through the
//    function table (optixAccelComputeMemoryUsage, optixAccelBuild,
//    optixLaunch): the build records the AABB list; the launch restates the
//    OPTIMIZATION == 2 programs of src/ods/optixScan.cu:
//      __raygen__rg (:21-75): one ray per window point, origin =
//        float(points[idx]), payload 2 = idx % window_size;
//      traversal: a ray of length FLT_MIN from inside a box reports that
//        box; a box "contains" the float origin when min <= o <= max in
//        every dimension (the BVH itself cannot change the result);
//      __intersection__cube (:158-199): skip when count[prim] > K; test
//        |dx| < R (1-d) or dx^2+dy^2+dz^2 < R2 (3-d) in double on the double
//        points (evaluated here without FMA contraction); count[prim]++.
//    Pairs that pass the double test but whose float box misses the float
//    origin ("margin events") are counted: for them the result would depend
//    on OptiX's traversal precision, so fixtures use streams with none.
#include <cuda_runtime_api.h>
#include <optix.h>
#include <optix_function_table.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "optixScan.h"

extern OptixFunctionTable g_optixFunctionTable;

namespace rtod_ref {

// Hook: called by the fake cudaMemset when it clears `slide_marker`
// (detect_outlier clears params.outlier_num at the start of every slide,
// src/ods/optixScan.cpp:1047).
void* slide_marker = nullptr;
void (*on_slide_start)() = nullptr;
int64_t margin_events = 0;

namespace {
CUdeviceptr g_aabbs = 0;
unsigned g_num_prims = 0;
}  // namespace

}  // namespace rtod_ref

// ---------------------------------------------------------------------------
// CUDA runtime: host memory stands in for device memory
// ---------------------------------------------------------------------------
extern "C" {

cudaError_t cudaMalloc(void** p, size_t size) {
  *p = std::calloc(size ? size : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}

cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}

cudaError_t cudaMemcpy(void* dst, const void* src, size_t count, cudaMemcpyKind) {
  if (count) std::memmove(dst, src, count);
  return cudaSuccess;
}

cudaError_t cudaMemset(void* p, int value, size_t count) {
  if (p == rtod_ref::slide_marker && rtod_ref::on_slide_start) rtod_ref::on_slide_start();
  if (count) std::memset(p, value, count);
  return cudaSuccess;
}

cudaError_t cudaMemGetInfo(size_t* free_bytes, size_t* total) {
  *free_bytes = 0;
  *total = 0;
  return cudaSuccess;
}

cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }

cudaError_t cudaGetLastError(void) { return cudaSuccess; }

// src/ods/aabb.cu:5-45 on the host.
void kGenAABB(double3* points, double radius, unsigned int numPrims, OptixAabb* aabb) {
  for (unsigned i = 0; i < numPrims; ++i) {
    const double3 c = points[i];
    aabb[i] = OptixAabb{(float)(c.x - radius), (float)(c.y - radius), (float)(c.z - radius),
                        (float)(c.x + radius), (float)(c.y + radius), (float)(c.z + radius)};
  }
}

}  // extern "C"

namespace sutil {
const char* getInputData(const char*, const char*, const char*, size_t& size, const char**, const char**) {
  size = 0;
  return nullptr;  // no PTX on the host-side replay
}
}  // namespace sutil

// ---------------------------------------------------------------------------
// OptiX: acceleration build and launch
// ---------------------------------------------------------------------------
namespace rtod_ref {
namespace {

OptixResult fake_memory_usage(OptixDeviceContext, const OptixAccelBuildOptions*, const OptixBuildInput*,
                              unsigned int, OptixAccelBufferSizes* sizes) {
  sizes->outputSizeInBytes = 64;
  sizes->tempSizeInBytes = 64;
  sizes->tempUpdateSizeInBytes = 64;
  return OPTIX_SUCCESS;
}

OptixResult fake_build(OptixDeviceContext, CUstream, const OptixAccelBuildOptions*, const OptixBuildInput* in,
                       unsigned int, CUdeviceptr, size_t, CUdeviceptr, size_t, OptixTraversableHandle* handle,
                       const OptixAccelEmitDesc*, unsigned int) {
  g_aabbs = in[0].customPrimitiveArray.aabbBuffers[0];
  g_num_prims = in[0].customPrimitiveArray.numPrimitives;
  *handle = 1;
  return OPTIX_SUCCESS;
}

inline bool box_contains(const OptixAabb& b, float x, float y, float z) {
  return b.minX <= x && x <= b.maxX && b.minY <= y && y <= b.maxY && b.minZ <= z && z <= b.maxZ;
}

// src/ods/optixScan.cu:158-199 (OPTIMIZATION == 2), without contraction.
inline bool exact_test(const Params& p, const double3& ray_orig, const double3& point) {
#if DIMENSION == 1
  return std::fabs(ray_orig.x - point.x) < p.R;
#else
  const double ox = ray_orig.x - point.x, oy = ray_orig.y - point.y, oz = ray_orig.z - point.z;
  const double sqdist = ox * ox + oy * oy + oz * oz;  // built with -ffp-contract=off
  return sqdist < p.R2;
#endif
}

OptixResult fake_launch(OptixPipeline, CUstream, CUdeviceptr params_ptr, size_t, const OptixShaderBindingTable*,
                        unsigned int width, unsigned int, unsigned int) {
  const Params& p = *reinterpret_cast<const Params*>(params_ptr);
  const OptixAabb* box = reinterpret_cast<const OptixAabb*>(g_aabbs);
  for (unsigned idx = 0; idx < width; ++idx) {
    const double3 o = p.points[idx % (unsigned)p.window_size];
    const float ox = (float)o.x, oy = (float)o.y, oz = (float)o.z;  // __raygen__rg origin
    for (unsigned prim = 0; prim < g_num_prims; ++prim) {
      const bool hit_box = box_contains(box[prim], ox, oy, oz);
      const bool exact = exact_test(p, o, p.ray_origin_list[prim]);
      if (exact && !hit_box) ++margin_events;
      if (!hit_box) continue;
      if (p.outlier_neighbor_num[prim] > p.K) continue;
      if (exact) p.outlier_neighbor_num[prim] += 1;
    }
  }
  return OPTIX_SUCCESS;
}

}  // namespace

void install_optix_fakes() {
  g_optixFunctionTable.optixAccelComputeMemoryUsage = fake_memory_usage;
  g_optixFunctionTable.optixAccelBuild = fake_build;
  g_optixFunctionTable.optixLaunch = fake_launch;
}

}  // namespace rtod_ref
