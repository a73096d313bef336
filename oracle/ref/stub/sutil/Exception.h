// Stand-in for sutil/Exception.h: the CUDA_CHECK / OPTIX_CHECK family of
// macros that optixScan.cpp wraps its runtime calls in. A failed call throws
// std::runtime_error (the SDK throws sutil::Exception).
#pragma once
#include <cuda_runtime.h>
#include <optix.h>
#include <stdexcept>
#include <string>

#define CUDA_CHECK(call)                                                          \
  do {                                                                            \
    cudaError_t rc_ = (call);                                                     \
    if (rc_ != cudaSuccess) throw std::runtime_error(std::string("CUDA call failed: ") + #call); \
  } while (0)

#define CUDA_SYNC_CHECK()                                                          \
  do {                                                                             \
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) \
      throw std::runtime_error("CUDA synchronisation failed");                     \
  } while (0)

#define OPTIX_CHECK(call)                                                         \
  do {                                                                            \
    OptixResult rc_ = (call);                                                     \
    if (rc_ != OPTIX_SUCCESS) throw std::runtime_error(std::string("OptiX call failed: ") + #call); \
  } while (0)

#define OPTIX_CHECK_LOG(call) OPTIX_CHECK(call)
