// Stand-in for the parts of sutil/sutil.h that optixScan.cpp names: the
// standard containers the SDK header brings in, roundUp, and getInputData.
// Only the OptiX module setup (make_module) calls getInputData, and the
// host-side replay never runs it; its definition (ref_fakes.cpp) reports an
// error.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

template <typename T>
T roundUp(T x, T y) {
  return ((x + y - 1) / y) * y;
}

namespace sutil {
const char* getInputData(const char* sample, const char* sampleDir, const char* filename, size_t& dataSize,
                         const char** log = nullptr, const char** compilerOptions = nullptr);
}
