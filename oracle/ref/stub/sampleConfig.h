// Stand-in for the cmake-generated sampleConfig.h of RTOD's SDK build: the
// host-side replay never loads PTX, so the sample directories stay empty.
#pragma once
#define SAMPLES_DIR ""
#define SAMPLES_PTX_DIR ""
#define SAMPLES_CUDA_DIR ""
#define CUDA_NVRTC_ENABLED 0
#ifndef OPTIX_SAMPLE_NAME
#define OPTIX_SAMPLE_NAME "optixScan"
#endif
#ifndef OPTIX_SAMPLE_DIR
#define OPTIX_SAMPLE_DIR ""
#endif
