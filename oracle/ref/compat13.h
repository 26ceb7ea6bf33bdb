/* Force-included when compiling the reference's refine.cu with CUDA 12.9.
 * The reference calls the CUDA 13 spellings of three graph-construction
 * APIs; CUDA 12.9 provides the same signatures under versioned names. */
#pragma once
#include <cuda_runtime.h>
#define cudaGraphAddNode cudaGraphAddNode_v2
#define cudaGraphAddDependencies cudaGraphAddDependencies_v2
#define cudaStreamGetCaptureInfo cudaStreamGetCaptureInfo_v3
