/*
 * helper_cuda.h -- stand-in for the CUDA samples header of that name, which
 * the culip reference includes (libs/utils/types.cuh:22) for
 * _cudaGetErrorEnum in its CHECK_CUDA macro.  TEST INFRASTRUCTURE ONLY
 * (reference build, oracle/build_ref.py).
 */
#pragma once
#include <cuda_runtime.h>

static inline const char* _cudaGetErrorEnum(cudaError_t e) { return cudaGetErrorName(e); }
