/* Stand-in for the NVIDIA SDK cutil header the reference includes.  Only the
 * CUDA_SAFE_CALL macro is used by the reference's simulation code; here it
 * reports a failing call on stderr instead of exiting the process. */
#pragma once
#include <cstdio>
#include <cuda_runtime.h>
#define CUDA_SAFE_CALL(call)                                                   \
  do {                                                                         \
    cudaError_t crp_ref_err_ = (call);                                         \
    if (crp_ref_err_ != cudaSuccess)                                           \
      fprintf(stderr, "reference harness: %s at %s:%d\n",                     \
              cudaGetErrorString(crp_ref_err_), __FILE__, __LINE__);           \
  } while (0)
