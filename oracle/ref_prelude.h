/* Prelude for compiling the reference's own simulation source (src/bubble_CUDA.cu,
 * which pulls in inc/bubble_CUDA_kernel.cuh) with CUDA 12.9 for sm_100a.
 *
 * Test infrastructure only: the library built from it (oracle/_ref/libcrp_ref.so)
 * pins the oracle and the CUDA path to the reference's own arithmetic.  It is
 * never linked into the product.
 *
 * Two incompatibilities between the 2010-era reference and CUDA 12.9 are
 * neutralised here without touching the reference's text:
 *   1. `using namespace thrust;` (src/bubble_CUDA.cu:7) makes `cuda::` and `cub::`
 *      ambiguous inside the stub code nvcc generates for cub kernels.  The token
 *      `thrust` is redirected to a namespace that re-exports only the thrust
 *      names the reference uses.
 *   2. The reference defines its own CAS-loop atomicAdd(double*, double)
 *      (inc/bubble_CUDA_kernel.cuh:95-114), which clashes with the built-in one
 *      on sm_60+.  The token is renamed so the reference's version is kept and
 *      used by its own kernels.
 * All CUDA and thrust headers are included first so neither macro reaches them.
 */
#pragma once
#include <cuda_runtime.h>
#include <pthread.h>
#include <string>
#include <thrust/device_vector.h>
#include <thrust/extrema.h>
#include <thrust/functional.h>
#include <thrust/gather.h>
#include <thrust/host_vector.h>
#include <thrust/iterator/constant_iterator.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/reduce.h>
#include <thrust/scatter.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/transform_reduce.h>
#include <thrust/tuple.h>

namespace crp_thrust_shadow {
using thrust::counting_iterator;
using thrust::device_ptr;
using thrust::device_vector;
using thrust::get;
using thrust::host_vector;
using thrust::make_tuple;
using thrust::make_zip_iterator;
using thrust::maximum;
using thrust::raw_pointer_cast;
using thrust::reduce;
using thrust::transform_reduce;
using thrust::tuple;
}  // namespace crp_thrust_shadow

#define thrust crp_thrust_shadow
#define atomicAdd crp_ref_cas_atomic_add
