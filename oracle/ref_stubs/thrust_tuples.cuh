/* Compile-only stand-in for inc/thrust_tuples.cuh, which the reference
 * includes (inc/bubble_CUDA_kernel.cuh:4) but does not ship.  The four functor
 * templates are used only by determine_focal_point (inc/bubble_CUDA_kernel.cuh:
 * 1132-1166), the focal-point tracker, which is outside the simulated path.
 * The harness never reads its result; these definitions exist so that the
 * reference translation unit compiles. */
#pragma once
#include <thrust/tuple.h>

template <typename I, typename T> struct padded_grid_tuple {
  I width, pitch_width;
  __host__ __device__ padded_grid_tuple(I w, I pw) : width(w), pitch_width(pw) {}
  __host__ __device__ thrust::tuple<bool, T> operator()(const thrust::tuple<I, T>& t) const {
    return thrust::make_tuple((thrust::get<0>(t) % pitch_width) < width, thrust::get<1>(t));
  }
};

template <typename I, typename T> struct reduce_max_tuple {
  __host__ __device__ thrust::tuple<bool, T> operator()(const thrust::tuple<bool, T>& a,
                                                        const thrust::tuple<bool, T>& b) const {
    return thrust::make_tuple(true, thrust::get<1>(a) > thrust::get<1>(b) ? thrust::get<1>(a) : thrust::get<1>(b));
  }
};

template <typename I, typename T> struct weighted_coordinate_tuple {
  I width, pitch_width;
  T dx, dy, peak;
  __host__ __device__ weighted_coordinate_tuple(I w, I pw, T dx_, T dy_, T m)
      : width(w), pitch_width(pw), dx(dx_), dy(dy_), peak(m) {}
  __host__ __device__ thrust::tuple<bool, T, T> operator()(const thrust::tuple<I, T>&) const {
    return thrust::make_tuple(true, T(0), T(0));
  }
};

template <typename I, typename T> struct reduce_add_tuple {
  __host__ __device__ thrust::tuple<bool, T, T> operator()(const thrust::tuple<bool, T, T>& a,
                                                           const thrust::tuple<bool, T, T>& b) const {
    return thrust::make_tuple(true, thrust::get<1>(a) + thrust::get<1>(b), thrust::get<2>(a) + thrust::get<2>(b));
  }
};
