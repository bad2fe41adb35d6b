#pragma once
#include <cuda_runtime.h>
template <typename T> int launch_aos_to_planes(T *dst, const double *src, long long n, cudaStream_t s);
template <typename T> int launch_planes_to_aos(double *dst, const T *src, long long n, cudaStream_t s);
template <typename T> int launch_convert(T *dst, const double *src, long long n, cudaStream_t s);
template <typename T> int launch_convert_back(double *dst, const T *src, long long n, cudaStream_t s);
