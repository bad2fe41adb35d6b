#pragma once
#include <cuda_runtime.h>
template <typename T> int launch_aos_to_planes(T *dst, const double *src, long long n, cudaStream_t s);
template <typename T> int launch_planes_to_aos(double *dst, const T *src, long long n, cudaStream_t s);
template <typename T> int launch_convert(T *dst, const double *src, long long n, cudaStream_t s);
template <typename T> int launch_convert_back(double *dst, const T *src, long long n, cudaStream_t s);
// a caller's device AoS vectors (S = float or double) <-> planes (T); dot (device, zeroed by the
// caller) receives sum_i M_i . H_i when not null
template <typename S, typename T> int launch_daos_to_planes(T *dst, const S *src, long long n, cudaStream_t s);
template <typename S, typename T>
int launch_planes_to_daos(S *dst, const T *src, long long n, int add, const S *M, double *dot, cudaStream_t s);
