// Layout conversions between the host AoS FP64 vectors and the device component planes.
#include "kernels.h"
#include "util.h"

template <typename T>
__global__ void k_aos_to_planes(T *dst, const double *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        dst[i] = (T)src[3 * i];
        dst[n + i] = (T)src[3 * i + 1];
        dst[2 * n + i] = (T)src[3 * i + 2];
    }
}

template <typename T>
__global__ void k_planes_to_aos(double *dst, const T *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        dst[3 * i] = (double)src[i];
        dst[3 * i + 1] = (double)src[n + i];
        dst[3 * i + 2] = (double)src[2 * n + i];
    }
}

template <typename T>
__global__ void k_convert(T *dst, const double *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (T)src[i];
}

template <typename T>
__global__ void k_convert_back(double *dst, const T *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

static int gridn(long long n)
{
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

template <typename T> int launch_aos_to_planes(T *dst, const double *src, long long n, cudaStream_t s)
{
    k_aos_to_planes<T><<<gridn(n), 256, 0, s>>>(dst, src, n);
    return (int)cudaGetLastError();
}
template <typename T> int launch_planes_to_aos(double *dst, const T *src, long long n, cudaStream_t s)
{
    k_planes_to_aos<T><<<gridn(n), 256, 0, s>>>(dst, src, n);
    return (int)cudaGetLastError();
}
template <typename T> int launch_convert(T *dst, const double *src, long long n, cudaStream_t s)
{
    k_convert<T><<<gridn(n), 256, 0, s>>>(dst, src, n);
    return (int)cudaGetLastError();
}
template <typename T> int launch_convert_back(double *dst, const T *src, long long n, cudaStream_t s)
{
    k_convert_back<T><<<gridn(n), 256, 0, s>>>(dst, src, n);
    return (int)cudaGetLastError();
}

template int launch_aos_to_planes<float>(float *, const double *, long long, cudaStream_t);
template int launch_aos_to_planes<double>(double *, const double *, long long, cudaStream_t);
template int launch_planes_to_aos<float>(double *, const float *, long long, cudaStream_t);
template int launch_planes_to_aos<double>(double *, const double *, long long, cudaStream_t);
template int launch_convert<float>(float *, const double *, long long, cudaStream_t);
template int launch_convert<double>(double *, const double *, long long, cudaStream_t);
template int launch_convert_back<float>(double *, const float *, long long, cudaStream_t);
template int launch_convert_back<double>(double *, const double *, long long, cudaStream_t);
