// Layout conversions between the host AoS FP64 vectors and the device component planes, and between
// a caller's device AoS vectors (float or double, e.g. the reference's cuVEC<cuReal3> data) and the
// planes.
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

// device AoS (S) -> planes (T)
template <typename S, typename T>
__global__ void k_daos_to_planes(T *dst, const S *__restrict__ src, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        dst[i] = (T)src[3 * i];
        dst[n + i] = (T)src[3 * i + 1];
        dst[2 * n + i] = (T)src[3 * i + 2];
    }
}

// planes (T) -> device AoS (S), set or added; with dot != nullptr also sum_i M_i . H_i in FP64 (M AoS)
template <typename S, typename T>
__global__ void k_planes_to_daos(S *dst, const T *__restrict__ src, long long n, int add, const S *__restrict__ M,
                                 double *dot)
{
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const S v = (S)src[c * n + i];
            dst[3 * i + c] = add ? (S)(dst[3 * i + c] + v) : v;
            if (dot) acc += (double)M[3 * i + c] * (double)v;
        }
    }
    if (dot) {
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(dot, acc);
    }
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

template <typename S, typename T> int launch_daos_to_planes(T *dst, const S *src, long long n, cudaStream_t s)
{
    k_daos_to_planes<S, T><<<gridn(n), 256, 0, s>>>(dst, src, n);
    return (int)cudaGetLastError();
}
template <typename S, typename T>
int launch_planes_to_daos(S *dst, const T *src, long long n, int add, const S *M, double *dot, cudaStream_t s)
{
    k_planes_to_daos<S, T><<<gridn(n), 256, 0, s>>>(dst, src, n, add, M, dot);
    return (int)cudaGetLastError();
}
template int launch_daos_to_planes<float, float>(float *, const float *, long long, cudaStream_t);
template int launch_daos_to_planes<float, double>(double *, const float *, long long, cudaStream_t);
template int launch_daos_to_planes<double, float>(float *, const double *, long long, cudaStream_t);
template int launch_daos_to_planes<double, double>(double *, const double *, long long, cudaStream_t);
template int launch_planes_to_daos<float, float>(float *, const float *, long long, int, const float *, double *, cudaStream_t);
template int launch_planes_to_daos<float, double>(float *, const double *, long long, int, const float *, double *, cudaStream_t);
template int launch_planes_to_daos<double, float>(double *, const float *, long long, int, const double *, double *, cudaStream_t);
template int launch_planes_to_daos<double, double>(double *, const double *, long long, int, const double *, double *, cudaStream_t);
template int launch_aos_to_planes<float>(float *, const double *, long long, cudaStream_t);
template int launch_aos_to_planes<double>(double *, const double *, long long, cudaStream_t);
template int launch_planes_to_aos<float>(double *, const float *, long long, cudaStream_t);
template int launch_planes_to_aos<double>(double *, const double *, long long, cudaStream_t);
template int launch_convert<float>(float *, const double *, long long, cudaStream_t);
template int launch_convert<double>(double *, const double *, long long, cudaStream_t);
template int launch_convert_back<float>(double *, const float *, long long, cudaStream_t);
template int launch_convert_back<double>(double *, const double *, long long, cudaStream_t);
