// Compile-time register FFTs.
//
// RegFFT<T, N, INV>::run(v, tw, ts) transforms N complex values held in registers (natural
// order in, natural order out). N is 2^p or 3 * 2^p up to 64. Composite lengths use one
// Cooley-Tukey split N = N1 * N2 (N1 the largest of 16, 8, 4, 3, 2 dividing N with N2 >= 2):
//   u_{n1}[k2] = DFT_N2( x[n1 + N1 n2] ),  u_{n1}[k2] *= w_N^(n1 k2),
//   X[k2 + N2 k1] = DFT_N1 over n1 of u_{n1}[k2].
// All indices are compile-time, so the arrays stay in registers and products with known
// zeros (zero-padded inputs) and unused outputs fold away. Twiddles w_N^m are read from a
// table of exp(-2 pi i j / L) at index m * ts (ts = L / N), rounded from FP64 on the host.
#pragma once
#include "fft.cuh"

template <int N> struct rf_split {
    static constexpr int n1 = (N % 16 == 0 && N / 16 >= 2) ? 16 : (N % 8 == 0 && N / 8 >= 2) ? 8 : (N % 4 == 0 && N / 4 >= 2) ? 4
                              : (N % 3 == 0 && N / 3 >= 2) ? 3 : 2;
    static constexpr int n2 = N / n1;
};

template <typename T, int N, bool INV> struct RegFFT {
    __device__ __forceinline__ static void run(cpx<T> *v, const cpx<T> *__restrict__ tw, int ts)
    {
        constexpr int N1 = rf_split<N>::n1, N2 = rf_split<N>::n2;
        cpx<T> u[N1][N2];
#pragma unroll
        for (int a = 0; a < N1; a++) {
#pragma unroll
            for (int b = 0; b < N2; b++) u[a][b] = v[a + N1 * b];
            RegFFT<T, N2, INV>::run(u[a], tw, ts * N1);
        }
#pragma unroll
        for (int a = 1; a < N1; a++)
#pragma unroll
            for (int b = 1; b < N2; b++) {
                cpx<T> w = tw[(a * b) * ts];
                if (INV) w.y = -w.y;
                u[a][b] = cmul(u[a][b], w);
            }
#pragma unroll
        for (int b = 0; b < N2; b++) {
            cpx<T> t[N1];
#pragma unroll
            for (int a = 0; a < N1; a++) t[a] = u[a][b];
            RegFFT<T, N1, INV>::run(t, tw, ts * N2);
#pragma unroll
            for (int a = 0; a < N1; a++) v[b + N2 * a] = t[a];
        }
    }
};

template <typename T, bool INV> struct RegFFT<T, 1, INV> {
    __device__ __forceinline__ static void run(cpx<T> *, const cpx<T> *, int) {}
};
template <typename T, bool INV> struct RegFFT<T, 2, INV> {
    __device__ __forceinline__ static void run(cpx<T> *v, const cpx<T> *, int) { dft2<T, INV>(v); }
};
template <typename T, bool INV> struct RegFFT<T, 3, INV> {
    __device__ __forceinline__ static void run(cpx<T> *v, const cpx<T> *, int) { dft3<T, INV>(v); }
};
template <typename T, bool INV> struct RegFFT<T, 4, INV> {
    __device__ __forceinline__ static void run(cpx<T> *v, const cpx<T> *, int) { dft4<T, INV>(v); }
};
template <typename T, bool INV> struct RegFFT<T, 8, INV> {
    __device__ __forceinline__ static void run(cpx<T> *v, const cpx<T> *, int) { dft8<T, INV>(v); }
};
template <typename T, bool INV> struct RegFFT<T, 16, INV> {
    __device__ __forceinline__ static void run(cpx<T> *v, const cpx<T> *, int) { dft16<T, INV>(v); }
};
