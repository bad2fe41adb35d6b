// Device passes of the multilayered convolution (the reference's SDemag multilayer branch,
// Boris/SDemag.cpp:786-900; GPU twin SDemagCUDA::UpdateField, Boris/SDemagCUDA.cpp:270, with the
// L x L products of Boris/DemagKernelCollectionCUDA_Mult.cu).
//
//   k_ml_gather   weighted mesh transfer in either direction (CSR lists built on the host)
//   k_zmid_ml     one pass over every layer's (kx, +-ky) pencils: forward z FFT of each layer's
//                 three components, Out_d = sum_s K_ds In_s for every destination d, inverse
//                 z FFT, store; in 2D (Nz = 1) the same pass is the plain L x L product
// The spectra are the single-mesh layout [c][z][y][kx] after the x and y passes (column 0 packs
// the DC and Nyquist x bins), one buffer per layer, all on the common N grid.
#include "ml.h"
#include "kernels.h"
#include "regfft.cuh"

template <typename T>
__device__ __forceinline__ bool ml_gated_out(const StepState *st, int gate)
{
    if (gate == BM_GATE_ALWAYS || st == nullptr) return false;
    if (gate == BM_GATE_ACCEPTED) return *((volatile const int *)&st->reject_flag) != 0;
    return *((volatile const int *)&st->need_restore) == 0;
}

// ------------------------------------------------------------------------------ transfers
template <typename T>
__global__ void k_ml_gather(T *__restrict__ dst, long long n_dst, long long dst_plane, const T *__restrict__ src,
                            long long src_plane, const int *__restrict__ ptr, const int *__restrict__ idx,
                            const T *__restrict__ w, StepState *st, int gate)
{
    if (ml_gated_out<T>(st, gate)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_dst; i += (long long)gridDim.x * blockDim.x) {
        T v0 = 0, v1 = 0, v2 = 0;
        const int q1 = ptr[i + 1];
        for (int q = ptr[i]; q < q1; q++) {
            const long long e = idx[q];
            const T wq = w[q];
            v0 += wq * src[e];
            v1 += wq * src[e + src_plane];
            v2 += wq * src[e + 2 * src_plane];
        }
        dst[i] = v0;
        dst[i + dst_plane] = v1;
        dst[i + 2 * dst_plane] = v2;
    }
}

template <typename T>
int launch_ml_gather(T *dst, long long n_dst, long long dst_plane, const T *src, long long src_plane, const int *ptr,
                     const int *idx, const T *w, StepState *st, int gate, cudaStream_t s)
{
    long long b = (n_dst + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    k_ml_gather<T><<<(int)b, 256, 0, s>>>(dst, n_dst, dst_plane, src, src_plane, ptr, idx, w, st, gate);
    return (int)cudaGetLastError();
}

template int launch_ml_gather<float>(float *, long long, long long, const float *, long long, const int *, const int *,
                                     const float *, StepState *, int, cudaStream_t);
template int launch_ml_gather<double>(double *, long long, long long, const double *, long long, const int *, const int *,
                                      const double *, StepState *, int, cudaStream_t);

// ------------------------------------------------------------------------------ kernel values
// 6 complex components (xx, yy, zz, xy, xz, yz) of one kernel at frequency (kx, ky, kz),
// kx in [0, Nx/2], ky in [0, Ny), kz in [0, Nz), expanded from the stored part:
//   self     real; Kxy odd in ky, Kxz odd in kz, Kyz odd in ky and kz
//   z-shift  Kxy, Kyz odd in ky; K(-kz) = conj(K(kz)) for xx, yy, zz, xy and -conj(K(kz)) for xz, yz
//   full     stored as is
// inv: the kernel was computed for the opposite z shift; Kxz and Kyz change sign.
template <typename T>
__device__ __forceinline__ void ml_kfetch(const T *__restrict__ K, const MLKDesc &d, int kx, int ky, int kz, int Kx1, int Ny,
                                          int Nz, cpx<T> k[6])
{
    const int Ky1 = Ny / 2 + 1, Kz1 = Nz / 2 + 1;
    const bool ylo = ky <= Ny / 2, zlo = kz <= Nz / 2;
    const int aky = ylo ? ky : Ny - ky, akz = zlo ? kz : Nz - kz;
    const T sy = ylo ? (T)1 : (T)-1, sz = zlo ? (T)1 : (T)-1;
    if (d.kind == BM_MLK_SELF) {
        const long long nk = (long long)Kx1 * Ky1 * Kz1;
        const T *b = K + d.off + ((long long)akz * Ky1 + aky) * Kx1 + kx;
#pragma unroll
        for (int c = 0; c < 6; c++) k[c] = mk<T>(__ldg(b + c * nk), (T)0);
        k[3].x *= sy;
        k[4].x *= sz;
        k[5].x *= sy * sz;
    } else if (d.kind == BM_MLK_ZSHIFT) {
        const long long nk = (long long)Kx1 * Ky1 * Kz1;
        const cpx<T> *b = reinterpret_cast<const cpx<T> *>(K + d.off) + ((long long)akz * Ky1 + aky) * Kx1 + kx;
#pragma unroll
        for (int c = 0; c < 6; c++) {
            cpx<T> v = b[c * nk];
            if (!zlo) {
                v = conj(v);
                if (c >= 4) v = mk<T>(-v.x, -v.y);
            }
            if (c == 3 || c == 5) v = cscale(v, sy);
            k[c] = v;
        }
    } else {
        const long long nk = (long long)Kx1 * Ny * Nz;
        const cpx<T> *b = reinterpret_cast<const cpx<T> *>(K + d.off) + ((long long)kz * Ny + ky) * Kx1 + kx;
#pragma unroll
        for (int c = 0; c < 6; c++) k[c] = b[c * nk];
    }
    if (d.inv) {
        k[4] = mk<T>(-k[4].x, -k[4].y);
        k[5] = mk<T>(-k[5].x, -k[5].y);
    }
}

// h += K m for the symmetric complex 3x3 kernel
template <typename T>
__device__ __forceinline__ void ml_kmac(const cpx<T> k[6], const cpx<T> m[3], cpx<T> h[3])
{
    h[0] = h[0] + cmul(k[0], m[0]) + cmul(k[3], m[1]) + cmul(k[4], m[2]);
    h[1] = h[1] + cmul(k[3], m[0]) + cmul(k[1], m[1]) + cmul(k[5], m[2]);
    h[2] = h[2] + cmul(k[4], m[0]) + cmul(k[5], m[1]) + cmul(k[2], m[2]);
}

// ------------------------------------------------------------------------------ fused z pass
// Block: W columns from kx0, the pencil pair ky / Ny - ky, every layer and component.
// Thread (l, c, p, w), w fastest, owns one z line of NZ points in registers. Shared memory:
// In [L][3][2][NZ][W] (forward spectra), Out [L][3][2][NZ][W] (products per destination).
template <typename T, int NZ>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid_ml(MLZArgs<T> a)
{
    if (ml_gated_out<T>(a.st, a.gate)) return;
    extern __shared__ unsigned char smraw[];
    const int W = a.W, L = a.L, Ny = a.Ny, nz = a.nz, LX = a.LX;
    const int lw = __ffs(W) - 1;
    const int Kx1 = LX + 1;
    cpx<T> *In = reinterpret_cast<cpx<T> *>(smraw);
    cpx<T> *Out = In + (size_t)L * 6 * NZ * W;
    auto IDX = [&](int l, int c, int p, int e, int w) -> int { return ((((l * 3 + c) * 2 + p) * NZ + e) << lw) + w; };
    const int kx0 = blockIdx.x * W;
    const int ky = blockIdx.y, kym = (Ny - ky) % Ny;
    const bool single = (ky == kym);
    const int np = single ? 1 : 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int w = tid & (W - 1);
    const int p = (tid >> lw) & 1;
    const int lc = tid >> (lw + 1);
    const int l = lc / 3, c = lc - 3 * (lc / 3);
    const int kx = kx0 + w;
    const bool line = (l < L);
    const bool own = line && (p < np) && (kx < LX);
    const int kyp = p ? kym : ky;
    const long long gbase = ((long long)c * nz * Ny + kyp) * LX + kx;
    const long long gstride = (long long)Ny * LX;
    cpx<T> v[NZ];
#pragma unroll
    for (int e = 0; e < NZ; e++) v[e] = mk<T>(0, 0);
    if (own) {
        const cpx<T> *S = a.S2[l];
#pragma unroll
        for (int e = 0; e < (NZ + 1) / 2; e++)
            if (e < nz) v[e] = S[gbase + e * gstride];
    }
    RegFFT<T, NZ, false>::run(v, a.twz, 1);
    if (line) {
#pragma unroll
        for (int e = 0; e < NZ; e++) In[IDX(l, c, p, e, w)] = v[e];
    }
    __syncthreads();
    // products for every destination
    const int tot = L * np * NZ * W;
    for (int t = tid; t < tot; t += nt) {
        const int ww = t & (W - 1);
        int r = t >> lw;
        const int kz = r % NZ;
        r /= NZ;
        const int pp = r % np, d = r / np;
        const int kxx = kx0 + ww;
        if (kxx >= LX) continue;
        if (kxx == 0) {
            // packed DC / Nyquist column: pair (p = 0, kz) with (mirror pencil, -kz)
            if (pp == 1) continue;
            if (single && kz > NZ / 2) continue;
            const int pm = single ? 0 : 1;
            const int kzm = (NZ - kz) % NZ;
            cpx<T> Ap[3] = {mk<T>(0, 0), mk<T>(0, 0), mk<T>(0, 0)}, Bp[3] = {mk<T>(0, 0), mk<T>(0, 0), mk<T>(0, 0)};
            for (int s = 0; s < L; s++) {
                cpx<T> A[3], B[3];
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    cpx<T> C = In[IDX(s, cc, 0, kz, ww)], cj = conj(In[IDX(s, cc, pm, kzm, ww)]);
                    A[cc] = cscale(C + cj, (T)0.5);
                    B[cc] = cscale(mul_mi(C - cj), (T)0.5);
                }
                cpx<T> k0[6], kn[6];
                ml_kfetch<T>(a.K, a.kd[d * L + s], 0, ky, kz, Kx1, Ny, NZ, k0);
                ml_kfetch<T>(a.K, a.kd[d * L + s], LX, ky, kz, Kx1, Ny, NZ, kn);
                ml_kmac<T>(k0, A, Ap);
                ml_kmac<T>(kn, B, Bp);
            }
            const bool self = single && (kzm == kz);
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                Out[IDX(d, cc, 0, kz, ww)] = Ap[cc] + mul_i(Bp[cc]);
                if (!self) Out[IDX(d, cc, pm, kzm, ww)] = conj(Ap[cc]) + mul_i(conj(Bp[cc]));
            }
        } else {
            const int kyq = pp ? kym : ky;
            cpx<T> h[3] = {mk<T>(0, 0), mk<T>(0, 0), mk<T>(0, 0)};
            for (int s = 0; s < L; s++) {
                cpx<T> m[3] = {In[IDX(s, 0, pp, kz, ww)], In[IDX(s, 1, pp, kz, ww)], In[IDX(s, 2, pp, kz, ww)]};
                cpx<T> k[6];
                ml_kfetch<T>(a.K, a.kd[d * L + s], kxx, kyq, kz, Kx1, Ny, NZ, k);
                ml_kmac<T>(k, m, h);
            }
#pragma unroll
            for (int cc = 0; cc < 3; cc++) Out[IDX(d, cc, pp, kz, ww)] = h[cc];
        }
    }
    __syncthreads();
    if (line) {
#pragma unroll
        for (int e = 0; e < NZ; e++) v[e] = Out[IDX(l, c, p, e, w)];
    }
    RegFFT<T, NZ, true>::run(v, a.twz, 1);
    if (own) {
        cpx<T> *S = a.S2[l];
#pragma unroll
        for (int e = 0; e < (NZ + 1) / 2; e++)
            if (e < nz) S[gbase + e * gstride] = v[e];
    }
}

template <typename T, int NZ>
static int launch_zmid_ml_t(const MLZArgs<T> &a, cudaStream_t s)
{
    int nt = (6 * a.L * a.W + 31) & ~31;
    if (nt > bm_lb<T>::v) return 304;
    size_t smem = zmid_ml_smem<T>(a.L, NZ, a.W);
    if (smem > 200 * 1024) return 305;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_zmid_ml<T, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    dim3 grid((a.LX + a.W - 1) / a.W, a.Ny / 2 + 1);
    k_zmid_ml<T, NZ><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

bool zmid_ml_supported(int Nz)
{
    return Nz == 1 || Nz == 4 || Nz == 6 || Nz == 8 || Nz == 12 || Nz == 16 || Nz == 24 || Nz == 32 || Nz == 48 || Nz == 64;
}

template <typename T> int launch_zmid_ml(const MLZArgs<T> &a, cudaStream_t s)
{
    if (a.W < 1 || (a.W & (a.W - 1)) || a.L < 1 || a.L > BM_ML_MAXL) return 301;
    switch (a.Nz) {
    case 1: return launch_zmid_ml_t<T, 1>(a, s);
    case 4: return launch_zmid_ml_t<T, 4>(a, s);
    case 6: return launch_zmid_ml_t<T, 6>(a, s);
    case 8: return launch_zmid_ml_t<T, 8>(a, s);
    case 12: return launch_zmid_ml_t<T, 12>(a, s);
    case 16: return launch_zmid_ml_t<T, 16>(a, s);
    case 24: return launch_zmid_ml_t<T, 24>(a, s);
    case 32: return launch_zmid_ml_t<T, 32>(a, s);
    case 48: return launch_zmid_ml_t<T, 48>(a, s);
    case 64: return launch_zmid_ml_t<T, 64>(a, s);
    default: return 302;
    }
}

template int launch_zmid_ml<float>(const MLZArgs<float> &, cudaStream_t);
template int launch_zmid_ml<double>(const MLZArgs<double> &, cudaStream_t);
