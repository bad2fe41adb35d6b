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
    if (gate == BM_GATE_ES || gate == BM_GATE_ES_ACC)
        return *((volatile const int *)&st->es_mode) != 1 ||
               (gate == BM_GATE_ES_ACC && *((volatile const int *)&st->reject_flag) != 0);
    return *((volatile const int *)&st->need_restore) == 0;
}

// ------------------------------------------------------------------------------ transfers
template <typename T>
__global__ void k_ml_gather(T *__restrict__ dst, long long n_dst, long long dst_plane, const T *__restrict__ src,
                            long long src_plane, const int *__restrict__ ptr, const int *__restrict__ idx,
                            const T *__restrict__ w, StepState *st, int gate, int add)
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
        if (add) {
            v0 += dst[i];
            v1 += dst[i + dst_plane];
            v2 += dst[i + 2 * dst_plane];
        }
        dst[i] = v0;
        dst[i + dst_plane] = v1;
        dst[i + 2 * dst_plane] = v2;
    }
}

template <typename T>
int launch_ml_gather(T *dst, long long n_dst, long long dst_plane, const T *src, long long src_plane, const int *ptr,
                     const int *idx, const T *w, StepState *st, int gate, cudaStream_t s, int add)
{
    long long b = (n_dst + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    k_ml_gather<T><<<(int)b, 256, 0, s>>>(dst, n_dst, dst_plane, src, src_plane, ptr, idx, w, st, gate, add);
    return (int)cudaGetLastError();
}

template int launch_ml_gather<float>(float *, long long, long long, const float *, long long, const int *, const int *,
                                     const float *, StepState *, int, cudaStream_t, int);
template int launch_ml_gather<double>(double *, long long, long long, const double *, long long, const int *, const int *,
                                      const double *, StepState *, int, cudaStream_t, int);

// ------------------------------------------------------------------------------ fused z pass
// Block: W columns from kx0, the pencil pair ky / Ny - ky (ky <= Ny/2), every layer and component.
// Thread (l, c, p, w), w fastest, owns one z line of NZ points in registers: it loads layer l's
// component c of pencil p, transforms it forward, and after the shared exchange computes layer
// l's output of component c on that same line, row c of sum_s K_ls In_s, then transforms back.
// Shared memory: In [L][3][2][NZ][W], then one tile per unique kernel with its stored values at
// this block's columns (and at the x Nyquist column kx = Nx/2 that column 0 carries), copied by
// cp.async while the forward transforms run. The stored part and the symmetries that give the
// rest (true DFT values of the real-space tensors):
//   self     ky <= Ny/2, kz <= Nz/2, real; Kxy odd in ky, Kxz odd in kz, Kyz odd in both
//   z-shift  ky <= Ny/2, kz <= Nz/2; Kxy, Kyz odd in ky; K(-kz) = conj(K(kz)) for xx, yy, zz,
//            xy and -conj(K(kz)) for xz, yz
//   full     every ky and kz
// pinv: the kernel was computed for the opposite z shift, so Kxz and Kyz change sign.
// The symmetry signs are per (source, component) pairs of multipliers for the real and the
// imaginary part, one for kz <= Nz/2 and one for kz > Nz/2, applied in the unrolled kz loop.

// multipliers (re, im) of a stored self / z-shift value for kz <= Nz/2 (lo) and kz > Nz/2 (hi)
template <typename T>
__device__ __forceinline__ void ml_signs(int kind, int comp, bool ylo, bool inv, cpx<T> &lo, cpx<T> &hi)
{
    T sy = (!ylo && (comp == 3 || comp == 5)) ? (T)-1 : (T)1;
    if (inv && comp >= 4) sy = -sy;
    lo = mk<T>(sy, sy);
    if (kind == BM_MLK_SELF) hi = mk<T>(comp >= 4 ? -sy : sy, (T)0);
    else hi = (comp >= 4) ? mk<T>(-sy, sy) : mk<T>(sy, -sy);
    if (kind == BM_MLK_SELF) lo.y = (T)0;
}

// one stored value of a kernel at (comp, kz, pencil) of column w (w = -1: Nyquist column)
template <typename T, int NZ>
__device__ __forceinline__ cpx<T> ml_tile_get(const unsigned char *tile, int kind, int comp, int kz, int p, bool ylo, bool inv,
                                              int mainb, int w, int lw)
{
    if (kind == BM_MLK_FULL) {
        const cpx<T> *t = reinterpret_cast<const cpx<T> *>(tile);
        cpx<T> v = (w >= 0) ? t[(((comp * NZ + kz) * 2 + p) << lw) + w]
                            : reinterpret_cast<const cpx<T> *>(tile + mainb)[(comp * NZ + kz) * 2 + p];
        if (inv && comp >= 4) v = mk<T>(-v.x, -v.y);
        return v;
    }
    constexpr int KZ1 = NZ / 2 + 1;
    const int akz = kz <= NZ / 2 ? kz : NZ - kz;
    cpx<T> v;
    if (kind == BM_MLK_SELF) {
        const T *t = reinterpret_cast<const T *>(tile);
        v = mk<T>((w >= 0) ? t[((comp * KZ1 + akz) << lw) + w] : reinterpret_cast<const T *>(tile + mainb)[comp * KZ1 + akz], (T)0);
    } else {
        const cpx<T> *t = reinterpret_cast<const cpx<T> *>(tile);
        v = (w >= 0) ? t[((comp * KZ1 + akz) << lw) + w] : reinterpret_cast<const cpx<T> *>(tile + mainb)[comp * KZ1 + akz];
    }
    cpx<T> lo, hi;
    ml_signs<T>(kind, comp, ylo, inv, lo, hi);
    const cpx<T> sg = kz <= NZ / 2 ? lo : hi;
    return mk<T>(v.x * sg.x, v.y * sg.y);
}

template <int NZ> struct zml_bounds {
    static constexpr int blocks = NZ <= 16 ? 2 : 1;
};

// WC: the tile width as a compile-time constant (0: a.W at run time), so that the shared-memory
// addresses of the products become a base plus an immediate offset
template <typename T, int NZ, int WC>
__global__ void __launch_bounds__(bm_lb<T>::v, zml_bounds<NZ>::blocks) k_zmid_ml(MLZArgs<T> a)
{
    if (ml_gated_out<T>(a.st, a.gate)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int KZ1 = NZ / 2 + 1;
    const int W = WC ? WC : a.W, L = a.L, Ny = a.Ny, nz = a.nz, LX = a.LX;
    const int lw = WC ? (WC == 32 ? 5 : WC == 16 ? 4 : WC == 8 ? 3 : WC == 4 ? 2 : WC == 2 ? 1 : 0) : __ffs(W) - 1;
    const int Kx1 = LX + 1, Ky1 = Ny / 2 + 1;
    cpx<T> *In = reinterpret_cast<cpx<T> *>(smraw);
    unsigned char *Ks = smraw + (size_t)L * 6 * NZ * W * sizeof(cpx<T>);
    auto IDX = [&](int l, int c, int p, int e, int w) -> int { return ((((l * 3 + c) * 2 + p) * NZ + e) << lw) + w; };
    const int kx0 = blockIdx.x * W;
    const int ky = blockIdx.y, kym = (Ny - ky) % Ny;
    const bool single = (ky == kym);
    const int np = single ? 1 : 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    // kernel tiles (async): thread group g (W threads, one column each) copies rows g, g + ng, ...
    // of every unique kernel, one address computation per element
    {
        const int w = tid & (W - 1), g = tid >> lw, ng = nt >> lw;
        const int kx = kx0 + w;
        const bool okx = kx < LX;
        for (int u = 0; u < a.nu; u++) {
            const MLUDesc d = a.u[u];
            unsigned char *tb = Ks + d.sm;
            const int mainb = zmid_ml_tile_main<T>(d.kind, NZ, W);
            if (d.kind == BM_MLK_FULL) {
                const long long nk = (long long)Kx1 * Ny * NZ;
                const cpx<T> *K = reinterpret_cast<const cpx<T> *>(a.K + d.off);
                cpx<T> *t = reinterpret_cast<cpx<T> *>(tb);
                cpx<T> *tn = reinterpret_cast<cpx<T> *>(tb + mainb);
                for (int j = g; j < 12 * NZ; j += ng) {
                    const int pp = j & 1, kz = (j >> 1) % NZ, comp = (j >> 1) / NZ;
                    const bool ok = okx && pp < np;
                    const long long q = comp * nk + ((long long)kz * Ny + (pp ? kym : ky)) * Kx1;
                    cp_async_cpx<T>(&t[(j << lw) + w], ok ? &K[q + kx] : K, ok);
                    if (kx0 == 0 && w == 0) cp_async_cpx<T>(&tn[j], pp < np ? &K[q + LX] : K, pp < np);
                }
            } else if (d.kind == BM_MLK_SELF) {
                const long long nk = (long long)Kx1 * Ky1 * KZ1;
                const T *K = a.K + d.off;
                T *t = reinterpret_cast<T *>(tb);
                T *tn = reinterpret_cast<T *>(tb + mainb);
                for (int j = g; j < 6 * KZ1; j += ng) {
                    const int kz = j % KZ1, comp = j / KZ1;
                    const long long q = comp * nk + ((long long)kz * Ky1 + ky) * Kx1;
                    cp_async_real<T>(&t[(j << lw) + w], okx ? &K[q + kx] : K, okx);
                    if (kx0 == 0 && w == 0) cp_async_real<T>(&tn[j], &K[q + LX], true);
                }
            } else {
                const long long nk = (long long)Kx1 * Ky1 * KZ1;
                const cpx<T> *K = reinterpret_cast<const cpx<T> *>(a.K + d.off);
                cpx<T> *t = reinterpret_cast<cpx<T> *>(tb);
                cpx<T> *tn = reinterpret_cast<cpx<T> *>(tb + mainb);
                for (int j = g; j < 6 * KZ1; j += ng) {
                    const int kz = j % KZ1, comp = j / KZ1;
                    const long long q = comp * nk + ((long long)kz * Ky1 + ky) * Kx1;
                    cp_async_cpx<T>(&t[(j << lw) + w], okx ? &K[q + kx] : K, okx);
                    if (kx0 == 0 && w == 0) cp_async_cpx<T>(&tn[j], &K[q + LX], true);
                }
            }
        }
    }
    cp_async_commit();
    // forward transforms of the owned lines
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
    cp_async_wait_all();
    __syncthreads();
    const int cmp[3] = {c == 0 ? 0 : (c == 1 ? 3 : 4), c == 0 ? 3 : (c == 1 ? 1 : 5), c == 0 ? 4 : (c == 1 ? 5 : 2)};
    // row c of sum_s K_ls In_s on this line
    if (own && kx != 0) {
#pragma unroll
        for (int e = 0; e < NZ; e++) v[e] = mk<T>(0, 0);
        for (int s = 0; s < L; s++) {
            const MLUDesc d = a.u[a.pu[l * L + s]];
            const bool inv = a.pinv[l * L + s] != 0;
            const cpx<T> *t = reinterpret_cast<const cpx<T> *>(Ks + d.sm);
            if (d.kind == BM_MLK_FULL) {
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    const T sg = (inv && cmp[cc] >= 4) ? (T)-1 : (T)1;
                    const cpx<T> *row = t + ((cmp[cc] * NZ * 2 + p) << lw) + w;
                    const cpx<T> *in = In + IDX(s, cc, p, 0, w);
#pragma unroll
                    for (int kz = 0; kz < NZ; kz++) v[kz] = v[kz] + cscale(cmul(row[(kz * 2) << lw], in[kz << lw]), sg);
                }
            } else if (d.kind == BM_MLK_SELF) {
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    cpx<T> lo, hi;
                    ml_signs<T>(d.kind, cmp[cc], p == 0, inv, lo, hi);
                    const T *row = reinterpret_cast<const T *>(Ks + d.sm) + ((cmp[cc] * KZ1) << lw) + w;
                    const cpx<T> *in = In + IDX(s, cc, p, 0, w);
#pragma unroll
                    for (int kz = 0; kz < NZ; kz++) {
                        const int akz = kz <= NZ / 2 ? kz : NZ - kz;
                        const T kr = (kz <= NZ / 2 ? lo.x : hi.x) * row[akz << lw];
                        const cpx<T> x = in[kz << lw];
                        v[kz] = mk<T>(v[kz].x + kr * x.x, v[kz].y + kr * x.y);
                    }
                }
            } else {
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    cpx<T> lo, hi;
                    ml_signs<T>(d.kind, cmp[cc], p == 0, inv, lo, hi);
                    const cpx<T> *row = t + ((cmp[cc] * KZ1) << lw) + w;
                    const cpx<T> *in = In + IDX(s, cc, p, 0, w);
#pragma unroll
                    for (int kz = 0; kz < NZ; kz++) {
                        const int akz = kz <= NZ / 2 ? kz : NZ - kz;
                        const cpx<T> sg = kz <= NZ / 2 ? lo : hi;
                        const cpx<T> kr = row[akz << lw];
                        v[kz] = v[kz] + cmul(mk<T>(kr.x * sg.x, kr.y * sg.y), in[kz << lw]);
                    }
                }
            }
        }
    }
    if (kx0 == 0) {
        // column 0 packs the DC (kx = 0) and Nyquist (kx = Nx/2) spectra; both are unpacked with
        // the Hermitian mirror (pencil 0, kz) <-> (pencil pm, -kz), multiplied and re-packed. The
        // results go through a small shared buffer after the tiles so that the kz loop can stay
        // rolled (only the first block column runs this).
        cpx<T> *O = reinterpret_cast<cpx<T> *>(Ks + a.ksm);
        if (own && kx == 0) {
            const int pm = single ? 0 : 1;
            for (int kz = 0; kz < NZ; kz++) {
                const int kr = p == 0 ? kz : (NZ - kz) % NZ;   // frequency in pencil-0 terms
                const int krm = (NZ - kr) % NZ;
                cpx<T> acc = mk<T>(0, 0);
                for (int s = 0; s < L; s++) {
                    const MLUDesc d = a.u[a.pu[l * L + s]];
                    const bool inv = a.pinv[l * L + s] != 0;
                    const unsigned char *tile = Ks + d.sm;
                    const int mainb = zmid_ml_tile_main<T>(d.kind, NZ, W);
                    cpx<T> ap = mk<T>(0, 0), bp = mk<T>(0, 0);
                    for (int cc = 0; cc < 3; cc++) {
                        const cpx<T> C = In[IDX(s, cc, 0, kr, 0)], cj = conj(In[IDX(s, cc, pm, krm, 0)]);
                        const cpx<T> A = cscale(C + cj, (T)0.5), B = cscale(mul_mi(C - cj), (T)0.5);
                        const cpx<T> k0 = ml_tile_get<T, NZ>(tile, d.kind, cmp[cc], kr, 0, true, inv, mainb, 0, lw);
                        const cpx<T> kn = ml_tile_get<T, NZ>(tile, d.kind, cmp[cc], kr, 0, true, inv, mainb, -1, lw);
                        ap = ap + cmul(k0, A);
                        bp = bp + cmul(kn, B);
                    }
                    acc = acc + (p == 0 ? ap + mul_i(bp) : conj(ap) + mul_i(conj(bp)));
                }
                O[((l * 3 + c) * 2 + p) * NZ + kz] = acc;
            }
        }
        __syncthreads();
        if (own && kx == 0) {
#pragma unroll
            for (int e = 0; e < NZ; e++) v[e] = O[((l * 3 + c) * 2 + p) * NZ + e];
        }
    }
    RegFFT<T, NZ, true>::run(v, a.twz, 1);
    if (own) {
        cpx<T> *S = a.S2[l];
#pragma unroll
        for (int e = 0; e < (NZ + 1) / 2; e++)
            if (e < nz) S[gbase + e * gstride] = v[e];
    }
}

template <typename T, int NZ, int WC>
static int launch_zmid_ml_w(const MLZArgs<T> &a, cudaStream_t s)
{
    int nt = (6 * a.L * a.W + 31) & ~31;
    if (nt > bm_lb<T>::v) return 304;
    size_t smem = zmid_ml_smem<T>(a.L, NZ, a.W, a.ksm);
    if (smem > 200 * 1024) return 305;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_zmid_ml<T, NZ, WC>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    dim3 grid((a.LX + a.W - 1) / a.W, a.Ny / 2 + 1);
    k_zmid_ml<T, NZ, WC><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T, int NZ>
static int launch_zmid_ml_t(const MLZArgs<T> &a, cudaStream_t s)
{
    return a.W == 16 ? launch_zmid_ml_w<T, NZ, 16>(a, s) : launch_zmid_ml_w<T, NZ, 0>(a, s);
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
