// Shared-memory FFTs for the demag convolution passes.
//
// Lines of length L = 2^p or 3 * 2^p live in shared memory; the FFT is a Stockham
// autosort sequence of radix-R passes (R in {16, 8, 4, 2}, then one radix-3 pass last
// so that every power-of-two pass sees a power-of-two stride Ns). Each pass loads R
// points per butterfly into registers, synchronises, applies twiddles, does an
// R-point DFT in registers and stores back in place, so a line needs no ping-pong copy.
// Twiddles come from a table of exp(-2 pi i m / L) rounded from FP64 on the host.
// A thread (l, t) works on line l; t indexes its butterflies j = t + i * TPL.
#pragma once

// Dynamic shared memory ceiling every kernel with more than 48 KB is opened to. The attribute is
// per kernel function, not per launch: captured graph nodes of one kernel with different sizes all
// launch against the last value set, so it is always set to this one ceiling (no launch here uses
// more; the B200 limit per block is 227 KB).
#define BM_SMEM_CAP (200 * 1024)
// dynamic shared memory above which a launch opens its kernel to BM_SMEM_CAP: the 48 KB default
// covers static plus dynamic shared memory, so the threshold leaves room for the static part
#define BM_SMEM_DEFAULT_SAFE (40 * 1024)
#include "common.cuh"

#define BM_FFT_MAXPASS 8

// per-precision block-size limit used by every FFT kernel (launch bounds and host tiling)
template <typename T> struct bm_lb { static constexpr int v = sizeof(T) == 8 ? 384 : 512; };

struct FFTPlan {
    int L;                       // transform length
    int np;                      // number of passes
    int radix[BM_FFT_MAXPASS];
    int ns[BM_FFT_MAXPASS];      // Stockham stride before this pass
    int tws[BM_FFT_MAXPASS];     // twiddle table step L / (ns * radix)
    int tpl;                     // threads per line (host-chosen)
};

// host: radix schedule for L (power-of-two part first in radices <= 16, then radix 3)
inline bool bm_make_plan(int L, FFTPlan &P)
{
    P.L = L; P.np = 0;
    if (L < 1) return false;
    int l2 = L, three = 0;
    if (l2 % 3 == 0) { three = 1; l2 /= 3; }
    if (l2 & (l2 - 1)) return false;
    int p = 0;
    while ((1 << p) < l2) p++;
    // split p into chunks of at most 4 bits, as even as possible; avoid radix 2 unless p == 1
    int nch = (p + 3) / 4;
    int rads[BM_FFT_MAXPASS];
    int nr = 0;
    if (p > 0) {
        int base = p / nch, extra = p % nch;
        for (int c = 0; c < nch; c++) rads[nr++] = 1 << (base + (c < extra ? 1 : 0));
    }
    if (three) rads[nr++] = 3;
    int ns = 1;
    for (int i = 0; i < nr; i++) {
        P.radix[i] = rads[i];
        P.ns[i] = ns;
        P.tws[i] = L / (ns * rads[i]);
        ns *= rads[i];
    }
    P.np = nr;
    int tpl = (L + 15) / 16;
    P.tpl = tpl < 1 ? 1 : tpl;
    return true;
}

// ---------------------------------------------------------------- register DFTs
// in-place R-point DFT, natural order, forward sign exp(-2 pi i rq/R) unless INV

template <typename T, bool INV> BM_HD void dft2(cpx<T> *v)
{
    cpx<T> a = v[0], b = v[1];
    v[0] = a + b; v[1] = a - b;
}

template <typename T, bool INV> BM_HD cpx<T> rot90(cpx<T> a)   // a * (-i) forward, a * (+i) inverse
{
    return INV ? mul_i(a) : mul_mi(a);
}

template <typename T, bool INV> BM_HD void dft4(cpx<T> *v)
{
    cpx<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
    cpx<T> b0 = v[1] + v[3], b1 = rot90<T, INV>(v[1] - v[3]);
    v[0] = a0 + b0; v[2] = a0 - b0;
    v[1] = a1 + b1; v[3] = a1 - b1;
}

template <typename T, bool INV> BM_HD void dft8(cpx<T> *v)
{
    const T s = (T)0.70710678118654752440;
    // split even/odd, 4-point each, combine with exp(-+ 2 pi i q / 8)
    cpx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cpx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4<T, INV>(e);
    dft4<T, INV>(o);
    // w^1 = s(1 -+ i), w^2 = -+i, w^3 = s(-1 -+ i)
    cpx<T> o1 = INV ? mk<T>(s * (o[1].x - o[1].y), s * (o[1].x + o[1].y)) : mk<T>(s * (o[1].x + o[1].y), s * (o[1].y - o[1].x));
    cpx<T> o2 = rot90<T, INV>(o[2]);
    cpx<T> o3 = INV ? mk<T>(-s * (o[3].x + o[3].y), s * (o[3].x - o[3].y)) : mk<T>(s * (o[3].y - o[3].x), -s * (o[3].x + o[3].y));
    v[0] = e[0] + o[0]; v[4] = e[0] - o[0];
    v[1] = e[1] + o1;   v[5] = e[1] - o1;
    v[2] = e[2] + o2;   v[6] = e[2] - o2;
    v[3] = e[3] + o3;   v[7] = e[3] - o3;
}

template <typename T, bool INV> BM_HD void dft16(cpx<T> *v)
{
    // 4 x 4: columns n1 (stride 4), twiddle exp(-+2 pi i n1 k2 / 16), rows
    const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, h = (T)0.70710678118654752440;
    cpx<T> a[4][4];
#pragma unroll
    for (int n1 = 0; n1 < 4; n1++) {
        cpx<T> t[4] = {v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]};
        dft4<T, INV>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) a[n1][k2] = t[k2];
    }
    // twiddles w16^(n1*k2), n1,k2 in 0..3 ; table of cos/sin of 2 pi m / 16 for m = 0..9
    const T cs[10] = {(T)1, c1, h, s1, (T)0, -s1, -h, -c1, (T)-1, -c1};
    const T sn[10] = {(T)0, s1, h, c1, (T)1, c1, h, s1, (T)0, -s1};
#pragma unroll
    for (int n1 = 1; n1 < 4; n1++)
#pragma unroll
        for (int k2 = 1; k2 < 4; k2++) {
            int m = n1 * k2;
            cpx<T> w = mk<T>(cs[m], INV ? sn[m] : -sn[m]);
            a[n1][k2] = cmul(a[n1][k2], w);
        }
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) {
        cpx<T> t[4] = {a[0][k2], a[1][k2], a[2][k2], a[3][k2]};
        dft4<T, INV>(t);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) v[k2 + 4 * k1] = t[k1];
    }
}

template <typename T, bool INV> BM_HD void dft3(cpx<T> *v)
{
    const T c = (T)-0.5, s = (T)0.86602540378443864676;
    cpx<T> a = v[0], b = v[1], d = v[2];
    cpx<T> sum = b + d, dif = b - d;
    cpx<T> m = mk<T>(a.x + c * sum.x, a.y + c * sum.y);
    // forward: exp(-2 pi i/3) = c - i s ; the +- i s (b - d) term
    cpx<T> r = INV ? mk<T>(-s * dif.y, s * dif.x) : mk<T>(s * dif.y, -s * dif.x);
    v[0] = a + sum;
    v[1] = m + r;
    v[2] = m - r;
}

template <typename T, int R, bool INV> BM_HD void dftR(cpx<T> *v)
{
    if constexpr (R == 2) dft2<T, INV>(v);
    else if constexpr (R == 3) dft3<T, INV>(v);
    else if constexpr (R == 4) dft4<T, INV>(v);
    else if constexpr (R == 8) dft8<T, INV>(v);
    else dft16<T, INV>(v);
}

// element address inside a line: padded (1 slot per 16) for unit-stride lines, strided otherwise
template <bool PAD> BM_HD int eaddr(int e, int es) { return PAD ? (e + (e >> 4)) : e * es; }

// Split of one pass into the load phase and the compute/store phase so a CPU emulation
// can run all loads before all stores exactly as __syncthreads orders them on the GPU.
template <typename T, int R, bool PAD>
BM_HD void pass_load(const cpx<T> *base, int es, int j, int Lr, cpx<T> *v)
{
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = base[eaddr<PAD>(j + r * Lr, es)];
}

template <typename T, int R, bool PAD, bool INV>
BM_HD void pass_store(cpx<T> *base, int es, int j, int ns, int tws, const cpx<T> *tw, cpx<T> *v)
{
    int k = j & (ns - 1);
    if (ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) {
            cpx<T> w = tw[r * k * tws];
            if (INV) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
    }
    dftR<T, R, INV>(v);
    int d = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) base[eaddr<PAD>(d + r * ns, es)] = v[r];
}

template <int R> struct bmax_of { static const int v = (R == 16) ? 1 : (R == 8) ? 2 : (R == 4) ? 4 : (R == 3) ? 6 : 8; };

#ifdef __CUDACC__
template <typename T, int R, bool PAD, bool INV>
__device__ __forceinline__ void fft_pass(cpx<T> *base, int es, int t, int tpl, bool active, int L, int ns, int tws,
                                         const cpx<T> *__restrict__ tw)
{
    constexpr int BM = bmax_of<R>::v;
    cpx<T> v[BM][R];
    int Lr = L / R;
#pragma unroll
    for (int i = 0; i < BM; i++) {
        int j = t + i * tpl;
        if (active && j < Lr) pass_load<T, R, PAD>(base, es, j, Lr, v[i]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < BM; i++) {
        int j = t + i * tpl;
        if (active && j < Lr) pass_store<T, R, PAD, INV>(base, es, j, ns, tws, tw, v[i]);
    }
    __syncthreads();
}

// Full in-place FFT of this thread's line. All threads of the block must call it
// (inactive ones with active = false) because passes synchronise the block. The plan lists
// its radices in descending order, so the passes run as one loop per radix; keeping each
// radix's code in its own loop keeps register live ranges short.
template <typename T, bool PAD, bool INV>
__device__ __forceinline__ void fft_line(cpx<T> *base, int es, int t, bool active, const FFTPlan &P,
                                         const cpx<T> *__restrict__ tw)
{
    int p = 0;
    while (p < P.np && P.radix[p] == 16) { fft_pass<T, 16, PAD, INV>(base, es, t, P.tpl, active, P.L, P.ns[p], P.tws[p], tw); p++; }
    while (p < P.np && P.radix[p] == 8) { fft_pass<T, 8, PAD, INV>(base, es, t, P.tpl, active, P.L, P.ns[p], P.tws[p], tw); p++; }
    while (p < P.np && P.radix[p] == 4) { fft_pass<T, 4, PAD, INV>(base, es, t, P.tpl, active, P.L, P.ns[p], P.tws[p], tw); p++; }
    while (p < P.np && P.radix[p] == 2) { fft_pass<T, 2, PAD, INV>(base, es, t, P.tpl, active, P.L, P.ns[p], P.tws[p], tw); p++; }
    while (p < P.np && P.radix[p] == 3) { fft_pass<T, 3, PAD, INV>(base, es, t, P.tpl, active, P.L, P.ns[p], P.tws[p], tw); p++; }
}
#endif

// padded length of a unit-stride line of L elements
BM_HD int padded_len(int L) { return L + (L >> 4) + 1; }
