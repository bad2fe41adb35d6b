// y and z passes of the demag FFT convolution (reference: Boris/Convolution.h:262 Convolute_2D,
// :659 Convolute_3D; kernel product Boris/DemagKernel.cpp:42 KernelMultiplication_2D_line and
// :85 KernelMultiplication_3D_line).
//
// Spectrum layout after the x pass: S1[c][z][y][kx], kx in [0, LX), LX = Nx/2. Column 0 packs
// the two purely-real-input x bins (DC in .x, Nyquist in .y after the R2C split), so every row
// is exactly LX complex values. The y/z transforms are linear and carry the packed pair along;
// wherever the 3x3 kernel product happens, column 0 is unpacked with the Hermitian mirror
// (ky, kz) <-> (-ky, -kz), multiplied by K(kx=0) and K(kx=Nx/2) respectively, and re-packed.
//
// 2D (nz == 1):  ymid2d   y FFT, 3x3 product, inverse y FFT, in place on S1 (n.y rows kept)
// 3D:            yfwd     S1 (n.z planes, n.y rows) -> S2 (n.z planes, Ny rows)
//                zmid     z FFT over n.z nonzero planes, product, inverse, first n.z planes kept
//                yinv     S2 -> S1 (first n.y rows kept)
#include "kernels.h"

template <typename T>
__device__ __forceinline__ bool gated_out(const StepState *st, int gate)
{
    if (gate == BM_GATE_ALWAYS || st == nullptr) return false;
    if (gate == BM_GATE_ACCEPTED) return *((volatile const int *)&st->reject_flag) != 0;
    return *((volatile const int *)&st->need_restore) == 0;
}

template <typename T>
__device__ __forceinline__ void kapply(const T k[6], const cpx<T> m[3], cpx<T> h[3])
{
    h[0] = mk<T>(k[0] * m[0].x + k[3] * m[1].x + k[4] * m[2].x, k[0] * m[0].y + k[3] * m[1].y + k[4] * m[2].y);
    h[1] = mk<T>(k[3] * m[0].x + k[1] * m[1].x + k[5] * m[2].x, k[3] * m[0].y + k[1] * m[1].y + k[5] * m[2].y);
    h[2] = mk<T>(k[4] * m[0].x + k[5] * m[1].x + k[2] * m[2].x, k[4] * m[0].y + k[5] * m[1].y + k[2] * m[2].y);
}

// ------------------------------------------------------------------------------ 2D
// smem: data [3][Ny][W] complex, kernel tile [4][Ky1][W] real (xx, yy, zz, xy at kz = 0),
// column-0 Nyquist kernel [4][Ky1] real. All tiles arrive by cp.async (one DRAM latency).
template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ymid2d(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    extern __shared__ unsigned char smraw[];
    const int W = a.W, Ny = a.Ny, ny = a.ny, LX = a.LX;
    const int Ky1 = Ny / 2 + 1, Kx1 = LX + 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 3 * Ny * W);
    T *Kn = Ks + 4 * Ky1 * W;
    const int kx0 = blockIdx.x * W;
    const int nt = blockDim.x, tid = threadIdx.x;
    const long long plane = (long long)ny * LX;   // one component (nz == 1)
    const long long nk = (long long)Kx1 * Ky1;
    for (int idx = tid; idx < 3 * Ny * W; idx += nt) {
        int w = idx % W, e = (idx / W) % Ny, c = idx / (W * Ny);
        int kx = kx0 + w;
        bool ok = (e < ny && kx < LX);
        cp_async_cpx<T>(&sm[(c * Ny + e) * W + w], ok ? &a.S1[c * plane + (long long)e * LX + kx] : a.S1, ok);
    }
    for (int idx = tid; idx < 4 * Ky1 * W; idx += nt) {
        int w = idx % W, ky = (idx / W) % Ky1, c = idx / (W * Ky1);
        int kx = kx0 + w;
        bool ok = kx < LX;
        cp_async_real<T>(&Ks[(c * Ky1 + ky) * W + w], ok ? &a.K[c * nk + (long long)ky * Kx1 + kx] : a.K, ok);
    }
    if (kx0 == 0) {
        for (int idx = tid; idx < 4 * Ky1; idx += nt) {
            int ky = idx % Ky1, c = idx / Ky1;
            cp_async_real<T>(&Kn[c * Ky1 + ky], &a.K[c * nk + (long long)ky * Kx1 + LX], true);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int tpl = a.py.tpl;
    const int l = tid % W, t = tid / W;
    const bool act = t < tpl;
    // three explicit calls: a loop around fft_line defeats register allocation
    fft_line<T, false, false>(sm + 0 * Ny * W + l, W, t, act, a.py, a.twy);
    fft_line<T, false, false>(sm + 1 * Ny * W + l, W, t, act, a.py, a.twy);
    fft_line<T, false, false>(sm + 2 * Ny * W + l, W, t, act, a.py, a.twy);
    // product: Kxy odd in y (KernelMultiplication_2D_line, DemagKernel.cpp:42)
    for (int idx = tid; idx < W * Ny; idx += nt) {
        int w = idx % W, ky = idx / W, kx = kx0 + w;
        if (kx >= LX) continue;
        if (kx == 0) {
            if (ky > Ny / 2) continue;
            int kym = (Ny - ky) % Ny;
            cpx<T> C[3], Cm[3], A[3], B[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                C[c] = sm[(c * Ny + ky) * W + w];
                Cm[c] = sm[(c * Ny + kym) * W + w];
                cpx<T> cc = conj(Cm[c]);
                A[c] = cscale(C[c] + cc, (T)0.5);
                B[c] = cscale(mul_mi(C[c] - cc), (T)0.5);
            }
            T k0[6] = {Ks[(0 * Ky1 + ky) * W + w], Ks[(1 * Ky1 + ky) * W + w], Ks[(2 * Ky1 + ky) * W + w],
                       Ks[(3 * Ky1 + ky) * W + w], (T)0, (T)0};
            T kn[6] = {Kn[0 * Ky1 + ky], Kn[1 * Ky1 + ky], Kn[2 * Ky1 + ky], Kn[3 * Ky1 + ky], (T)0, (T)0};
            cpx<T> Ap[3], Bp[3];
            kapply<T>(k0, A, Ap);
            kapply<T>(kn, B, Bp);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                sm[(c * Ny + ky) * W + w] = Ap[c] + mul_i(Bp[c]);
                if (kym != ky) sm[(c * Ny + kym) * W + w] = conj(Ap[c]) + mul_i(conj(Bp[c]));
            }
        } else {
            int aky = ky <= Ny / 2 ? ky : Ny - ky;
            T sy = ky <= Ny / 2 ? (T)1 : (T)-1;
            T k[6] = {Ks[(0 * Ky1 + aky) * W + w], Ks[(1 * Ky1 + aky) * W + w], Ks[(2 * Ky1 + aky) * W + w],
                      sy * Ks[(3 * Ky1 + aky) * W + w], (T)0, (T)0};
            cpx<T> m[3], h[3];
#pragma unroll
            for (int c = 0; c < 3; c++) m[c] = sm[(c * Ny + ky) * W + w];
            kapply<T>(k, m, h);
#pragma unroll
            for (int c = 0; c < 3; c++) sm[(c * Ny + ky) * W + w] = h[c];
        }
    }
    __syncthreads();
    fft_line<T, false, true>(sm + 0 * Ny * W + l, W, t, act, a.py, a.twy);
    fft_line<T, false, true>(sm + 1 * Ny * W + l, W, t, act, a.py, a.twy);
    fft_line<T, false, true>(sm + 2 * Ny * W + l, W, t, act, a.py, a.twy);
    for (int idx = tid; idx < 3 * ny * W; idx += nt) {
        int w = idx % W, e = (idx / W) % ny, cc = idx / (W * ny);
        int kx = kx0 + w;
        if (kx < LX) a.S1[cc * plane + (long long)e * LX + kx] = sm[(cc * Ny + e) * W + w];
    }
}

// ------------------------------------------------------------------------------ 3D y passes
template <typename T, bool INV>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ypass3d(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    extern __shared__ unsigned char smraw[];
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    const int W = a.W, Ny = a.Ny, ny = a.ny, LX = a.LX, nz = a.nz;
    const int kx0 = blockIdx.x * W, z = blockIdx.y, c = blockIdx.z;
    const int nt = blockDim.x, tid = threadIdx.x;
    const cpx<T> *src;
    cpx<T> *dst;
    int nin, nout;
    if (!INV) {
        src = a.S1 + ((long long)c * nz + z) * ny * LX; nin = ny;
        dst = a.S2 + ((long long)c * nz + z) * Ny * LX; nout = Ny;
    } else {
        src = a.S2 + ((long long)c * nz + z) * Ny * LX; nin = Ny;
        dst = a.S1 + ((long long)c * nz + z) * ny * LX; nout = ny;
    }
    for (int idx = tid; idx < Ny * W; idx += nt) {
        int w = idx % W, e = idx / W, kx = kx0 + w;
        bool ok = (e < nin && kx < LX);
        cp_async_cpx<T>(&sm[e * W + w], ok ? &src[(long long)e * LX + kx] : src, ok);
    }
    cp_async_wait_all();
    __syncthreads();
    const int tpl = a.py.tpl;
    const int l = tid % W, t = tid / W;
    fft_line<T, false, INV>(sm + l, W, t, t < tpl, a.py, a.twy);
    for (int idx = tid; idx < nout * W; idx += nt) {
        int w = idx % W, e = idx / W, kx = kx0 + w;
        if (kx < LX) dst[(long long)e * LX + kx] = sm[e * W + w];
    }
}

// ------------------------------------------------------------------------------ 3D z pass + product
// Block: W columns kx0.., the mirror pencils ky and Ny - ky (which share |ky|), 3 components.
// smem: data [3][2][Nz][W] complex, kernel tile [6][Kz1][W] real at |ky|, column-0 Nyquist
// kernel [6][Kz1] real.
template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    extern __shared__ unsigned char smraw[];
    const int W = a.W, Ny = a.Ny, Nz = a.Nz, nz = a.nz, LX = a.LX;
    const int Kx1 = LX + 1, Ky1 = Ny / 2 + 1, Kz1 = Nz / 2 + 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 6 * Nz * W);
    T *Kn = Ks + 6 * Kz1 * W;
    const int kx0 = blockIdx.x * W;
    const int ky = blockIdx.y, kym = (Ny - ky) % Ny;
    const bool single = (ky == kym);
    const int nt = blockDim.x, tid = threadIdx.x;
    const long long nk = (long long)Kx1 * Ky1 * Kz1;
    auto S = [&](int c, int p, int e, int w) -> cpx<T> & { return sm[((c * 2 + p) * Nz + e) * W + w]; };
    const int np = single ? 1 : 2;
    for (int idx = tid; idx < 3 * np * Nz * W; idx += nt) {
        int w = idx % W, e = (idx / W) % Nz, cp = idx / (W * Nz);
        int c = cp / np, p = cp % np;
        int kyp = p ? kym : ky, kx = kx0 + w;
        bool ok = (e < nz && kx < LX);
        cp_async_cpx<T>(&S(c, p, e, w), ok ? &a.S2[(((long long)c * nz + e) * Ny + kyp) * LX + kx] : a.S2, ok);
    }
    for (int idx = tid; idx < 6 * Kz1 * W; idx += nt) {
        int w = idx % W, kz = (idx / W) % Kz1, c = idx / (W * Kz1);
        int kx = kx0 + w;
        bool ok = kx < LX;
        cp_async_real<T>(&Ks[(c * Kz1 + kz) * W + w], ok ? &a.K[c * nk + ((long long)kz * Ky1 + ky) * Kx1 + kx] : a.K, ok);
    }
    if (kx0 == 0) {
        for (int idx = tid; idx < 6 * Kz1; idx += nt) {
            int kz = idx % Kz1, c = idx / Kz1;
            cp_async_real<T>(&Kn[c * Kz1 + kz], &a.K[c * nk + ((long long)kz * Ky1 + ky) * Kx1 + LX], true);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int tpl = a.pz.tpl;
    const int gp = tid / (W * tpl), l = tid % W, t = (tid / W) % tpl;
    const bool act = gp < np;
    const int gq = act ? gp : 0;
    fft_line<T, false, false>(sm + ((0 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    fft_line<T, false, false>(sm + ((1 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    fft_line<T, false, false>(sm + ((2 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    // product with mirror signs (KernelMultiplication_3D_line, DemagKernel.cpp:85)
    for (int idx = tid; idx < np * Nz * W; idx += nt) {
        int w = idx % W, kz = (idx / W) % Nz, p = idx / (W * Nz);
        int kx = kx0 + w;
        if (kx >= LX) continue;
        int akz = kz <= Nz / 2 ? kz : Nz - kz;
        T sz = kz <= Nz / 2 ? (T)1 : (T)-1;
        if (kx == 0) {
            // pair (p, kz) <-> (mirror pencil, -kz); representatives: p == 0 (all kz) when two pencils,
            // kz <= Nz/2 when the pencil is its own mirror
            if (p == 1) continue;
            if (single && kz > Nz / 2) continue;
            int pm = single ? 0 : 1;
            int kzm = (Nz - kz) % Nz;
            cpx<T> A[3], B[3], Ap[3], Bp[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                cpx<T> C = S(c, 0, kz, w), cc = conj(S(c, pm, kzm, w));
                A[c] = cscale(C + cc, (T)0.5);
                B[c] = cscale(mul_mi(C - cc), (T)0.5);
            }
            T k0[6] = {Ks[(0 * Kz1 + akz) * W + w], Ks[(1 * Kz1 + akz) * W + w], Ks[(2 * Kz1 + akz) * W + w],
                       Ks[(3 * Kz1 + akz) * W + w], sz * Ks[(4 * Kz1 + akz) * W + w], sz * Ks[(5 * Kz1 + akz) * W + w]};
            T kn[6] = {Kn[0 * Kz1 + akz], Kn[1 * Kz1 + akz], Kn[2 * Kz1 + akz],
                       Kn[3 * Kz1 + akz], sz * Kn[4 * Kz1 + akz], sz * Kn[5 * Kz1 + akz]};
            kapply<T>(k0, A, Ap);
            kapply<T>(kn, B, Bp);
            bool self = single && (kzm == kz);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                S(c, 0, kz, w) = Ap[c] + mul_i(Bp[c]);
                if (!self) S(c, pm, kzm, w) = conj(Ap[c]) + mul_i(conj(Bp[c]));
            }
        } else {
            T sy = (p == 0) ? (T)1 : (T)-1;
            T k[6] = {Ks[(0 * Kz1 + akz) * W + w], Ks[(1 * Kz1 + akz) * W + w], Ks[(2 * Kz1 + akz) * W + w],
                      sy * Ks[(3 * Kz1 + akz) * W + w], sz * Ks[(4 * Kz1 + akz) * W + w],
                      sy * sz * Ks[(5 * Kz1 + akz) * W + w]};
            cpx<T> m[3], h[3];
#pragma unroll
            for (int c = 0; c < 3; c++) m[c] = S(c, p, kz, w);
            kapply<T>(k, m, h);
#pragma unroll
            for (int c = 0; c < 3; c++) S(c, p, kz, w) = h[c];
        }
    }
    __syncthreads();
    fft_line<T, false, true>(sm + ((0 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    fft_line<T, false, true>(sm + ((1 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    fft_line<T, false, true>(sm + ((2 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    for (int idx = tid; idx < 3 * np * nz * W; idx += nt) {
        int w = idx % W, e = (idx / W) % nz, cp = idx / (W * nz);
        int c = cp / np, p = cp % np;
        int kyp = p ? kym : ky, kx = kx0 + w;
        if (kx < LX) a.S2[(((long long)c * nz + e) * Ny + kyp) * LX + kx] = S(c, p, e, w);
    }
}

// ------------------------------------------------------------------------------ launchers
template <typename KF>
static int launch_common(KF kern, dim3 grid, int nt, size_t smem, cudaStream_t s)
{
    if (nt > 1024 || nt < 1) return 101;
    if (smem > 227 * 1024) return 102;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}

template <typename T> int launch_ymid2d(const YZArgs<T> &a, cudaStream_t s)
{
    int nt = a.W * a.py.tpl;
    if (nt < 32) nt = 32;
    if (nt > bm_lb<T>::v) return 103;
    size_t smem = ymid2d_smem<T>(a.Ny, a.W);
    dim3 grid((a.LX + a.W - 1) / a.W);
    int rc = launch_common(k_ymid2d<T>, grid, nt, smem, s);
    if (rc) return rc;
    k_ymid2d<T><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T> int launch_yfwd(const YZArgs<T> &a, cudaStream_t s)
{
    int nt = a.W * a.py.tpl;
    if (nt < 32) nt = 32;
    if (nt > bm_lb<T>::v) return 103;
    size_t smem = (size_t)a.Ny * a.W * sizeof(cpx<T>);
    dim3 grid((a.LX + a.W - 1) / a.W, a.nz, 3);
    int rc = launch_common(k_ypass3d<T, false>, grid, nt, smem, s);
    if (rc) return rc;
    k_ypass3d<T, false><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T> int launch_yinv(const YZArgs<T> &a, cudaStream_t s)
{
    int nt = a.W * a.py.tpl;
    if (nt < 32) nt = 32;
    if (nt > bm_lb<T>::v) return 103;
    size_t smem = (size_t)a.Ny * a.W * sizeof(cpx<T>);
    dim3 grid((a.LX + a.W - 1) / a.W, a.nz, 3);
    int rc = launch_common(k_ypass3d<T, true>, grid, nt, smem, s);
    if (rc) return rc;
    k_ypass3d<T, true><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T> int launch_zmid(const YZArgs<T> &a, cudaStream_t s)
{
    int nt = 2 * a.W * a.pz.tpl;
    if (nt < 32) nt = 32;
    if (nt > bm_lb<T>::v) return 103;
    size_t smem = zmid_smem<T>(a.Nz, a.W);
    dim3 grid((a.LX + a.W - 1) / a.W, a.Ny / 2 + 1);
    int rc = launch_common(k_zmid<T>, grid, nt, smem, s);
    if (rc) return rc;
    k_zmid<T><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template int launch_ymid2d<float>(const YZArgs<float> &, cudaStream_t);
template int launch_ymid2d<double>(const YZArgs<double> &, cudaStream_t);
template int launch_yfwd<float>(const YZArgs<float> &, cudaStream_t);
template int launch_yfwd<double>(const YZArgs<double> &, cudaStream_t);
template int launch_yinv<float>(const YZArgs<float> &, cudaStream_t);
template int launch_yinv<double>(const YZArgs<double> &, cudaStream_t);
template int launch_zmid<float>(const YZArgs<float> &, cudaStream_t);
template int launch_zmid<double>(const YZArgs<double> &, cudaStream_t);
