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
#include "regfft.cuh"

template <typename T>
__device__ __forceinline__ bool gated_out(const StepState *st, int gate)
{
    if (gate == BM_GATE_ALWAYS || st == nullptr) return false;
    if (gate == BM_GATE_ACCEPTED) return *((volatile const int *)&st->reject_flag) != 0;
    if (gate == BM_GATE_ES || gate == BM_GATE_ES_ACC)
        return *((volatile const int *)&st->es_mode) != 1 ||
               (gate == BM_GATE_ES_ACC && *((volatile const int *)&st->reject_flag) != 0);
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
__device__ __forceinline__ void ymid2d_body(const YZArgs<T> &a, int bx)
{
    extern __shared__ unsigned char smraw[];
    const int W = a.W, Ny = a.Ny, ny = a.ny, LX = a.LX;
    const int Ky1 = Ny / 2 + 1, Kx1 = LX + 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 3 * Ny * W);
    T *Kn = Ks + 4 * Ky1 * W;
    const int kx0 = bx * W;
    const int nt = blockDim.x, tid = threadIdx.x;
    const long long plane = (long long)ny * LX;   // one component (nz == 1)
    const long long nk = (long long)Kx1 * Ky1;
    // thread (column wq, row group g0): W is a power of two and divides the block size
    const int lw = __ffs(W) - 1, wq = tid & (W - 1), g0 = tid >> lw, ng = nt >> lw;
    const int kxq = kx0 + wq;
    const bool okx = kxq < LX;
    for (int c = 0; c < 3; c++)
        for (int e = g0; e < Ny; e += ng) {
            const bool ok = e < ny && okx;
            cp_async_cpx<T>(&sm[(c * Ny + e) * W + wq], ok ? &a.S1[c * plane + (long long)e * LX + kxq] : a.S1, ok);
        }
    for (int c = 0; c < 4; c++)
        for (int ky = g0; ky < Ky1; ky += ng)
            cp_async_real<T>(&Ks[(c * Ky1 + ky) * W + wq], okx ? &a.K[c * nk + (long long)ky * Kx1 + kxq] : a.K, okx);
    if (kx0 == 0) {
        for (int idx = tid; idx < 4 * Ky1; idx += nt) {
            int ky = idx % Ky1, c = idx / Ky1;
            cp_async_real<T>(&Kn[c * Ky1 + ky], &a.K[c * nk + (long long)ky * Kx1 + LX], true);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int tpl = a.py.tpl;
    const int l = wq, t = g0;
    const bool act = t < tpl;
    // three explicit calls: a loop around fft_line defeats register allocation
    fft_line<T, false, false>(sm + 0 * Ny * W + l, W, t, act, a.py, a.twy);
    fft_line<T, false, false>(sm + 1 * Ny * W + l, W, t, act, a.py, a.twy);
    fft_line<T, false, false>(sm + 2 * Ny * W + l, W, t, act, a.py, a.twy);
    // product: Kxy odd in y (KernelMultiplication_2D_line, DemagKernel.cpp:42)
    for (int ky = g0; ky < Ny; ky += ng) {
        const int w = wq, kx = kxq;
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
    if (okx)
        for (int cc = 0; cc < 3; cc++)
            for (int e = g0; e < ny; e += ng) a.S1[cc * plane + (long long)e * LX + kxq] = sm[(cc * Ny + e) * W + wq];
}

template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ymid2d(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    ymid2d_body<T>(a, blockIdx.x);
}

// many meshes in one launch: work item (mesh, column tile); every mesh shares the step state
template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ymid2d_batch(const YZArgs<T> *__restrict__ args, const int2 *__restrict__ work,
                                                                 int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    ymid2d_body<T>(args[it.x], it.y);
}

// ------------------------------------------------------------------------------ 3D y passes
template <typename T, bool INV>
__device__ __forceinline__ void ypass3d_body(const YZArgs<T> &a, int bx, int z, int c)
{
    extern __shared__ unsigned char smraw[];
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    const int W = a.W, Ny = a.Ny, ny = a.ny, LX = a.LX, nz = a.nz;
    const int kx0 = bx * W;
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
    // thread (column wq, row group g0): W is a power of two and divides the block size
    const int lw = __ffs(W) - 1, wq = tid & (W - 1), g0 = tid >> lw, ng = nt >> lw;
    const int kxq = kx0 + wq;
    const bool okx = kxq < LX;
    for (int e = g0; e < Ny; e += ng) {
        const bool ok = e < nin && okx;
        cp_async_cpx<T>(&sm[e * W + wq], ok ? &src[(long long)e * LX + kxq] : src, ok);
    }
    cp_async_wait_all();
    __syncthreads();
    const int tpl = a.py.tpl;
    fft_line<T, false, INV>(sm + wq, W, g0, g0 < tpl, a.py, a.twy);
    if (okx)
        for (int e = g0; e < nout; e += ng) dst[(long long)e * LX + kxq] = sm[e * W + wq];
}

template <typename T, bool INV>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ypass3d(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    ypass3d_body<T, INV>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// many meshes in one launch: work item (mesh, column tile + W-columns count * (z + nz * component))
template <typename T, bool INV>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ypass3d_batch(const YZArgs<T> *__restrict__ args, const int2 *__restrict__ work,
                                                                  int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    const YZArgs<T> &a = args[it.x];
    const int nbx = (a.LX + a.W - 1) / a.W;
    const int bx = it.y % nbx, r = it.y / nbx;
    ypass3d_body<T, INV>(a, bx, r % a.nz, r / a.nz);
}

// ------------------------------------------------------------------------------ 3D z pass + product
// Block: W columns kx0.., the mirror pencils ky and Ny - ky (which share |ky|), 3 components.
// smem: data [3][2][Nz][W] complex, kernel tile [6][Kz1][W] real at |ky|, column-0 Nyquist
// kernel [6][Kz1] real.
template <typename T>
__device__ __forceinline__ void zmid_body(const YZArgs<T> &a, int bx, int ky)
{
    extern __shared__ unsigned char smraw[];
    const int W = a.W, Ny = a.Ny, Nz = a.Nz, nz = a.nz, LX = a.LX;
    const int Kx1 = LX + 1, Ky1 = Ny / 2 + 1, Kz1 = Nz / 2 + 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 6 * Nz * W);
    T *Kn = Ks + 6 * Kz1 * W;
    const int kx0 = bx * W;
    const int kym = (Ny - ky) % Ny;
    const bool single = (ky == kym);
    const int nt = blockDim.x, tid = threadIdx.x;
    const long long nk = (long long)Kx1 * Ky1 * Kz1;
    auto S = [&](int c, int p, int e, int w) -> cpx<T> & { return sm[((c * 2 + p) * Nz + e) * W + w]; };
    const int np = single ? 1 : 2;
    // thread (column wq, row group g0): W is a power of two and divides the block size
    const int lw = __ffs(W) - 1, wq = tid & (W - 1), g0 = tid >> lw, ng = nt >> lw;
    const int kxq = kx0 + wq;
    const bool okx = kxq < LX;
    for (int c = 0; c < 3; c++)
        for (int p = 0; p < np; p++) {
            const int kyp = p ? kym : ky;
            for (int e = g0; e < Nz; e += ng) {
                const bool ok = e < nz && okx;
                cp_async_cpx<T>(&S(c, p, e, wq), ok ? &a.S2[(((long long)c * nz + e) * Ny + kyp) * LX + kxq] : a.S2, ok);
            }
        }
    for (int c = 0; c < 6; c++)
        for (int kz = g0; kz < Kz1; kz += ng)
            cp_async_real<T>(&Ks[(c * Kz1 + kz) * W + wq], okx ? &a.K[c * nk + ((long long)kz * Ky1 + ky) * Kx1 + kxq] : a.K, okx);
    if (kx0 == 0) {
        for (int idx = tid; idx < 6 * Kz1; idx += nt) {
            int kz = idx % Kz1, c = idx / Kz1;
            cp_async_real<T>(&Kn[c * Kz1 + kz], &a.K[c * nk + ((long long)kz * Ky1 + ky) * Kx1 + LX], true);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int tpl = a.pz.tpl;
    const int gp = g0 / tpl, l = wq, t = g0 - gp * tpl;
    const bool act = gp < np;
    const int gq = act ? gp : 0;
    fft_line<T, false, false>(sm + ((0 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    fft_line<T, false, false>(sm + ((1 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    fft_line<T, false, false>(sm + ((2 * 2 + gq) * Nz) * W + l, W, t, act, a.pz, a.twz);
    // product with mirror signs (KernelMultiplication_3D_line, DemagKernel.cpp:85)
    for (int r = g0; r < np * Nz; r += ng) {
        const int p = r >= Nz ? 1 : 0, kz = r - p * Nz;
        const int w = wq, kx = kxq;
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
    if (okx)
        for (int c = 0; c < 3; c++)
            for (int p = 0; p < np; p++) {
                const int kyp = p ? kym : ky;
                for (int e = g0; e < nz; e += ng) a.S2[(((long long)c * nz + e) * Ny + kyp) * LX + kxq] = S(c, p, e, wq);
            }
}

template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    zmid_body<T>(a, blockIdx.x, blockIdx.y);
}

// many meshes in one launch: work item (mesh, column tile + W-columns count * ky)
template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid_batch(const YZArgs<T> *__restrict__ args, const int2 *__restrict__ work,
                                                               int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    const YZArgs<T> &a = args[it.x];
    const int nbx = (a.LX + a.W - 1) / a.W;
    zmid_body<T>(a, it.y % nbx, it.y / nbx);
}

// ------------------------------------------------------------------------------ 3D z pass, register FFT
// Compile-time Nz (<= 64): one thread owns one (component, pencil, column) line of Nz points in
// registers. The upper half of the padded input is a compile-time zero and only the first
// Nz/2 inverse outputs are stored, so the zero-padding work folds away. Shared memory only
// carries the forward spectra to the 3x3 product: each thread reads the three components of its
// own (pencil, column) and forms its own output component in registers, so one barrier separates
// the transforms. The kernel tile arrives by cp.async while the forward transforms run (thread
// row j < 6 copies kernel component j for every kz). Thread (c, p, w): w fastest so global loads
// and stores coalesce.
// WC: the tile width as a compile-time constant (0: a.W at run time), so that every shared-memory
// address of the product becomes a base plus an immediate offset
template <typename T, int NZ, int WC>
__device__ __forceinline__ void zmid_reg_body(const YZArgs<T> &a, int bx, int ky)
{
    extern __shared__ unsigned char smraw[];
    const int W = WC ? WC : a.W, Ny = a.Ny, nz = a.nz, LX = a.LX;
    const int lw = WC ? (WC == 32 ? 5 : WC == 16 ? 4 : WC == 8 ? 3 : WC == 4 ? 2 : WC == 2 ? 1 : 0) : __ffs(W) - 1;
    constexpr int KZ1 = NZ / 2 + 1;
    const int Kx1 = LX + 1, Ky1 = Ny / 2 + 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 6 * NZ * W);
    T *Kn = Ks + 6 * KZ1 * W;
    const int kx0 = bx * W;
    const int kym = (Ny - ky) % Ny;
    const bool single = (ky == kym);
    const int np = single ? 1 : 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long nk = (long long)Kx1 * Ky1 * KZ1;
    const long long kzs = (long long)Ky1 * Kx1;   // kz stride of a kernel component
    const int w = tid & (W - 1);
    const int j = tid >> lw;
    const int kx = kx0 + w;
    // kernel tile (async)
    if (j < 6) {
        const bool ok = kx < LX;
        const T *src = a.K + j * nk + (long long)ky * Kx1 + (ok ? kx : 0);
#pragma unroll
        for (int kz = 0; kz < KZ1; kz++) cp_async_real<T>(&Ks[(j * KZ1 + kz) * W + w], src + kz * kzs, ok);
    }
    if (kx0 == 0) {
        for (int idx = tid; idx < 6 * KZ1; idx += nt) {
            int kz = idx % KZ1, c = idx / KZ1;
            cp_async_real<T>(&Kn[c * KZ1 + kz], &a.K[c * nk + kz * kzs + (long long)ky * Kx1 + LX], true);
        }
    }
    // forward transforms in registers
    const int p = j & 1;
    const int c = j >> 1;
    const bool own = (c < 3) && (p < np) && (kx < LX);
    const int kyp = p ? kym : ky;
    const long long gbase = ((long long)c * nz * Ny + kyp) * LX + kx;   // + e * Ny * LX
    const long long gstride = (long long)Ny * LX;
    cpx<T> v[NZ];
#pragma unroll
    for (int e = 0; e < NZ; e++) v[e] = mk<T>(0, 0);
    if (own) {
#pragma unroll
        for (int e = 0; e < NZ / 2; e++)
            if (e < nz) v[e] = a.S2[gbase + e * gstride];
    }
    RegFFT<T, NZ, false>::run(v, a.twz, 1);
    auto S = [&](int cc, int pp, int e) -> cpx<T> { return sm[((cc * 2 + pp) * NZ + e) * W + w]; };
    if (c < 3) {
#pragma unroll
        for (int e = 0; e < NZ; e++) sm[((c * 2 + p) * NZ + e) * W + w] = v[e];
    }
    cp_async_wait_all();
    __syncthreads();
    if (!own) return;
    // row c of the symmetric 3x3 kernel in (xx, yy, zz, xy, xz, yz) order, with the mirror signs
    // of KernelMultiplication_3D_line (DemagKernel.cpp:85): xy odd in y, xz odd in z, yz odd in both
    const int q0 = c == 0 ? 0 : c == 1 ? 3 : 4;
    const int q1 = c == 0 ? 3 : c == 1 ? 1 : 5;
    const int q2 = c == 0 ? 4 : c == 1 ? 5 : 2;
    auto has_y = [](int q) { return q == 3 || q == 5; };
    auto has_z = [](int q) { return q == 4 || q == 5; };
    if (kx != 0) {
        const T sy = p ? (T)-1 : (T)1;
        const T y0 = has_y(q0) ? sy : (T)1, y1 = has_y(q1) ? sy : (T)1, y2 = has_y(q2) ? sy : (T)1;
        const T z0 = has_z(q0) ? (T)-1 : (T)1, z1 = has_z(q1) ? (T)-1 : (T)1, z2 = has_z(q2) ? (T)-1 : (T)1;
#pragma unroll
        for (int kz = 0; kz < NZ; kz++) {
            const int akz = kz <= NZ / 2 ? kz : NZ - kz;
            const bool neg = kz > NZ / 2;
            const T a0 = (neg ? y0 * z0 : y0) * Ks[(q0 * KZ1 + akz) * W + w];
            const T a1 = (neg ? y1 * z1 : y1) * Ks[(q1 * KZ1 + akz) * W + w];
            const T a2 = (neg ? y2 * z2 : y2) * Ks[(q2 * KZ1 + akz) * W + w];
            const cpx<T> m0 = S(0, p, kz), m1 = S(1, p, kz), m2 = S(2, p, kz);
            v[kz] = mk<T>(a0 * m0.x + a1 * m1.x + a2 * m2.x, a0 * m0.y + a1 * m1.y + a2 * m2.y);
        }
    } else {
        // packed column: DC (kernel column 0) + i Nyquist (kernel column LX); the x-odd entries
        // vanish there, and the z sign follows the line's primary kz (p = 0 pencil, kz <= Nz/2
        // for a self-mirrored pencil) so that both mirror halves see the same kernel values. Only
        // the column-0 threads take this path: a rolled loop through their own slots of O keeps it
        // from adding registers to the unrolled path above.
        cpx<T> *O = sm + 6 * NZ * W + ((6 * KZ1 * (W + 1) * sizeof(T) + sizeof(cpx<T>) - 1) / sizeof(cpx<T>)) + (c * 2 + p) * NZ;
        const int pm = single ? 0 : 1 - p;
        const T zq0 = has_z(q0) ? (T)-1 : (T)1, zq1 = has_z(q1) ? (T)-1 : (T)1, zq2 = has_z(q2) ? (T)-1 : (T)1;
#pragma unroll 1
        for (int kz = 0; kz < NZ; kz++) {
            const int kzm = (NZ - kz) % NZ;
            const int akz = kz <= NZ / 2 ? kz : NZ - kz;
            const int kq = single ? (kz <= NZ / 2 ? kz : kzm) : (p == 0 ? kz : kzm);
            const bool neg = kq > NZ / 2;
            cpx<T> A[3], B[3];
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                const cpx<T> C = S(cc, p, kz), cj = conj(S(cc, pm, kzm));
                A[cc] = cscale(C + cj, (T)0.5);
                B[cc] = cscale(mul_mi(C - cj), (T)0.5);
            }
            const T s0 = neg ? zq0 : (T)1, s1 = neg ? zq1 : (T)1, s2 = neg ? zq2 : (T)1;
            const T a0 = s0 * Ks[(q0 * KZ1 + akz) * W + w], a1 = s1 * Ks[(q1 * KZ1 + akz) * W + w],
                    a2 = s2 * Ks[(q2 * KZ1 + akz) * W + w];
            const T b0 = s0 * Kn[q0 * KZ1 + akz], b1 = s1 * Kn[q1 * KZ1 + akz], b2 = s2 * Kn[q2 * KZ1 + akz];
            const cpx<T> Ap = mk<T>(a0 * A[0].x + a1 * A[1].x + a2 * A[2].x, a0 * A[0].y + a1 * A[1].y + a2 * A[2].y);
            const cpx<T> Bp = mk<T>(b0 * B[0].x + b1 * B[1].x + b2 * B[2].x, b0 * B[0].y + b1 * B[1].y + b2 * B[2].y);
            O[kz] = Ap + mul_i(Bp);
        }
#pragma unroll
        for (int kz = 0; kz < NZ; kz++) v[kz] = O[kz];
    }
    RegFFT<T, NZ, true>::run(v, a.twz, 1);
#pragma unroll
    for (int e = 0; e < NZ / 2; e++)
        if (e < nz) a.S2[gbase + e * gstride] = v[e];
}

// L2 prefetch of the bytes p0 .. p1 of one row segment (at most two 128-byte lines)
__device__ __forceinline__ void pf_segment(const void *p0, const void *p1)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p0));
    if ((reinterpret_cast<uintptr_t>(p0) >> 7) != (reinterpret_cast<uintptr_t>(p1) >> 7))
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p1));
}

template <typename T, int NZ, int WC>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid_reg(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    zmid_reg_body<T, NZ, WC>(a, blockIdx.x, blockIdx.y);
}

// many meshes with the same Nz in one launch: work item (mesh, column tile + W-columns count * ky)
template <typename T, int NZ>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid_reg_batch(const YZArgs<T> *__restrict__ args,
                                                                   const int2 *__restrict__ work, int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    const YZArgs<T> &a = args[it.x];
    const int nbx = (a.LX + a.W - 1) / a.W;
    zmid_reg_body<T, NZ, 0>(a, it.y % nbx, it.y / nbx);
}

template <typename T, int NZ, int WC>
static int launch_zmid_reg_w(const YZArgs<T> &a, cudaStream_t s)
{
    int nt = (6 * a.W + 31) & ~31;
    if (nt > bm_lb<T>::v) return 104;
    size_t smem = zmid_reg_smem<T>(NZ, a.W);
    if (smem > 200 * 1024) return 105;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_zmid_reg<T, NZ, WC>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    dim3 grid((a.LX + a.W - 1) / a.W, a.Ny / 2 + 1);
    k_zmid_reg<T, NZ, WC><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T, int NZ>
static int launch_zmid_reg(const YZArgs<T> &a, cudaStream_t s)
{
    switch (a.W) {
    case 8: return launch_zmid_reg_w<T, NZ, 8>(a, s);
    case 16: return launch_zmid_reg_w<T, NZ, 16>(a, s);
    case 32: return launch_zmid_reg_w<T, NZ, 32>(a, s);
    default: return launch_zmid_reg_w<T, NZ, 0>(a, s);
    }
}

// lengths with a register z pass
bool zmid_has_reg(int Nz)
{
    return Nz == 4 || Nz == 6 || Nz == 8 || Nz == 12 || Nz == 16 || Nz == 24 || Nz == 32 || Nz == 48 || Nz == 64;
}

// ------------------------------------------------------------------------------ 3D z pass, parity split
// The register z pass with each pencil's even and odd kz in two threads, so a thread holds Nz/2
// values instead of Nz (fewer registers, twice the resident warps). With the upper half of the
// padded input zero, X[2k + h] = DFT_{Nz/2}( x[e] w_Nz^(e h) )[k] for parity h; each thread forms
// its own output component for its Nz/2 values of kz from the shared forward spectra, and inverts:
// z_h[e] = w_Nz^(-e h) IDFT_{Nz/2}(Y_h)[e]; the pencil's inverse is z_0 + z_1, each thread adding
// half of the outputs through shared memory. The block is two groups of whole warps, one per
// parity (G threads each: the 6 W threads (c, p, w), w fastest, rounded up to warps), so both
// parities run compile-time code paths. Shared memory and the kernel tile are those of
// zmid_reg_body.
template <typename T, int NZ, int HP>
__device__ __forceinline__ void zpar_forward(const YZArgs<T> &a, cpx<T> *v, bool own, long long gbase, long long gstride, int nz)
{
    constexpr int H = NZ / 2;
#pragma unroll
    for (int e = 0; e < H; e++) v[e] = mk<T>(0, 0);
    if (own) {
#pragma unroll
        for (int e = 0; e < H; e++)
            if (e < nz) v[e] = a.S2[gbase + e * gstride];
    }
    if (HP) {
#pragma unroll
        for (int e = 1; e < H; e++) v[e] = cmul(v[e], a.twz[e]);
    }
    RegFFT<T, H, false>::run(v, a.twz, 2);
}

template <typename T, int NZ, int HP, int WC>
__device__ __forceinline__ void zpar_product(const YZArgs<T> &a, cpx<T> *v, const cpx<T> *sm, const T *Ks, const T *Kn, cpx<T> *O,
                                             int c, int p, int w, int kx, bool single, int W)
{
    constexpr int H = NZ / 2, KZ1 = NZ / 2 + 1;
    auto S = [&](int cc, int pp, int e) -> cpx<T> { return sm[((cc * 2 + pp) * NZ + e) * W + w]; };
    const int q0 = c == 0 ? 0 : c == 1 ? 3 : 4;
    const int q1 = c == 0 ? 3 : c == 1 ? 1 : 5;
    const int q2 = c == 0 ? 4 : c == 1 ? 5 : 2;
    auto has_y = [](int q) { return q == 3 || q == 5; };
    auto has_z = [](int q) { return q == 4 || q == 5; };
    if (kx != 0) {
        const T sy = p ? (T)-1 : (T)1;
        const T y0 = has_y(q0) ? sy : (T)1, y1 = has_y(q1) ? sy : (T)1, y2 = has_y(q2) ? sy : (T)1;
        const T z0 = has_z(q0) ? (T)-1 : (T)1, z1 = has_z(q1) ? (T)-1 : (T)1, z2 = has_z(q2) ? (T)-1 : (T)1;
#pragma unroll
        for (int k = 0; k < H; k++) {
            const int kz = 2 * k + HP;
            const int akz = kz <= NZ / 2 ? kz : NZ - kz;
            const bool neg = kz > NZ / 2;
            const T a0 = (neg ? y0 * z0 : y0) * Ks[(q0 * KZ1 + akz) * W + w];
            const T a1 = (neg ? y1 * z1 : y1) * Ks[(q1 * KZ1 + akz) * W + w];
            const T a2 = (neg ? y2 * z2 : y2) * Ks[(q2 * KZ1 + akz) * W + w];
            const cpx<T> m0 = S(0, p, kz), m1 = S(1, p, kz), m2 = S(2, p, kz);
            v[k] = mk<T>(a0 * m0.x + a1 * m1.x + a2 * m2.x, a0 * m0.y + a1 * m1.y + a2 * m2.y);
        }
    } else {
        // the packed column (as zmid_reg_body), for this thread's kz
        const int pm = single ? 0 : 1 - p;
        const T zq0 = has_z(q0) ? (T)-1 : (T)1, zq1 = has_z(q1) ? (T)-1 : (T)1, zq2 = has_z(q2) ? (T)-1 : (T)1;
#pragma unroll 1
        for (int k = 0; k < H; k++) {
            const int kz = 2 * k + HP;
            const int kzm = (NZ - kz) % NZ;
            const int akz = kz <= NZ / 2 ? kz : NZ - kz;
            const int kq = single ? (kz <= NZ / 2 ? kz : kzm) : (p == 0 ? kz : kzm);
            const bool neg = kq > NZ / 2;
            cpx<T> A[3], B[3];
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                const cpx<T> C = S(cc, p, kz), cj = conj(S(cc, pm, kzm));
                A[cc] = cscale(C + cj, (T)0.5);
                B[cc] = cscale(mul_mi(C - cj), (T)0.5);
            }
            const T s0 = neg ? zq0 : (T)1, s1 = neg ? zq1 : (T)1, s2 = neg ? zq2 : (T)1;
            const T a0 = s0 * Ks[(q0 * KZ1 + akz) * W + w], a1 = s1 * Ks[(q1 * KZ1 + akz) * W + w],
                    a2 = s2 * Ks[(q2 * KZ1 + akz) * W + w];
            const T b0 = s0 * Kn[q0 * KZ1 + akz], b1 = s1 * Kn[q1 * KZ1 + akz], b2 = s2 * Kn[q2 * KZ1 + akz];
            const cpx<T> Ap = mk<T>(a0 * A[0].x + a1 * A[1].x + a2 * A[2].x, a0 * A[0].y + a1 * A[1].y + a2 * A[2].y);
            const cpx<T> Bp = mk<T>(b0 * B[0].x + b1 * B[1].x + b2 * B[2].x, b0 * B[0].y + b1 * B[1].y + b2 * B[2].y);
            O[kz] = Ap + mul_i(Bp);
        }
#pragma unroll
        for (int k = 0; k < H; k++) v[k] = O[2 * k + HP];
    }
    RegFFT<T, H, true>::run(v, a.twz, 2);
    if (HP) {
#pragma unroll
        for (int e = 1; e < H; e++) {
            cpx<T> t = a.twz[e];
            t.y = -t.y;
            v[e] = cmul(v[e], t);
        }
    }
}

template <typename T, int NZ, int WC>
__device__ __forceinline__ void zpar_body(const YZArgs<T> &a, int bx, int ky)
{
    extern __shared__ unsigned char smraw[];
    constexpr int H = NZ / 2, KZ1 = NZ / 2 + 1;
    const int W = WC, Ny = a.Ny, nz = a.nz, LX = a.LX;
    constexpr int lw = WC == 16 ? 4 : 3;
    const int Kx1 = LX + 1, Ky1 = Ny / 2 + 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 6 * NZ * W);
    T *Kn = Ks + 6 * KZ1 * W;
    const int kx0 = bx * W;
    const int kym = (Ny - ky) % Ny;
    const bool single = (ky == kym);
    const int np = single ? 1 : 2;
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long nk = (long long)Kx1 * Ky1 * KZ1;
    const long long kzs = (long long)Ky1 * Kx1;
    constexpr int G = ((6 * WC + 31) / 32) * 32;   // threads per parity group
    const int h = tid >= G ? 1 : 0;                 // warp-uniform
    const int r = tid - h * G;
    const int w = r & (W - 1);
    const int jj = r >> lw;                         // (c, p) row, 0 .. 5 (idle rows past 5)
    const int kx = kx0 + w;
    if (h == 0 && jj < 6) {
        const bool ok = kx < LX;
        const T *src = a.K + jj * nk + (long long)ky * Kx1 + (ok ? kx : 0);
#pragma unroll
        for (int kz = 0; kz < KZ1; kz++) cp_async_real<T>(&Ks[(jj * KZ1 + kz) * W + w], src + kz * kzs, ok);
    }
    if (kx0 == 0) {
        for (int idx = tid; idx < 6 * KZ1; idx += nt) {
            int kz = idx % KZ1, c = idx / KZ1;
            cp_async_real<T>(&Kn[c * KZ1 + kz], &a.K[c * nk + kz * kzs + (long long)ky * Kx1 + LX], true);
        }
    }
    const int p = jj & 1, c = jj >> 1;
    const bool own = (jj < 6) && (p < np) && (kx < LX);
    const int kyp = p ? kym : ky;
    const long long gbase = ((long long)c * nz * Ny + kyp) * LX + kx;
    const long long gstride = (long long)Ny * LX;
    cpx<T> v[H];
    if (h == 0) zpar_forward<T, NZ, 0>(a, v, own, gbase, gstride, nz);
    else zpar_forward<T, NZ, 1>(a, v, own, gbase, gstride, nz);
    if (jj < 6) {
#pragma unroll
        for (int k = 0; k < H; k++) sm[((c * 2 + p) * NZ + 2 * k + h) * W + w] = v[k];
    }
    cp_async_wait_all();
    __syncthreads();
    cpx<T> *O = sm + 6 * NZ * W + ((6 * KZ1 * (W + 1) * sizeof(T) + sizeof(cpx<T>) - 1) / sizeof(cpx<T>)) + (c * 2 + p) * NZ;
    if (own) {
        if (h == 0) zpar_product<T, NZ, 0, WC>(a, v, sm, Ks, Kn, O, c, p, w, kx, single, W);
        else zpar_product<T, NZ, 1, WC>(a, v, sm, Ks, Kn, O, c, p, w, kx, single, W);
    }
    __syncthreads();   // every spectrum read before the slab takes the halves
    // z_0 + z_1: parity h keeps outputs [h H/2, (h + 1) H/2) and hands the other half to its partner
    // through its (c, p) slab of the spectra (slots e of column w)
    cpx<T> *X = sm + (size_t)(c * 2 + p) * NZ * W + w;
    if (own) {
#pragma unroll
        for (int e = 0; e < H; e++)
            if ((e < H / 2) == (h == 1)) X[e * W] = v[e];
    }
    __syncthreads();
    if (own) {
#pragma unroll
        for (int e = 0; e < H; e++) {
            if ((e < H / 2) != (h == 0)) continue;
            const cpx<T> o = X[e * W];
            if (e < nz) a.S2[gbase + e * gstride] = v[e] + o;
        }
    }
}

template <typename T, int NZ, int WC>
__global__ void __launch_bounds__(bm_lb<T>::v) k_zmid_par(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    zpar_body<T, NZ, WC>(a, blockIdx.x, blockIdx.y);
}

// whether the parity-split z pass applies: Nz 12, 16, 24, 32, 48 or 64, a tile width of 8 or 16
bool zmid_has_par(int Nz, int W)
{
    return (Nz == 12 || Nz == 16 || Nz == 24 || Nz == 32 || Nz == 48 || Nz == 64) && (W == 8 || W == 16);
}

template <typename T, int NZ, int WC>
static int launch_zmid_par_w(const YZArgs<T> &a, cudaStream_t s)
{
    const int nt = 2 * (((6 * WC + 31) / 32) * 32);   // two parity groups of whole warps
    if (nt > bm_lb<T>::v) return 104;
    size_t smem = zmid_reg_smem<T>(NZ, WC);
    if (smem > 200 * 1024) return 105;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_zmid_par<T, NZ, WC>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    dim3 grid((a.LX + WC - 1) / WC, a.Ny / 2 + 1);
    k_zmid_par<T, NZ, WC><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T, int NZ>
static int launch_zmid_par(const YZArgs<T> &a, cudaStream_t s)
{
    switch (a.W) {
    case 8: return launch_zmid_par_w<T, NZ, 8>(a, s);
    case 16: return launch_zmid_par_w<T, NZ, 16>(a, s);
    default: return 104;
    }
}

// ------------------------------------------------------------------------------ 3D y passes, two-level register FFT
// Ny = P * Q (P <= Q <= 32). Stage 1: thread (w, n1) holds x[n1 + P n2], n2 < Q, in registers,
// does DFT_Q, twiddles by w_Ny^(n1 k2) and writes u[k2][n1] to shared memory. Stage 2: thread
// (w, k2) reads u[k2][.], does DFT_P and owns X[k2 + Q k1]. Forward: the input rows >= ny are
// compile-time zeros (n2 >= Q/2). Inverse: only rows < ny (k1 < P/2) are written. One shared
// transpose per transform instead of one per radix pass; no runtime division.
template <typename T, int P, int Q, bool INV>
__device__ __forceinline__ void ypass_reg_body(const YZArgs<T> &a, int bx, int z, int c)
{
    extern __shared__ unsigned char smraw[];
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    constexpr int L = P * Q;
    const int W = a.W, ny = a.ny, LX = a.LX, nz = a.nz;
    const int lw = __ffs(W) - 1;
    const int kx0 = bx * W;
    const int tid = threadIdx.x;
    const int w = tid & (W - 1), r = tid >> lw;
    const int kx = kx0 + w;
    const bool colok = kx < LX;
    const cpx<T> *src;
    cpx<T> *dst;
    if (!INV) {
        src = a.S1 + ((long long)c * nz + z) * ny * LX + kx;
        dst = a.S2 + ((long long)c * nz + z) * L * LX + kx;
    } else {
        src = a.S2 + ((long long)c * nz + z) * L * LX + kx;
        dst = a.S1 + ((long long)c * nz + z) * ny * LX + kx;
    }
    cpx<T> v[Q];
    if (r < P) {
        const int n1 = r;
#pragma unroll
        for (int n2 = 0; n2 < Q; n2++) {
            v[n2] = mk<T>(0, 0);
            const int e = n1 + P * n2;
            if (!INV) {
                if (n2 < Q / 2 && colok && e < ny) v[n2] = src[(long long)e * LX];
            } else {
                if (colok) v[n2] = src[(long long)e * LX];
            }
        }
        RegFFT<T, Q, INV>::run(v, a.twy, P);
#pragma unroll
        for (int k2 = 0; k2 < Q; k2++) {
            cpx<T> t = v[k2];
            if (k2 > 0 && n1 > 0) {
                cpx<T> tw = a.twy[n1 * k2];
                if (INV) tw.y = -tw.y;
                t = cmul(t, tw);
            }
            sm[(k2 * P + n1) * W + w] = t;
        }
    }
    __syncthreads();
    if (r < Q) {
        const int k2 = r;
        cpx<T> u[P];
#pragma unroll
        for (int n1 = 0; n1 < P; n1++) u[n1] = sm[(k2 * P + n1) * W + w];
        RegFFT<T, P, INV>::run(u, a.twy, Q);
        if (colok) {
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) {
                const int e = k2 + Q * k1;
                if (!INV) dst[(long long)e * LX] = u[k1];
                else if (k1 < P / 2 && e < ny) dst[(long long)e * LX] = u[k1];
            }
        }
    }
}

// Look-ahead L2 prefetch of a y pass: the block one residency wave ahead in launch order (a.pf_ahead
// = blocks of the grid resident at once) starts about when this one ends, so this block asks L2 for
// that block's input column tile (rows rows of the plane at stride LX, columns kx0 .. kx1) before its
// own loads. Its loads then hit L2, and DRAM keeps streaming while the resident blocks transform.
// Every prefetched address lies inside the input plane.
template <typename T, bool INV>
__device__ __forceinline__ void ypass_prefetch_ahead(const YZArgs<T> &a, int L)
{
    const long long gx = gridDim.x, gy = gridDim.y;
    const long long nxt = blockIdx.x + gx * (blockIdx.y + gy * blockIdx.z) + a.pf_ahead;
    if (nxt >= gx * gy * gridDim.z) return;
    const int bx = (int)(nxt % gx);
    const long long rest = nxt / gx;
    const int z = (int)(rest % gy), c = (int)(rest / gy);
    const int LX = a.LX, rows = INV ? L : a.ny;
    const int kx0 = bx * a.W, kx1 = min(kx0 + a.W, LX) - 1;
    const cpx<T> *base = (INV ? a.S2 : a.S1) + ((long long)c * a.nz + z) * rows * LX;
    for (int e = threadIdx.x; e < rows; e += blockDim.x) {
        pf_segment(base + (long long)e * LX + kx0, base + (long long)e * LX + kx1);
    }
}

template <typename T, int P, int Q, bool INV>
__global__ void __launch_bounds__(yreg_maxt<T>::v) k_ypass_reg(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    if (a.pf_ahead > 0) ypass_prefetch_ahead<T, INV>(a, P * Q);
    ypass_reg_body<T, P, Q, INV>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// many meshes with the same Ny in one launch: work item (mesh, column tile + W-columns count *
// (z + nz * component))
template <typename T, int P, int Q, bool INV>
__global__ void __launch_bounds__(yreg_maxt<T>::v) k_ypass_reg_batch(const YZArgs<T> *__restrict__ args,
                                                                    const int2 *__restrict__ work, int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    const YZArgs<T> &a = args[it.x];
    const int nbx = (a.LX + a.W - 1) / a.W;
    const int bx = it.y % nbx, r = it.y / nbx;
    ypass_reg_body<T, P, Q, INV>(a, bx, r % a.nz, r / a.nz);
}

template <int L> struct ysplit {
    // P <= Q, both <= 32
    static constexpr int q = (L >= 1024) ? 32 : (L >= 256) ? 16 : (L >= 64) ? 8 : (L >= 16) ? 4 : 2;
    static constexpr int p = L / q;
};

template <typename T, int L, bool INV>
static int launch_ypass_reg(const YZArgs<T> &a, cudaStream_t s)
{
    constexpr int P = ysplit<L>::p, Q = ysplit<L>::q;
    int nt = a.W * (P > Q ? P : Q);
    if (nt > yreg_maxt<T>::v) return 106;
    if (nt < 32) nt = 32;
    size_t smem = (size_t)L * a.W * sizeof(cpx<T>);
    if (smem > 200 * 1024) return 107;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_ypass_reg<T, P, Q, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    dim3 grid((a.LX + a.W - 1) / a.W, a.nz, 3);
    YZArgs<T> b = a;
    b.pf_ahead = resident_blocks(k_ypass_reg<T, P, Q, INV>, nt, smem);
    k_ypass_reg<T, P, Q, INV><<<grid, nt, smem, s>>>(b);
    return (int)cudaGetLastError();
}

// ------------------------------------------------------------------------------ 2D y pass, two-level register FFT
// Ny = P * Q (as k_ypass_reg). Block: W columns x 3 components x R = max(P, Q) threads, w fastest.
// Forward: stage 1 reads the S1 rows straight from global memory (rows >= ny are zeros, those >=
// Ny / 2 fold away), one shared transpose, stage 2 leaves the spectrum in the shared tile
// [3][Ny][W] in natural order. The 2D kernel product runs on the tile exactly as in the generic
// kernel (KernelMultiplication_2D_line, DemagKernel.cpp:42). Inverse: stage 1 from the tile, one
// shared transpose, stage 2 writes rows < ny to S1.
// stage 1 of the two-level y transform on values already in registers: DFT_Q of x[n1 + P n2],
// twiddle, and the transposed store u[k2][n1] into this component's tile column (col = tile + w)
template <typename T, int P, int Q, bool INV>
__device__ __forceinline__ void y2d_stage1(const YZArgs<T> &a, cpx<T> *col, cpx<T> (&v)[Q], int n1, int W)
{
    RegFFT<T, Q, INV>::run(v, a.twy, P);
#pragma unroll
    for (int k2 = 0; k2 < Q; k2++) {
        cpx<T> t = v[k2];
        if (k2 > 0 && n1 > 0) {
            cpx<T> tw = a.twy[n1 * k2];
            if (INV) tw.y = -tw.y;
            t = cmul(t, tw);
        }
        col[(k2 * P + n1) * W] = t;
    }
}

template <typename T, int P, int Q>
__device__ __forceinline__ void ymid2d_reg_body(const YZArgs<T> &a, int bx)
{
    extern __shared__ unsigned char smraw[];
    constexpr int Ny = P * Q, R = P > Q ? P : Q, Ky1 = Ny / 2 + 1;
    const int W = a.W, ny = a.ny, LX = a.LX;
    const int Kx1 = LX + 1;
    const int lw = __ffs(W) - 1;
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    T *Ks = reinterpret_cast<T *>(sm + 3 * Ny * W);
    T *Kn = Ks + 4 * Ky1 * W;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int kx0 = bx * W;
    const int w = tid & (W - 1), g = tid >> lw, ng = nt >> lw;
    const int r = g % R, c = g / R;   // line component and row thread
    const int kx = kx0 + w;
    const bool colok = kx < LX;
    const long long plane = (long long)ny * LX;
    const long long nk = (long long)Kx1 * Ky1;
    // kernel tiles (async)
    for (int cc = 0; cc < 4; cc++)
        for (int ky = g; ky < Ky1; ky += ng)
            cp_async_real<T>(&Ks[(cc * Ky1 + ky) * W + w], colok ? &a.K[cc * nk + (long long)ky * Kx1 + kx] : a.K, colok);
    if (kx0 == 0)
        for (int i = tid; i < 4 * Ky1; i += nt) {
            const int ky = i % Ky1, cc = i / Ky1;
            cp_async_real<T>(&Kn[cc * Ky1 + ky], &a.K[cc * nk + (long long)ky * Kx1 + LX], true);
        }
    cp_async_commit();
    cpx<T> *col = sm + (c < 3 ? c : 0) * Ny * W + w;
    const bool line = c < 3;
    // forward stage 1 from the S1 rows (rows >= ny read as zeros; n2 >= Q / 2 are rows >= Ny / 2)
    if (line && r < P) {
        const cpx<T> *src = a.S1 + c * plane + kx;
        cpx<T> v[Q];
#pragma unroll
        for (int n2 = 0; n2 < Q; n2++) {
            const int e = r + P * n2;
            v[n2] = (n2 < Q / 2 && colok && e < ny) ? src[(long long)e * LX] : mk<T>(0, 0);
        }
        y2d_stage1<T, P, Q, false>(a, col, v, r, W);
    }
    __syncthreads();
    {
        cpx<T> u[P];
        if (line && r < Q) {
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) u[n1] = col[(r * P + n1) * W];
            RegFFT<T, P, false>::run(u, a.twy, Q);
        }
        __syncthreads();
        if (line && r < Q) {
#pragma unroll
            for (int k1 = 0; k1 < P; k1++) col[(r + Q * k1) * W] = u[k1];
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // product: Kxy odd in y (KernelMultiplication_2D_line, DemagKernel.cpp:42)
    for (int ky = g; ky < Ny; ky += ng) {
        if (kx >= LX) continue;
        if (kx == 0) {
            if (ky > Ny / 2) continue;
            const int kym = (Ny - ky) % Ny;
            cpx<T> A[3], B[3];
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                const cpx<T> C = sm[(cc * Ny + ky) * W + w], cj = conj(sm[(cc * Ny + kym) * W + w]);
                A[cc] = cscale(C + cj, (T)0.5);
                B[cc] = cscale(mul_mi(C - cj), (T)0.5);
            }
            T k0[6] = {Ks[(0 * Ky1 + ky) * W + w], Ks[(1 * Ky1 + ky) * W + w], Ks[(2 * Ky1 + ky) * W + w],
                       Ks[(3 * Ky1 + ky) * W + w], (T)0, (T)0};
            T kn[6] = {Kn[0 * Ky1 + ky], Kn[1 * Ky1 + ky], Kn[2 * Ky1 + ky], Kn[3 * Ky1 + ky], (T)0, (T)0};
            cpx<T> Ap[3], Bp[3];
            kapply<T>(k0, A, Ap);
            kapply<T>(kn, B, Bp);
#pragma unroll
            for (int cc = 0; cc < 3; cc++) {
                sm[(cc * Ny + ky) * W + w] = Ap[cc] + mul_i(Bp[cc]);
                if (kym != ky) sm[(cc * Ny + kym) * W + w] = conj(Ap[cc]) + mul_i(conj(Bp[cc]));
            }
        } else {
            const int aky = ky <= Ny / 2 ? ky : Ny - ky;
            const T sy = ky <= Ny / 2 ? (T)1 : (T)-1;
            T k[6] = {Ks[(0 * Ky1 + aky) * W + w], Ks[(1 * Ky1 + aky) * W + w], Ks[(2 * Ky1 + aky) * W + w],
                      sy * Ks[(3 * Ky1 + aky) * W + w], (T)0, (T)0};
            cpx<T> m[3], h[3];
#pragma unroll
            for (int cc = 0; cc < 3; cc++) m[cc] = sm[(cc * Ny + ky) * W + w];
            kapply<T>(k, m, h);
#pragma unroll
            for (int cc = 0; cc < 3; cc++) sm[(cc * Ny + ky) * W + w] = h[cc];
        }
    }
    __syncthreads();
    // inverse stage 1: every thread reads its tile values, then the tile is rewritten
    {
        cpx<T> v[Q];
        if (line && r < P) {
#pragma unroll
            for (int n2 = 0; n2 < Q; n2++) v[n2] = col[(r + P * n2) * W];
        }
        __syncthreads();
        if (line && r < P) y2d_stage1<T, P, Q, true>(a, col, v, r, W);
    }
    __syncthreads();
    if (line && r < Q) {
        cpx<T> u[P];
#pragma unroll
        for (int n1 = 0; n1 < P; n1++) u[n1] = col[(r * P + n1) * W];
        RegFFT<T, P, true>::run(u, a.twy, Q);
        if (colok) {
            cpx<T> *dst = a.S1 + c * plane + kx;
#pragma unroll
            for (int k1 = 0; k1 < P / 2; k1++) {
                const int e = r + Q * k1;
                if (e < ny) dst[(long long)e * LX] = u[k1];
            }
        }
    }
}

template <typename T, int P, int Q>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ymid2d_reg(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    ymid2d_reg_body<T, P, Q>(a, blockIdx.x);
}

// many meshes with the same Ny in one launch: work item (mesh, column tile)
template <typename T, int P, int Q>
__global__ void __launch_bounds__(bm_lb<T>::v) k_ymid2d_reg_batch(const YZArgs<T> *__restrict__ args,
                                                                     const int2 *__restrict__ work, int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    ymid2d_reg_body<T, P, Q>(args[it.x], it.y);
}

template <typename T> size_t ymid2d_reg_smem(int Ny, int W) { return ymid2d_smem<T>(Ny, W); }
int ymid2d_reg_threads(int Ny, int W)
{
    int q = (Ny >= 1024) ? 32 : (Ny >= 256) ? 16 : (Ny >= 64) ? 8 : (Ny >= 16) ? 4 : 2;
    int p = Ny / q;
    return 3 * W * (p > q ? p : q);
}

bool ypass_has_reg(int Ny)
{
    return Ny == 8 || Ny == 16 || Ny == 32 || Ny == 64 || Ny == 128 || Ny == 256 || Ny == 512 || Ny == 1024;
}

int ypass_reg_threads(int Ny, int W)
{
    int q = (Ny >= 1024) ? 32 : (Ny >= 256) ? 16 : (Ny >= 64) ? 8 : (Ny >= 16) ? 4 : 2;
    int p = Ny / q;
    return W * (p > q ? p : q);
}

template <typename T, bool INV>
static int launch_ypass_dispatch(const YZArgs<T> &a, cudaStream_t s)
{
    if ((a.W & (a.W - 1)) != 0) return -1;
    switch (a.Ny) {
    case 8: return launch_ypass_reg<T, 8, INV>(a, s);
    case 16: return launch_ypass_reg<T, 16, INV>(a, s);
    case 32: return launch_ypass_reg<T, 32, INV>(a, s);
    case 64: return launch_ypass_reg<T, 64, INV>(a, s);
    case 128: return launch_ypass_reg<T, 128, INV>(a, s);
    case 256: return launch_ypass_reg<T, 256, INV>(a, s);
    case 512: return launch_ypass_reg<T, 512, INV>(a, s);
    case 1024: return launch_ypass_reg<T, 1024, INV>(a, s);
    default: return -1;
    }
}

// ------------------------------------------------------------------------------ 3D y passes, radix-16 Stockham
// Ny = 256 .. 2048. Block: W columns x Ny / 16 threads per column (w fastest), 16 values per
// thread in every pass. The first pass reads its butterfly inputs straight from global memory
// (forward: rows >= ny are zeros, and those >= Ny / 2 fold away at compile time) and the last
// pass writes straight to global memory (inverse: rows < ny only); the passes in between go
// through a shared tile [Ny][W] skewed by 8 elements per 16 rows, so that the stride-16 stores
// of the first pass and the unit-stride accesses of the others are both conflict-free.
__device__ __forceinline__ int ysk(int e, int w, int W) { return e * W + w + ((e >> 4) << 3); }

// Stockham shape of the y transform: power-of-two Ny, 16 values per thread (radix 16, then the rest);
// Ny = 3 * 2^k, 12 values per thread (radix 4, one radix 2 where the power of two is odd, radix 3 last)
template <int L> struct ys_shape {
    static constexpr int V = (L % 3 == 0) ? 12 : 16;
    static constexpr int TPL = L / V;
};
template <int L, int NS> struct ys_radix {
    static constexpr int M = L / NS;
    static constexpr int v = (L % 3) ? (M >= 16 ? 16 : M) : ((M % 4 == 0 && M / 4 >= 3) ? 4 : (M % 2 == 0 && M / 2 >= 3) ? 2 : 3);
};

template <typename T, int L, int NS, bool INV>
__device__ __forceinline__ void ypass_st_pass(cpx<T> *tile, const cpx<T> *src, cpx<T> *dst, int ld, int ny, int t, int w,
                                              int W, bool colok, bool act, const cpx<T> *__restrict__ tw)
{
    constexpr int TPL = ys_shape<L>::TPL;
    constexpr int R = ys_radix<L, NS>::v;
    constexpr int LR = L / R, BPT = LR / TPL, TWS = L / (NS * R);
    constexpr bool FIRST = NS == 1, LAST = NS * R == L;
    cpx<T> v[BPT][R];
    if (act) {
#pragma unroll
        for (int b = 0; b < BPT; b++)
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int e = t + b * TPL + r * LR;
                if (FIRST) {
                    if (!INV) v[b][r] = (2 * r < R && colok && e < ny) ? src[(long long)e * ld] : mk<T>(0, 0);
                    else v[b][r] = colok ? src[(long long)e * ld] : mk<T>(0, 0);
                } else {
                    v[b][r] = tile[ysk(e, w, W)];
                }
            }
    }
    if (!FIRST && !LAST) __syncthreads();   // every load of this pass before any store into the tile
    if (act)
#pragma unroll
    for (int b = 0; b < BPT; b++) {
        const int j = t + b * TPL;
        const int k = j & (NS - 1);
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                cpx<T> wv = tw[r * k * TWS];
                if (INV) wv.y = -wv.y;
                v[b][r] = cmul(v[b][r], wv);
            }
        }
        dftR<T, R, INV>(v[b]);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int e = d + r * NS;
            if (LAST) {
                if (colok && (!INV || e < ny)) dst[(long long)e * ld] = v[b][r];
            } else {
                tile[ysk(e, w, W)] = v[b][r];
            }
        }
    }
    if constexpr (!LAST) {
        __syncthreads();
        ypass_st_pass<T, L, NS * R, INV>(tile, src, dst, ld, ny, t, w, W, colok, act, tw);
    }
}

template <typename T, int L, bool INV>
__device__ __forceinline__ void ypass_st_body(const YZArgs<T> &a, int bx, int z, int c)
{
    extern __shared__ unsigned char smraw[];
    cpx<T> *tile = reinterpret_cast<cpx<T> *>(smraw);
    const int W = a.W, ny = a.ny, LX = a.LX, nz = a.nz;
    const int lw = __ffs(W) - 1;
    const int kx0 = bx * W;
    const int tid = threadIdx.x;
    const int w = tid & (W - 1), t = tid >> lw;
    const bool act = t < ys_shape<L>::TPL;
    const int kx = kx0 + w;
    const bool colok = kx < LX;
    const cpx<T> *src;
    cpx<T> *dst;
    if (!INV) {
        src = a.S1 + ((long long)c * nz + z) * ny * LX + (colok ? kx : 0);
        dst = a.S2 + ((long long)c * nz + z) * L * LX + kx;
    } else {
        src = a.S2 + ((long long)c * nz + z) * L * LX + (colok ? kx : 0);
        dst = a.S1 + ((long long)c * nz + z) * ny * LX + kx;
    }
    ypass_st_pass<T, L, 1, INV>(tile, src, dst, LX, ny, t, w, W, colok, act, a.twy);
}

template <typename T, int L, bool INV>
__global__ void __launch_bounds__(bm_lb<T>::v, sizeof(T) == 4 ? 2 : 1) k_ypass_st(YZArgs<T> a)
{
    if (gated_out<T>(a.st, a.gate)) return;
    ypass_st_body<T, L, INV>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// many meshes with the same Ny in one launch: work item (mesh, column tile + W-columns count *
// (z + nz * component))
template <typename T, int L, bool INV>
__global__ void __launch_bounds__(bm_lb<T>::v, sizeof(T) == 4 ? 2 : 1) k_ypass_st_batch(const YZArgs<T> *__restrict__ args,
                                                                                       const int2 *__restrict__ work, int nwork)
{
    if (gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    const YZArgs<T> &a = args[it.x];
    const int nbx = (a.LX + a.W - 1) / a.W;
    const int bx = it.y % nbx, r = it.y / nbx;
    ypass_st_body<T, L, INV>(a, bx, r % a.nz, r / a.nz);
}

bool ypass_has_st(int Ny)
{
    return Ny == 256 || Ny == 512 || Ny == 1024 || Ny == 2048 || Ny == 192 || Ny == 384 || Ny == 768 || Ny == 1536;
}
int ypass_st_threads(int Ny, int W) { return W * (Ny / (Ny % 3 ? 16 : 12)); }
template <typename T> size_t ypass_st_smem(int Ny, int W) { return ((size_t)Ny * W + (size_t)(Ny / 16) * 8) * sizeof(cpx<T>); }

template <typename T, int L, bool INV>
static int launch_ypass_st(const YZArgs<T> &a, cudaStream_t s)
{
    int nt = a.W * ys_shape<L>::TPL;
    if (nt > bm_lb<T>::v) return 108;
    if (nt % 32) return 108;
    size_t smem = ypass_st_smem<T>(L, a.W);
    if (smem > 200 * 1024) return 109;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_ypass_st<T, L, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    dim3 grid((a.LX + a.W - 1) / a.W, a.nz, 3);
    k_ypass_st<T, L, INV><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <typename T, bool INV>
static int launch_ypass_st_dispatch(const YZArgs<T> &a, cudaStream_t s)
{
    if ((a.W & (a.W - 1)) != 0) return -1;
    switch (a.Ny) {
    case 256: return launch_ypass_st<T, 256, INV>(a, s);
    case 512: return launch_ypass_st<T, 512, INV>(a, s);
    case 1024: return launch_ypass_st<T, 1024, INV>(a, s);
    case 2048: return launch_ypass_st<T, 2048, INV>(a, s);
    case 192: return launch_ypass_st<T, 192, INV>(a, s);
    case 384: return launch_ypass_st<T, 384, INV>(a, s);
    case 768: return launch_ypass_st<T, 768, INV>(a, s);
    case 1536: return launch_ypass_st<T, 1536, INV>(a, s);
    default: return -1;
    }
}

template <typename T, int L, bool INV>
static int launch_ypass_st_batch(const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s)
{
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_ypass_st_batch<T, L, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return 2000 + (int)e;
    }
    k_ypass_st_batch<T, L, INV><<<nwork, nt, smem, s>>>(dargs, dwork, nwork);
    return (int)cudaGetLastError();
}

template <typename T, bool INV>
static int ypass_st_batch_dispatch(int Ny, const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem,
                                   cudaStream_t s)
{
    switch (Ny) {
    case 256: return launch_ypass_st_batch<T, 256, INV>(dargs, dwork, nwork, nt, smem, s);
    case 512: return launch_ypass_st_batch<T, 512, INV>(dargs, dwork, nwork, nt, smem, s);
    case 1024: return launch_ypass_st_batch<T, 1024, INV>(dargs, dwork, nwork, nt, smem, s);
    case 2048: return launch_ypass_st_batch<T, 2048, INV>(dargs, dwork, nwork, nt, smem, s);
    case 192: return launch_ypass_st_batch<T, 192, INV>(dargs, dwork, nwork, nt, smem, s);
    case 384: return launch_ypass_st_batch<T, 384, INV>(dargs, dwork, nwork, nt, smem, s);
    case 768: return launch_ypass_st_batch<T, 768, INV>(dargs, dwork, nwork, nt, smem, s);
    case 1536: return launch_ypass_st_batch<T, 1536, INV>(dargs, dwork, nwork, nt, smem, s);
    default: return 111;
    }
}

// ------------------------------------------------------------------------------ launchers
template <typename KF>
static int launch_common(KF kern, dim3 grid, int nt, size_t smem, cudaStream_t s)
{
    if (nt > 1024 || nt < 1) return 101;
    if (smem > 227 * 1024) return 102;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}

template <typename T, int L>
static int launch_ymid2d_reg(const YZArgs<T> &a, cudaStream_t s)
{
    constexpr int P = ysplit<L>::p, Q = ysplit<L>::q;
    int nt = (ymid2d_reg_threads(L, a.W) + 31) & ~31;
    if (nt > bm_lb<T>::v) return 112;
    size_t smem = ymid2d_smem<T>(L, a.W);
    if (smem > 200 * 1024) return 113;
    dim3 grid((a.LX + a.W - 1) / a.W);
    int rc = launch_common(k_ymid2d_reg<T, P, Q>, grid, nt, smem, s);
    if (rc) return rc;
    k_ymid2d_reg<T, P, Q><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

// the register 2D y pass for this tile width, or -1 when it does not apply
template <typename T>
static int launch_ymid2d_reg_dispatch(const YZArgs<T> &a, cudaStream_t s)
{
    if ((a.W & (a.W - 1)) != 0 || !ypass_has_reg(a.Ny)) return -1;
    if (((ymid2d_reg_threads(a.Ny, a.W) + 31) & ~31) > bm_lb<T>::v || ymid2d_smem<T>(a.Ny, a.W) > 200 * 1024) return -1;
    switch (a.Ny) {
    case 8: return launch_ymid2d_reg<T, 8>(a, s);
    case 16: return launch_ymid2d_reg<T, 16>(a, s);
    case 32: return launch_ymid2d_reg<T, 32>(a, s);
    case 64: return launch_ymid2d_reg<T, 64>(a, s);
    case 128: return launch_ymid2d_reg<T, 128>(a, s);
    case 256: return launch_ymid2d_reg<T, 256>(a, s);
    case 512: return launch_ymid2d_reg<T, 512>(a, s);
    case 1024: return launch_ymid2d_reg<T, 1024>(a, s);
    default: return -1;
    }
}

template <typename T> int launch_ymid2d(const YZArgs<T> &a, cudaStream_t s)
{
    {
        int rc = launch_ymid2d_reg_dispatch<T>(a, s);
        if (rc >= 0) return rc;
    }
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
    if (a.yv == 2) {
        int rc = launch_ypass_tma<T, false>(a, s);
        if (rc >= 0) return rc;
    }
    if (a.yv == 1) {
        int rc = launch_ypass_st_dispatch<T, false>(a, s);
        if (rc >= 0) return rc;
    }
    {
        int rc = launch_ypass_dispatch<T, false>(a, s);
        if (rc >= 0) return rc;
    }
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
    if (a.yv == 2) {
        int rc = launch_ypass_tma<T, true>(a, s);
        if (rc >= 0) return rc;
    }
    if (a.yv == 1) {
        int rc = launch_ypass_st_dispatch<T, true>(a, s);
        if (rc >= 0) return rc;
    }
    {
        int rc = launch_ypass_dispatch<T, true>(a, s);
        if (rc >= 0) return rc;
    }
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
    if (a.zv == 1 && zmid_has_par(a.Nz, a.W)) {
        switch (a.Nz) {
        case 12: return launch_zmid_par<T, 12>(a, s);
        case 16: return launch_zmid_par<T, 16>(a, s);
        case 24: return launch_zmid_par<T, 24>(a, s);
        case 32: return launch_zmid_par<T, 32>(a, s);
        case 48: return launch_zmid_par<T, 48>(a, s);
        case 64: return launch_zmid_par<T, 64>(a, s);
        default: break;
        }
    }
    if ((a.W & (a.W - 1)) == 0) {
        switch (a.Nz) {
        case 4: return launch_zmid_reg<T, 4>(a, s);
        case 6: return launch_zmid_reg<T, 6>(a, s);
        case 8: return launch_zmid_reg<T, 8>(a, s);
        case 12: return launch_zmid_reg<T, 12>(a, s);
        case 16: return launch_zmid_reg<T, 16>(a, s);
        case 24: return launch_zmid_reg<T, 24>(a, s);
        case 32: return launch_zmid_reg<T, 32>(a, s);
        case 48: return launch_zmid_reg<T, 48>(a, s);
        case 64: return launch_zmid_reg<T, 64>(a, s);
        default: break;
        }
    }
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

// ------------------------------------------------------------------------------ batched launchers
// One launch over a work list of (mesh, tile) items, one block per item; nt and smem are the
// maxima over the meshes. (A grid-stride loop over the items around the FFT bodies made the
// compiler fall back to 32 registers with kilobytes of per-thread stack, so each block takes one
// item and the hardware block scheduler balances the uneven items.)
template <typename KF>
static int launch_batch_common(KF kern, int nwork, int nt, size_t smem, int *grid)
{
    int rc = launch_common(kern, dim3(1), nt, smem, 0);
    if (rc) return rc;
    *grid = nwork;
    return 0;
}

template <typename T, int NZ>
static int launch_zmid_reg_batch(const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s)
{
    int grid = 1, rc = launch_batch_common(k_zmid_reg_batch<T, NZ>, nwork, nt, smem, &grid);
    if (rc) return rc;
    k_zmid_reg_batch<T, NZ><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
    return (int)cudaGetLastError();
}

template <typename T, int L>
static int launch_ymid2d_reg_batch(const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s)
{
    constexpr int P = ysplit<L>::p, Q = ysplit<L>::q;
    int grid = 1, rc = launch_batch_common(k_ymid2d_reg_batch<T, P, Q>, nwork, nt, smem, &grid);
    if (rc) return rc;
    k_ymid2d_reg_batch<T, P, Q><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
    return (int)cudaGetLastError();
}

template <typename T, int L, bool INV>
static int launch_ypass_reg_batch(const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s)
{
    constexpr int P = ysplit<L>::p, Q = ysplit<L>::q;
    int grid = 1, rc = launch_batch_common(k_ypass_reg_batch<T, P, Q, INV>, nwork, nt, smem, &grid);
    if (rc) return rc;
    k_ypass_reg_batch<T, P, Q, INV><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
    return (int)cudaGetLastError();
}

template <typename T, bool INV>
static int ypass_reg_batch_dispatch(int Ny, const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem,
                                    cudaStream_t s)
{
    switch (Ny) {
    case 8: return launch_ypass_reg_batch<T, 8, INV>(dargs, dwork, nwork, nt, smem, s);
    case 16: return launch_ypass_reg_batch<T, 16, INV>(dargs, dwork, nwork, nt, smem, s);
    case 32: return launch_ypass_reg_batch<T, 32, INV>(dargs, dwork, nwork, nt, smem, s);
    case 64: return launch_ypass_reg_batch<T, 64, INV>(dargs, dwork, nwork, nt, smem, s);
    case 128: return launch_ypass_reg_batch<T, 128, INV>(dargs, dwork, nwork, nt, smem, s);
    case 256: return launch_ypass_reg_batch<T, 256, INV>(dargs, dwork, nwork, nt, smem, s);
    case 512: return launch_ypass_reg_batch<T, 512, INV>(dargs, dwork, nwork, nt, smem, s);
    case 1024: return launch_ypass_reg_batch<T, 1024, INV>(dargs, dwork, nwork, nt, smem, s);
    default: return 111;
    }
}

template <typename T>
int launch_yz_batch(int kind, int key, const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem,
                    cudaStream_t s)
{
    if (nwork < 1) return 0;
    int grid = 1, rc = 0;
    switch (kind) {
    case BM_BATCH_YMID2D:
        if ((rc = launch_batch_common(k_ymid2d_batch<T>, nwork, nt, smem, &grid))) return rc;
        k_ymid2d_batch<T><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
        break;
    case BM_BATCH_YFWD:
        if ((rc = launch_batch_common(k_ypass3d_batch<T, false>, nwork, nt, smem, &grid))) return rc;
        k_ypass3d_batch<T, false><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
        break;
    case BM_BATCH_YINV:
        if ((rc = launch_batch_common(k_ypass3d_batch<T, true>, nwork, nt, smem, &grid))) return rc;
        k_ypass3d_batch<T, true><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
        break;
    case BM_BATCH_ZMID:
        if ((rc = launch_batch_common(k_zmid_batch<T>, nwork, nt, smem, &grid))) return rc;
        k_zmid_batch<T><<<grid, nt, smem, s>>>(dargs, dwork, nwork);
        break;
    case BM_BATCH_ZMID_REG:
        switch (key) {
        case 4: return launch_zmid_reg_batch<T, 4>(dargs, dwork, nwork, nt, smem, s);
        case 6: return launch_zmid_reg_batch<T, 6>(dargs, dwork, nwork, nt, smem, s);
        case 8: return launch_zmid_reg_batch<T, 8>(dargs, dwork, nwork, nt, smem, s);
        case 12: return launch_zmid_reg_batch<T, 12>(dargs, dwork, nwork, nt, smem, s);
        case 16: return launch_zmid_reg_batch<T, 16>(dargs, dwork, nwork, nt, smem, s);
        case 24: return launch_zmid_reg_batch<T, 24>(dargs, dwork, nwork, nt, smem, s);
        case 32: return launch_zmid_reg_batch<T, 32>(dargs, dwork, nwork, nt, smem, s);
        case 48: return launch_zmid_reg_batch<T, 48>(dargs, dwork, nwork, nt, smem, s);
        case 64: return launch_zmid_reg_batch<T, 64>(dargs, dwork, nwork, nt, smem, s);
        default: return 111;
        }
    case BM_BATCH_YMID2D_REG:
        switch (key) {
        case 8: return launch_ymid2d_reg_batch<T, 8>(dargs, dwork, nwork, nt, smem, s);
        case 16: return launch_ymid2d_reg_batch<T, 16>(dargs, dwork, nwork, nt, smem, s);
        case 32: return launch_ymid2d_reg_batch<T, 32>(dargs, dwork, nwork, nt, smem, s);
        case 64: return launch_ymid2d_reg_batch<T, 64>(dargs, dwork, nwork, nt, smem, s);
        case 128: return launch_ymid2d_reg_batch<T, 128>(dargs, dwork, nwork, nt, smem, s);
        case 256: return launch_ymid2d_reg_batch<T, 256>(dargs, dwork, nwork, nt, smem, s);
        case 512: return launch_ymid2d_reg_batch<T, 512>(dargs, dwork, nwork, nt, smem, s);
        case 1024: return launch_ymid2d_reg_batch<T, 1024>(dargs, dwork, nwork, nt, smem, s);
        default: return 111;
        }
    case BM_BATCH_YFWD_ST: return ypass_st_batch_dispatch<T, false>(key, dargs, dwork, nwork, nt, smem, s);
    case BM_BATCH_YINV_ST: return ypass_st_batch_dispatch<T, true>(key, dargs, dwork, nwork, nt, smem, s);
    case BM_BATCH_YFWD_REG: return ypass_reg_batch_dispatch<T, false>(key, dargs, dwork, nwork, nt, smem, s);
    case BM_BATCH_YINV_REG: return ypass_reg_batch_dispatch<T, true>(key, dargs, dwork, nwork, nt, smem, s);
    default: return 110;
    }
    return (int)cudaGetLastError();
}

template int launch_yz_batch<float>(int, int, const YZArgs<float> *, const int2 *, int, int, size_t, cudaStream_t);
template int launch_yz_batch<double>(int, int, const YZArgs<double> *, const int2 *, int, int, size_t, cudaStream_t);
