// Discrete adjoint of the RK4 step (reverse mode through the stages, the renormalisation to Ms and
// the field terms), the device kernels. The forward step is the one of Boris/DiffEqFM_Evals_RK4.cpp
// with the LLG of Boris/DiffEqFM_Equations.cpp:12 and the fields of Boris/Zeeman.cpp:164,
// Boris/Demag.cpp:170, Boris/Exchange.cpp:108 (Neumann Laplacian) and Boris/Anisotropy.cpp:82
// (K2 = 0); the reference itself has no adjoint.
//
// For f = a (X x H) + a (alpha / Ms) X x (X x H), a = -gamma grel / (1 + alpha^2), and a cotangent mu:
//   dX: a (H x mu) + a (alpha/Ms) [(X.H) mu + (mu.X) H - 2 (mu.H) X]
//   dH: a (mu x X) + a (alpha/Ms) [(mu.X) X - |X|^2 mu]
//   dMs: -a alpha / Ms^2 mu . (X (X.H) - H |X|^2)
// and dH is carried back through H = Ha + D X + c L X + kappa (X.e) e, c = 2A/(mu0 Ms^2),
// kappa = 2 K1/(mu0 Ms^2): D and the Neumann Laplacian L are symmetric. Gradients accumulate in FP64.
#include "kernels.h"

template <typename T> __device__ __forceinline__ T adj_ms(const AdjArgs<T> &a, long long i) { return a.Ms_map ? a.Ms_map[i] : a.Ms; }
template <typename T> __device__ __forceinline__ T adj_k1(const AdjArgs<T> &a, long long i) { return a.K1_map ? a.K1_map[i] : a.K1; }

static int adj_grid(long long n)
{
    long long b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return (int)(b < 1 ? 1 : b);
}

// per-block sum of a double into *out (atomic)
__device__ __forceinline__ void block_sum_add(double v, double *out)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) t += red[w];
        atomicAdd(out, t);
    }
    __syncthreads();
}

// Neumann Laplacian of one component at cell (x, y, z): only existing neighbours; along a periodic
// axis the far-side cell, times the axis' sign, stands in for the missing one (the operator stays
// symmetric for either sign)
template <typename T>
__device__ __forceinline__ T adj_lap(const T *V, int x, int y, int z, long long cell, const AdjArgs<T> &a)
{
    const T v = V[cell];
    T s = 0;
    const long long nxy = (long long)a.nx * a.ny;
    const long long wx = a.nx - 1, wy = (long long)(a.ny - 1) * a.nx, wz = (long long)(a.nz - 1) * nxy;
    const bool px = a.pbc[0] && a.nx > 1, py = a.pbc[1] && a.ny > 1, pz = a.pbc[2] && a.nz > 1;
    if (x > 0) s += (V[cell - 1] - v) / (a.hx * a.hx);
    else if (px) s += ((T)a.pbc[0] * V[cell + wx] - v) / (a.hx * a.hx);
    if (x + 1 < a.nx) s += (V[cell + 1] - v) / (a.hx * a.hx);
    else if (px) s += ((T)a.pbc[0] * V[cell - wx] - v) / (a.hx * a.hx);
    if (y > 0) s += (V[cell - a.nx] - v) / (a.hy * a.hy);
    else if (py) s += ((T)a.pbc[1] * V[cell + wy] - v) / (a.hy * a.hy);
    if (y + 1 < a.ny) s += (V[cell + a.nx] - v) / (a.hy * a.hy);
    else if (py) s += ((T)a.pbc[1] * V[cell - wy] - v) / (a.hy * a.hy);
    if (z > 0) s += (V[cell - nxy] - v) / (a.hz * a.hz);
    else if (pz) s += ((T)a.pbc[2] * V[cell + wz] - v) / (a.hz * a.hz);
    if (z + 1 < a.nz) s += (V[cell + nxy] - v) / (a.hz * a.hz);
    else if (pz) s += ((T)a.pbc[2] * V[cell - wz] - v) / (a.hz * a.hz);
    return s;
}

// loss (1/n) sum |M/Ms - t|^2, its gradient in M (lam) and the direct part in Ms
template <typename T>
__global__ void k_adj_loss(AdjArgs<T> a, const T *__restrict__ M, const double *__restrict__ target, T *__restrict__ lam,
                           double *__restrict__ gMs, double *__restrict__ loss)
{
    const long long n = a.n;
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double Ms = (double)adj_ms(a, i);
        double g = 0.0;
        for (int c = 0; c < 3; c++) {
            const double m = (double)M[c * n + i] / Ms, r = m - target[3 * i + c];
            acc += r * r;
            lam[c * n + i] = (T)(2.0 / (double)n * r / Ms);
            g += 2.0 / (double)n * r * (-m / Ms);
        }
        gMs[i] += g;
    }
    block_sum_add(acc / (double)n, loss);
}

// M = Ms Y / |Y|: lamY = Ms/|Y| (lam - (y.lam) y), lam <- lamY, mu = dt/6 lamY, gMs += y.lam
template <typename T>
__global__ void k_adj_renorm(AdjArgs<T> a, T *__restrict__ lam, const T *__restrict__ Y, T *__restrict__ lamY, T *__restrict__ mu,
                             double dt, double *__restrict__ gMs)
{
    const long long n = a.n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const T Ms = adj_ms(a, i);
        T y[3] = {Y[i], Y[n + i], Y[2 * n + i]}, l[3] = {lam[i], lam[n + i], lam[2 * n + i]};
        const T nr = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
        const T yl = (y[0] * l[0] + y[1] * l[1] + y[2] * l[2]) / nr;
        gMs[i] += (double)yl;
        for (int c = 0; c < 3; c++) {
            const T v = Ms / nr * (l[c] - yl * y[c] / nr);
            lamY[c * n + i] = v;
            lam[c * n + i] = v;
            mu[c * n + i] = (T)(dt / 6.0) * v;
        }
    }
}

// LLG and local field terms: gH, the direct part of gX (LLG + anisotropy), w = c gH (exchange),
// and the Ms, K1 and Zeeman gradients of this stage
template <typename T>
__global__ void k_adj_vjp_a(AdjArgs<T> a, const T *__restrict__ X, const T *__restrict__ H, const T *__restrict__ mu,
                            T *__restrict__ gHo, T *__restrict__ gXd, T *__restrict__ w, double *__restrict__ gMs,
                            double *__restrict__ gK1, double *__restrict__ gHa3)
{
    const long long n = a.n;
    const T pre = -(T)BM_GAMMA * a.grel / (1 + a.alpha * a.alpha);
    double zs[3] = {0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const T Ms = adj_ms(a, i), b = pre * a.alpha / Ms;
        T x[3], h[3], m[3];
        for (int c = 0; c < 3; c++) { x[c] = X[c * n + i]; h[c] = H[c * n + i]; m[c] = mu[c * n + i]; }
        const T xh = x[0] * h[0] + x[1] * h[1] + x[2] * h[2];
        const T mx = m[0] * x[0] + m[1] * x[1] + m[2] * x[2];
        const T mh = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
        const T xx = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        const T hxm[3] = {h[1] * m[2] - h[2] * m[1], h[2] * m[0] - h[0] * m[2], h[0] * m[1] - h[1] * m[0]};
        const T mxx[3] = {m[1] * x[2] - m[2] * x[1], m[2] * x[0] - m[0] * x[2], m[0] * x[1] - m[1] * x[0]};
        T gx[3], gh[3];
        for (int c = 0; c < 3; c++) {
            gx[c] = pre * hxm[c] + b * (xh * m[c] + mx * h[c] - 2 * mh * x[c]);
            gh[c] = pre * mxx[c] + b * (mx * x[c] - xx * m[c]);
        }
        double gms = -(double)pre * (double)a.alpha / ((double)Ms * Ms) * ((double)mx * xh - (double)mh * xx);
        if (a.modules & BM_MOD_EXCH) {
            const T cst = 2 * a.A / ((T)BM_MU0 * Ms * Ms);
            const int xi = (int)(i % a.nx), yi = (int)((i / a.nx) % a.ny), zi = (int)(i / ((long long)a.nx * a.ny));
            double dot = 0.0;
            for (int c = 0; c < 3; c++) {
                dot += (double)gh[c] * (double)adj_lap(X + c * n, xi, yi, zi, i, a);
                w[c * n + i] = cst * gh[c];
            }
            gms += dot * (-2.0 * (double)cst / (double)Ms);
        }
        if (a.modules & BM_MOD_ANIUNI) {
            const T kap = 2 * adj_k1(a, i) / ((T)BM_MU0 * Ms * Ms);
            const T xe = x[0] * a.ea[0] + x[1] * a.ea[1] + x[2] * a.ea[2];
            const T ge = gh[0] * a.ea[0] + gh[1] * a.ea[1] + gh[2] * a.ea[2];
            for (int c = 0; c < 3; c++) gx[c] += kap * ge * a.ea[c];
            gK1[i] += (double)xe * ge * 2.0 / (BM_MU0 * (double)Ms * Ms);
            gms += (double)xe * ge * (-2.0 * (double)kap / (double)Ms);
        }
        gMs[i] += gms;
        for (int c = 0; c < 3; c++) {
            gHo[c * n + i] = gh[c];
            gXd[c * n + i] = gx[c];
            zs[c] += (double)gh[c];
        }
    }
    if (a.modules & BM_MOD_ZEEMAN) {
        block_sum_add(zs[0], gHa3 + 0);
        block_sum_add(zs[1], gHa3 + 1);
        block_sum_add(zs[2], gHa3 + 2);
    }
}

// gX = gXd + L(w) + gD; lam += gX; mu = cY lamY + cX gX (for the next earlier stage)
template <typename T>
__global__ void k_adj_vjp_c(AdjArgs<T> a, const T *__restrict__ gXd, const T *__restrict__ w, const T *__restrict__ gD,
                            const T *__restrict__ lamY, T *__restrict__ lam, T *__restrict__ mu, T cY, T cX, int write_mu)
{
    const long long n = a.n;
    const bool exch = (a.modules & BM_MOD_EXCH) != 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int xi = (int)(i % a.nx), yi = (int)((i / a.nx) % a.ny), zi = (int)(i / ((long long)a.nx * a.ny));
        for (int c = 0; c < 3; c++) {
            T g = gXd[c * n + i];
            if (exch) g += adj_lap(w + c * n, xi, yi, zi, i, a);
            if (gD) g += gD[c * n + i];
            lam[c * n + i] += g;
            if (write_mu) mu[c * n + i] = cY * lamY[c * n + i] + cX * g;
        }
    }
}

// initial state M0 = Ms m0: gMs += m0 . lam
template <typename T>
__global__ void k_adj_m0(AdjArgs<T> a, const T *__restrict__ M0, const T *__restrict__ lam, double *__restrict__ gMs)
{
    const long long n = a.n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double Ms = (double)adj_ms(a, i);
        double g = 0.0;
        for (int c = 0; c < 3; c++) g += (double)M0[c * n + i] / Ms * (double)lam[c * n + i];
        gMs[i] += g;
    }
}

template <typename T>
int launch_adj_loss(const AdjArgs<T> &a, const T *M, const double *target, T *lam, double *gMs, double *loss, cudaStream_t s)
{
    k_adj_loss<T><<<adj_grid(a.n), 256, 0, s>>>(a, M, target, lam, gMs, loss);
    return (int)cudaGetLastError();
}
template <typename T>
int launch_adj_renorm(const AdjArgs<T> &a, T *lam, const T *Y, T *lamY, T *mu, double dt, double *gMs, cudaStream_t s)
{
    k_adj_renorm<T><<<adj_grid(a.n), 256, 0, s>>>(a, lam, Y, lamY, mu, dt, gMs);
    return (int)cudaGetLastError();
}
template <typename T>
int launch_adj_vjp_a(const AdjArgs<T> &a, const T *X, const T *H, const T *mu, T *gH, T *gXd, T *w, double *gMs, double *gK1,
                     double *gHa3, cudaStream_t s)
{
    k_adj_vjp_a<T><<<adj_grid(a.n), 256, 0, s>>>(a, X, H, mu, gH, gXd, w, gMs, gK1, gHa3);
    return (int)cudaGetLastError();
}
template <typename T>
int launch_adj_vjp_c(const AdjArgs<T> &a, const T *gXd, const T *w, const T *gD, const T *lamY, T *lam, T *mu, double cY,
                     double cX, int write_mu, cudaStream_t s)
{
    k_adj_vjp_c<T><<<adj_grid(a.n), 256, 0, s>>>(a, gXd, w, gD, lamY, lam, mu, (T)cY, (T)cX, write_mu);
    return (int)cudaGetLastError();
}
template <typename T>
int launch_adj_m0(const AdjArgs<T> &a, const T *M0, const T *lam, double *gMs, cudaStream_t s)
{
    k_adj_m0<T><<<adj_grid(a.n), 256, 0, s>>>(a, M0, lam, gMs);
    return (int)cudaGetLastError();
}

#define BM_ADJ_INST(T)                                                                                                  \
    template int launch_adj_loss<T>(const AdjArgs<T> &, const T *, const double *, T *, double *, double *, cudaStream_t); \
    template int launch_adj_renorm<T>(const AdjArgs<T> &, T *, const T *, T *, T *, double, double *, cudaStream_t);    \
    template int launch_adj_vjp_a<T>(const AdjArgs<T> &, const T *, const T *, const T *, T *, T *, T *, double *,      \
                                     double *, double *, cudaStream_t);                                                 \
    template int launch_adj_vjp_c<T>(const AdjArgs<T> &, const T *, const T *, const T *, const T *, T *, T *, double,  \
                                     double, int, cudaStream_t);                                                        \
    template int launch_adj_m0<T>(const AdjArgs<T> &, const T *, const T *, double *, cudaStream_t);
BM_ADJ_INST(float)
BM_ADJ_INST(double)
