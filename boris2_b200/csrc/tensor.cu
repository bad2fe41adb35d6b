// FP64 demagnetising-tensor build and its transform into the real kernel spectra.
//
// Follows the reference's kernel construction:
//   Newell f, g               Boris/DemagTFunc_fg.cpp:10,45 (written here with asinh/atan directly)
//   27-point differences      Boris/DemagTFunc_L.cpp:8,59
//   octant fill + parity      Boris/DemagTFunc.cpp:21,95,172,237 (D = -N, "minus" = true)
//   switch to far field       ASYMPTOTIC_DISTANCE = 40 cells (Boris/DemagTFunc_Defs.h:9)
//   spectra                   Boris/DemagKernel.cpp:171,317: real parts of the DFT over the
//                             (Nx/2+1)(Ny/2+1)(Nz/2+1) octant, h normalised by max(h)
// The far field is this project's own expansion: the double cell average of
// (V / 4pi) d_i d_j (1/R), expanded with prod_k (1 + h_k^2 d_k^2/12 + h_k^4 d_k^4/360 + h_k^6 d_k^6/20160)
// to total derivative order 8; the polynomial coefficients are built on the host
// (tensor_host.cpp) and evaluated here in FP64.
#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"
#include "ml.h"
#include "boris_b200.h"

#include <string>
int bm_set_error(int code, const std::string &msg);

#define BM_ASYMPT_DIST 40

__host__ __device__ __forceinline__ double csum_d(const double *v, int n)
{
    double s = 0.0, c = 0.0;
    for (int i = 0; i < n; i++) {
        double t = s + v[i];
        if (fabs(s) >= fabs(v[i])) c += (s - t) + v[i];
        else c += (v[i] - t) + s;
        s = t;
    }
    return s + c;
}

__host__ __device__ double nf(double x, double y, double z)
{
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R = sqrt(x2 + y2 + z2);
    double t[4] = {0, 0, 0, 0};
    t[0] = (2.0 * x2 - y2 - z2) * R / 6.0;
    double rxz = sqrt(x2 + z2), rxy = sqrt(x2 + y2);
    if (rxz > 0.0) t[1] = 0.5 * y * (z2 - x2) * asinh(y / rxz);
    if (rxy > 0.0) t[2] = 0.5 * z * (y2 - x2) * asinh(z / rxy);
    if (x != 0.0 && R > 0.0) t[3] = -x * y * z * atan(y * z / (x * R));
    return csum_d(t, 4);
}

__host__ __device__ double ng(double x, double y, double z)
{
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R = sqrt(x2 + y2 + z2);
    double t[7] = {0, 0, 0, 0, 0, 0, 0};
    t[0] = -x * y * R / 3.0;
    double rxy = sqrt(x2 + y2), ryz = sqrt(y2 + z2), rxz = sqrt(x2 + z2);
    if (rxy > 0.0) t[1] = x * y * z * asinh(z / rxy);
    if (ryz > 0.0) t[2] = y * (3.0 * z2 - y2) * asinh(x / ryz) / 6.0;
    if (rxz > 0.0) t[3] = x * (3.0 * z2 - x2) * asinh(y / rxz) / 6.0;
    if (z != 0.0 && R > 0.0) t[4] = -z2 * z * atan(x * y / (z * R)) / 6.0;
    if (y != 0.0 && R > 0.0) t[5] = -y2 * z * atan(x * z / (y * R)) / 2.0;
    if (x != 0.0 && R > 0.0) t[6] = -x2 * z * atan(y * z / (x * R)) / 2.0;
    return csum_d(t, 7);
}

template <bool G>
__host__ __device__ double newellL(double x, double y, double z, double hx, double hy, double hz)
{
    double v[27];
    int m = 0;
    const double cw[3] = {-1.0, 2.0, -1.0};
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++) {
                double w = cw[a + 1] * cw[b + 1] * cw[c + 1];
                v[m++] = w * (G ? ng(x + a * hx, y + b * hy, z + c * hz) : nf(x + a * hx, y + b * hy, z + c * hz));
            }
    return csum_d(v, 27) / (4.0 * M_PI * hx * hy * hz);
}

// Self-demagnetising coefficients -N (the tensor's diagonal at the origin, DemagTFunc::SelfDemag,
// Boris/DemagTFunc_Self.cpp:6 with "minus"), on the host, cellsizes normalised by the largest.
void self_demag_host(double hx, double hy, double hz, double out3[3])
{
    double hm = fmax(hx, fmax(hy, hz));
    hx /= hm; hy /= hm; hz /= hm;
    out3[0] = -newellL<false>(0.0, 0.0, 0.0, hx, hy, hz);
    out3[1] = -newellL<false>(0.0, 0.0, 0.0, hy, hx, hz);
    out3[2] = -newellL<false>(0.0, 0.0, 0.0, hz, hy, hx);
}

// The self coefficients as the reference's evaluation speedup gets them: DemagTFunc::SelfDemag on the
// cellsize in metres (Boris/DemagCUDA.cpp:39, Boris/DemagTFunc_Self.cpp:6), whose Newell f
// (Boris/DemagTFunc_fg.cpp:10) leaves out a log or atan term when its squared length or coordinate is
// not above the library's zero threshold (BorisLib/Funcs_Aux_base.h:9,35: 1e-12 as a float). For
// nanometre cells those squared lengths (~1e-17 m^2) fall under it, so the coefficients differ from the
// tensor's own self term; this reproduces that.
namespace {
const double kRefZero = (double)1e-12f;
bool ref_nz(double v) { return v > kRefZero || v < -kRefZero; }

double f_thresholded(double x, double y, double z)
{
    const double xsq = x * x, ysq = y * y, zsq = z * z;
    const double Rxy = xsq + ysq, Rxz = xsq + zsq;
    const double R = sqrt(xsq + ysq + zsq);
    double t[4] = {(2.0 * xsq - ysq - zsq) * R / 6.0, 0.0, 0.0, 0.0};
    if (ref_nz(Rxz)) {
        const double arg = 2.0 * y * (y + R) / Rxz;
        if (arg > -1.0) t[1] = y * (zsq - xsq) * log1p(arg) / 4.0;
    }
    if (ref_nz(Rxy)) {
        const double arg = 2.0 * z * (z + R) / Rxy;
        if (arg > -1.0) t[2] = z * (ysq - xsq) * log1p(arg) / 4.0;
    }
    if (ref_nz(x)) t[3] = -x * y * z * atan(y * z / (x * R));
    return csum_d(t, 4);
}

// -N_xx of the cell (a, b, c): the second difference of f over the cell's 27 corner offsets
double self_thresholded(double a, double b, double c)
{
    double v[27];
    int m = 0;
    const double cw[3] = {-1.0, 2.0, -1.0};
    for (int i = -1; i <= 1; i++)
        for (int j = -1; j <= 1; j++)
            for (int k = -1; k <= 1; k++) v[m++] = cw[i + 1] * cw[j + 1] * cw[k + 1] * f_thresholded(i * a, j * b, k * c);
    return -csum_d(v, 27) / (4.0 * M_PI * a * b * c);
}
}  // namespace

void self_demag_metres_host(double hx, double hy, double hz, double out3[3])
{
    out3[0] = self_thresholded(hx, hy, hz);
    out3[1] = self_thresholded(hy, hx, hz);
    out3[2] = self_thresholded(hz, hy, hx);
}

extern "C" int bm_self_demag_metres(double hx, double hy, double hz, double *out3)
{
    if (!out3 || !(hx > 0) || !(hy > 0) || !(hz > 0)) return bm_set_error(BM_EINVAL, "bm_self_demag_metres: cellsizes must be > 0");
    self_demag_metres_host(hx, hy, hz, out3);
    return 0;
}

extern "C" int bm_self_demag(double hx, double hy, double hz, double *out3)
{
    if (!out3 || !(hx > 0) || !(hy > 0) || !(hz > 0)) return bm_set_error(BM_EINVAL, "bm_self_demag: cellsizes must be > 0");
    self_demag_host(hx, hy, hz, out3);
    return 0;
}

// far field: D_c = V/(4 pi) sum_n Q_{c,n}(u,v,w) / R^(n+1), coefficient layout per comp c:
// for n in {2,4,6,8}: monomials (i,j,k), i+j+k = n, ordered i descending then j descending
__host__ __device__ double far_eval(const double *__restrict__ q, double u, double v, double w, double R)
{
    double pu[9], pv[9], pw[9];
    pu[0] = pv[0] = pw[0] = 1.0;
    for (int i = 1; i < 9; i++) { pu[i] = pu[i - 1] * u; pv[i] = pv[i - 1] * v; pw[i] = pw[i - 1] * w; }
    double tot[4];
    int off = 0;
    for (int o = 0; o < 4; o++) {
        int n = 2 + 2 * o;
        double acc[45];
        int m = 0;
        for (int i = n; i >= 0; i--)
            for (int j = n - i; j >= 0; j--) {
                int k = n - i - j;
                acc[m++] = q[off++] * pu[i] * pv[j] * pw[k];
            }
        tot[o] = csum_d(acc, m) / pow(R, n + 1);
    }
    return csum_d(tot, 4);
}

// D = -N of one cell pair at the non-negative offset (i, j, k) cells (normalised cellsize): the
// exact Newell differences within 40 cells, the far-field expansion beyond, the reference's rule
// (Boris/DemagTFunc.cpp:40-58). v = xx, yy, zz, xy, xz, yz; a one-cell-thick mesh has no xz, yz.
__device__ __forceinline__ void tensor_point(int i, int j, int k, double hx, double hy, double hz,
                                             const double *__restrict__ farq, int two_d, double v[6])
{
    double x = i * hx, y = j * hy, z = k * hz;
    bool far = (i >= BM_ASYMPT_DIST || j >= BM_ASYMPT_DIST || k >= BM_ASYMPT_DIST ||
                (long long)i * i + (long long)j * j + (long long)k * k >= (long long)BM_ASYMPT_DIST * BM_ASYMPT_DIST);
    if (far) {
        double R = sqrt(x * x + y * y + z * z);
        double u = x / R, vv = y / R, w = z / R;
        double V = hx * hy * hz / (4.0 * M_PI);
        for (int c = 0; c < 6; c++) v[c] = (two_d && c >= 4) ? 0.0 : V * far_eval(farq + c * BM_FARQ_PER_COMP, u, vv, w, R);
    } else {
        v[0] = -newellL<false>(x, y, z, hx, hy, hz);
        v[1] = -newellL<false>(y, x, z, hy, hx, hz);
        v[2] = -newellL<false>(z, y, x, hz, hy, hx);
        v[3] = -newellL<true>(x, y, z, hx, hy, hz);
        v[4] = two_d ? 0.0 : -newellL<true>(x, z, y, hx, hz, hy);
        v[5] = two_d ? 0.0 : -newellL<true>(y, z, x, hy, hz, hx);
    }
}

// octant values D(i,j,k), i<nx, j<ny, k<nz -> oct[((k*ny + j)*nx + i)*6 + c], c = xx,yy,zz,xy,xz,yz
__global__ void k_tensor_octant(double *oct, int nx, int ny, int nz, double hx, double hy, double hz,
                                const double *__restrict__ farq, int two_d)
{
    long long N = (long long)nx * ny * nz;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % nx);
        int j = (int)((p / nx) % ny);
        int k = (int)(p / ((long long)nx * ny));
        double v[6];
        tensor_point(i, j, k, hx, hy, hz, farq, two_d, v);
        for (int c = 0; c < 6; c++) oct[p * 6 + c] = v[c];
    }
}

// ---------------------------------------------------------------- periodic boundary conditions
// The reference convolves a PBC axis cyclically over its n cells (FFT length n,
// Boris/ConvolutionData.cpp:115-145) with the tensor summed over +-images periods
// (Boris/DemagTFunc_PBC.cpp:5,97,185,300): D(i0) = sum_{m=-X..X} T(m n + i0) for i0 in [0, n), and it
// keeps only the real (even components) or imaginary (odd components) part of each axis' DFT
// (Boris/DemagKernel.cpp:250-300,365-460). Those parts are the DFT of the tensor made even or odd
// about i0 = 0 along the axis: Ds(i0) = (D(i0) +- D((n - i0) mod n)) / 2. A cyclic convolution of
// period n over n cells only uses offsets d in (-n, n), so it is the linear convolution with the
// kernel Ds(d mod n) there; this path therefore keeps its zero-padded transforms and fills the
// octant [0, n) of each PBC axis with Ds. Written out, with T(-x) = +-T(x):
//   i0 = 0:  Ds = sum_{m=-X..X} T(m n)                              (odd components: 0)
//   i0 > 0:  Ds = sum_{m=-X-1..X} w_m T(m n + i0), w = 1/2 at m = -X-1 and m = X, 1 otherwise,
// and Ds(n - i0) = +-Ds(i0), so a thread evaluates i0 <= n / 2 and writes both. Odd components take
// the sign of each offset with sign(0) = 0 (BorisLib/Funcs_Math.h:103, get_sign), as the reference.
struct PbcSpec {
    int n[3];     // cells per axis
    int img[3];   // images per axis (0: no PBC along it)
};

__device__ __forceinline__ int isgn(int v) { return (v > 0) - (v < 0); }

__global__ void k_tensor_octant_pbc(double *oct, PbcSpec P, double hx, double hy, double hz,
                                    const double *__restrict__ farq, int two_d)
{
    int ce[3];   // canonical extent per axis
    for (int a = 0; a < 3; a++) ce[a] = P.img[a] ? P.n[a] / 2 + 1 : P.n[a];
    const long long Nc = (long long)ce[0] * ce[1] * ce[2];
    const int nx = P.n[0], ny = P.n[1];
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < Nc; p += (long long)gridDim.x * blockDim.x) {
        int q[3];
        q[0] = (int)(p % ce[0]);
        q[1] = (int)((p / ce[0]) % ce[1]);
        q[2] = (int)(p / ((long long)ce[0] * ce[1]));
        // image range per axis: [lo, hi] with half weights at the ends when `half`
        int lo[3], hi[3], half[3];
        for (int a = 0; a < 3; a++) {
            const int X = P.img[a];
            if (!X) { lo[a] = hi[a] = 0; half[a] = 0; }
            else if (q[a] == 0) { lo[a] = -X; hi[a] = X; half[a] = 0; }
            else { lo[a] = -X - 1; hi[a] = X; half[a] = 1; }
        }
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int mx = lo[0]; mx <= hi[0]; mx++) {
            const double wx = (half[0] && (mx == lo[0] || mx == hi[0])) ? 0.5 : 1.0;
            const int i = mx * P.n[0] + q[0];
            for (int my = lo[1]; my <= hi[1]; my++) {
                const double wy = (half[1] && (my == lo[1] || my == hi[1])) ? 0.5 : 1.0;
                const int j = my * P.n[1] + q[1];
                for (int mz = lo[2]; mz <= hi[2]; mz++) {
                    const double w = wx * wy * ((half[2] && (mz == lo[2] || mz == hi[2])) ? 0.5 : 1.0);
                    const int k = mz * P.n[2] + q[2];
                    const int si = isgn(i), sj = isgn(j), sk = isgn(k);
                    double v[6];
                    tensor_point(abs(i), abs(j), abs(k), hx, hy, hz, farq, two_d, v);
                    acc[0] += w * v[0];
                    acc[1] += w * v[1];
                    acc[2] += w * v[2];
                    acc[3] += w * v[3] * (si * sj);
                    acc[4] += w * v[4] * (si * sk);
                    acc[5] += w * v[5] * (sj * sk);
                }
            }
        }
        if (q[0] == 0 && P.img[0]) { acc[3] = 0.0; acc[4] = 0.0; }
        if (q[1] == 0 && P.img[1]) { acc[3] = 0.0; acc[5] = 0.0; }
        if (q[2] == 0 && P.img[2]) { acc[4] = 0.0; acc[5] = 0.0; }
        // write the point and its mirrors n - i0 on the PBC axes (odd components change sign)
        for (int f = 0; f < 8; f++) {
            int r[3];
            int par[3] = {1, 1, 1};   // -1 on a mirrored axis
            bool ok = true;
            for (int a = 0; a < 3 && ok; a++) {
                if (f & (1 << a)) {
                    if (!P.img[a] || q[a] == 0 || 2 * q[a] == P.n[a]) { ok = false; break; }
                    r[a] = P.n[a] - q[a];
                    par[a] = -1;
                } else r[a] = q[a];
            }
            if (!ok) continue;
            const long long o = (((long long)r[2] * ny + r[1]) * nx + r[0]) * 6;
            oct[o + 0] = acc[0];
            oct[o + 1] = acc[1];
            oct[o + 2] = acc[2];
            oct[o + 3] = acc[3] * (par[0] * par[1]);
            oct[o + 4] = acc[4] * (par[0] * par[2]);
            oct[o + 5] = acc[5] * (par[1] * par[2]);
        }
    }
}

// Self coefficients of the evaluation speedup under PBC, DemagTFunc::SelfDemag_PBC
// (Boris/DemagTFunc_Self.cpp:57): the cell's own -N plus, for every image period other than the
// cell itself, the far-field D at the image's offset (images at multiples of the mesh length). As
// there, all three diagonal terms use the expansion of the (hx, hy, hz) cell with the xx form, the
// yy and zz terms at the offsets permuted (y, x, z) and (z, y, x). Cellsizes are normalised by the
// largest, as for the tensor.
void self_demag_pbc_host(double hx, double hy, double hz, const int n[3], const int img[3], double out3[3], int metres)
{
    // the reference's image loops run from -images to images: a negative count on any axis (a
    // stencil sign of -1) leaves them empty and the coefficient zero, self term included
    if (img[0] < 0 || img[1] < 0 || img[2] < 0) { out3[0] = out3[1] = out3[2] = 0.0; return; }
    if (metres) self_demag_metres_host(hx, hy, hz, out3);
    else self_demag_host(hx, hy, hz, out3);
    double hm = fmax(hx, fmax(hy, hz));
    hx /= hm; hy /= hm; hz /= hm;
    int X = img[0], Y = img[1], Z = img[2];
    if (!X && !Y && !Z) return;
    double q[6 * BM_FARQ_PER_COMP];
    bm_far_coeffs(hx, hy, hz, q);
    const double V = hx * hy * hz / (4.0 * M_PI);
    for (int a = -X; a <= X; a++)
        for (int b = -Y; b <= Y; b++)
            for (int c = -Z; c <= Z; c++) {
                if (!a && !b && !c) continue;
                double x = fabs((double)a * n[0]) * hx, y = fabs((double)b * n[1]) * hy, z = fabs((double)c * n[2]) * hz;
                double R = sqrt(x * x + y * y + z * z);
                out3[0] += V * far_eval(q, x / R, y / R, z / R, R);
                out3[1] += V * far_eval(q, y / R, x / R, z / R, R);
                out3[2] += V * far_eval(q, z / R, y / R, x / R, R);
            }
}

// fill one component on the full N grid (complex, imaginary zero) from the octant with parity
__global__ void k_tensor_fill(cpx<double> *F, const double *__restrict__ oct, int comp, int nx, int ny, int nz,
                              int Nx, int Ny, int Nz)
{
    long long Ntot = (long long)Nx * Ny * Nz;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < Ntot; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % Nx);
        int j = (int)((p / Nx) % Ny);
        int k = (int)(p / ((long long)Nx * Ny));
        int ai = i <= Nx / 2 ? i : Nx - i, sx = i <= Nx / 2 ? 1 : -1;
        int aj = j <= Ny / 2 ? j : Ny - j, sy = j <= Ny / 2 ? 1 : -1;
        int ak = k <= Nz / 2 ? k : Nz - k, sz = k <= Nz / 2 ? 1 : -1;
        double val = 0.0;
        if (ai < nx && aj < ny && ak < nz) {
            val = oct[(((long long)ak * ny + aj) * nx + ai) * 6 + comp];
            if (comp == 3) val *= sx * sy;
            else if (comp == 4) val *= sx * sz;
            else if (comp == 5) val *= sy * sz;
        }
        F[p] = mk<double>(val, 0.0);
    }
}

// extract Re on the octant into the kernel planes K[comp][(kz*Ky1 + ky)*Kx1 + kx] (type T)
template <typename T>
__global__ void k_tensor_extract(T *K, const cpx<double> *__restrict__ F, int comp, int Nx, int Ny, int Nz)
{
    int Kx1 = Nx / 2 + 1, Ky1 = Ny / 2 + 1, Kz1 = Nz / 2 + 1;
    long long nk = (long long)Kx1 * Ky1 * Kz1;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nk; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q % Kx1);
        int j = (int)((q / Kx1) % Ky1);
        int k = (int)(q / ((long long)Kx1 * Ky1));
        K[comp * nk + q] = (T)F[(long long)i + (long long)j * Nx + (long long)k * Nx * Ny].x;
    }
}

// Generic strided batched line FFT (setup path and tests): line li (0 <= li < ninner), outer index
// blockIdx.y; element e at data[li * ls + e * es + blockIdx.y * os]. A block transforms W lines.
template <typename T, bool INV>
__global__ void __launch_bounds__(bm_lb<T>::v) k_fft_strided(cpx<T> *data, FFTPlan P, const cpx<T> *__restrict__ tw, long long es, long long ls,
                              int ninner, int W, long long os)
{
    extern __shared__ unsigned char smraw[];
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    int L = P.L;
    int li0 = blockIdx.x * W;
    cpx<T> *g = data + (long long)blockIdx.y * os;
    int nt = blockDim.x;
    // load tile [e][w]
    for (int idx = threadIdx.x; idx < L * W; idx += nt) {
        int e, w;
        if (es == 1) { w = idx / L; e = idx % L; }
        else { e = idx / W; w = idx % W; }
        int li = li0 + w;
        sm[e * W + w] = (li < ninner) ? g[(long long)li * ls + (long long)e * es] : mk<T>(0, 0);
    }
    __syncthreads();
    int l = threadIdx.x % W, t = threadIdx.x / W;
    bool active = t < P.tpl;
    fft_line<T, false, INV>(sm + l, W, t, active, P, tw);
    for (int idx = threadIdx.x; idx < L * W; idx += nt) {
        int e, w;
        if (es == 1) { w = idx / L; e = idx % L; }
        else { e = idx / W; w = idx % W; }
        int li = li0 + w;
        if (li < ninner) g[(long long)li * ls + (long long)e * es] = sm[e * W + w];
    }
}

template <typename T>
int launch_fft_strided(cpx<T> *data, const FFTPlan &P, const cpx<T> *tw, long long es, long long ls, int ninner,
                       long long os, int nouter, bool inv, cudaStream_t s)
{
    int W = 1;
    while (W < 8 && W < ninner) W *= 2;
    size_t smem = (size_t)P.L * W * sizeof(cpx<T>);
    while ((smem > 96 * 1024 || W * P.tpl > bm_lb<T>::v) && W > 1) { W /= 2; smem = (size_t)P.L * W * sizeof(cpx<T>); }
    int nt = W * P.tpl;
    if (nt < 32) nt = 32;
    if (nt > bm_lb<T>::v) return 1;
    dim3 grid((ninner + W - 1) / W, nouter);
    if (inv) {
        if (smem > BM_SMEM_DEFAULT_SAFE) cudaFuncSetAttribute(k_fft_strided<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        k_fft_strided<T, true><<<grid, nt, smem, s>>>(data, P, tw, es, ls, ninner, W, os);
    } else {
        if (smem > BM_SMEM_DEFAULT_SAFE) cudaFuncSetAttribute(k_fft_strided<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        k_fft_strided<T, false><<<grid, nt, smem, s>>>(data, P, tw, es, ls, ninner, W, os);
    }
    return (int)cudaGetLastError();
}

template int launch_fft_strided<float>(cpx<float> *, const FFTPlan &, const cpx<float> *, long long, long long, int, long long, int, bool, cudaStream_t);
template int launch_fft_strided<double>(cpx<double> *, const FFTPlan &, const cpx<double> *, long long, long long, int, long long, int, bool, cudaStream_t);

static int grid_for(long long n)
{
    long long b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return (int)b;
}

static bool pbc_on(const int *pbc) { return pbc && (pbc[0] || pbc[1] || pbc[2]); }

static void launch_octant(double *oct, int nx, int ny, int nz, double hx, double hy, double hz, const double *farq_dev,
                          const int *pbc, cudaStream_t s)
{
    if (pbc_on(pbc)) {
        PbcSpec P;
        P.n[0] = nx; P.n[1] = ny; P.n[2] = nz;
        for (int a = 0; a < 3; a++) P.img[a] = abs(pbc[a]);
        long long nc = 1;
        for (int a = 0; a < 3; a++) nc *= P.img[a] ? P.n[a] / 2 + 1 : P.n[a];
        k_tensor_octant_pbc<<<grid_for(nc), 128, 0, s>>>(oct, P, hx, hy, hz, farq_dev, nz == 1);
    } else {
        k_tensor_octant<<<grid_for((long long)nx * ny * nz), 256, 0, s>>>(oct, nx, ny, nz, hx, hy, hz, farq_dev, nz == 1);
    }
}

// Build the kernel planes (6 components, type T) for one mesh on the device.
// twx/twy/twz are FP64 tables of exp(-2 pi i m / N) for N = Nx, Ny, Nz. pbc: images per axis
// (negative values count as their magnitude, as for the reference's demag) or nullptr.
template <typename T>
int build_kernels_device(T *K, int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
                         const double *farq_dev, const cpx<double> *twx, const cpx<double> *twy,
                         const cpx<double> *twz, cudaStream_t s, const int *pbc)
{
    double hm = fmax(hx, fmax(hy, hz));
    hx /= hm; hy /= hm; hz /= hm;
    long long noct = (long long)nx * ny * nz;
    long long Ntot = (long long)Nx * Ny * Nz;
    double *oct = nullptr;
    cpx<double> *F = nullptr;
    if (cudaMalloc(&oct, sizeof(double) * 6 * noct) != cudaSuccess) return 2;
    if (cudaMalloc(&F, sizeof(cpx<double>) * Ntot) != cudaSuccess) { cudaFree(oct); return 2; }
    launch_octant(oct, nx, ny, nz, hx, hy, hz, farq_dev, pbc, s);
    FFTPlan px, py, pz;
    bm_make_plan(Nx, px); bm_make_plan(Ny, py); bm_make_plan(Nz, pz);
    int rc = 0;
    for (int c = 0; c < 6 && !rc; c++) {
        if (nz == 1 && (c == 4 || c == 5)) {
            cudaMemsetAsync(K + (long long)c * (Nx / 2 + 1) * (Ny / 2 + 1) * (Nz / 2 + 1), 0,
                            sizeof(T) * (Nx / 2 + 1) * (Ny / 2 + 1) * (Nz / 2 + 1), s);
            continue;
        }
        k_tensor_fill<<<grid_for(Ntot), 256, 0, s>>>(F, oct, c, nx, ny, nz, Nx, Ny, Nz);
        // x lines: contiguous, Ny*Nz of them
        if (Nx > 1) rc |= launch_fft_strided<double>(F, px, twx, 1, Nx, Ny * Nz, 0, 1, false, s);
        // y lines: stride Nx, Nx lines per z plane
        if (Ny > 1) rc |= launch_fft_strided<double>(F, py, twy, Nx, 1, Nx, (long long)Nx * Ny, Nz, false, s);
        // z lines: stride Nx*Ny, Nx*Ny lines
        if (Nz > 1) rc |= launch_fft_strided<double>(F, pz, twz, (long long)Nx * Ny, 1, Nx * Ny, 0, 1, false, s);
        k_tensor_extract<T><<<grid_for((long long)(Nx / 2 + 1) * (Ny / 2 + 1) * (Nz / 2 + 1)), 256, 0, s>>>(K, F, c, Nx, Ny, Nz);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(oct);
    cudaFree(F);
    if (e != cudaSuccess) return 3;
    return rc ? 4 : (int)cudaGetLastError();
}

template int build_kernels_device<float>(float *, int, int, int, int, int, int, double, double, double, const double *,
                                         const cpx<double> *, const cpx<double> *, const cpx<double> *, cudaStream_t,
                                         const int *);
template int build_kernels_device<double>(double *, int, int, int, int, int, int, double, double, double, const double *,
                                          const cpx<double> *, const cpx<double> *, const cpx<double> *, cudaStream_t,
                                          const int *);

// raw tensor octant to host (tests); with pbc the octant of the periodic kernel
int tensor_octant_device(double *oct_dev, int nx, int ny, int nz, double hx, double hy, double hz, const double *farq_dev,
                         cudaStream_t s, const int *pbc)
{
    double hm = fmax(hx, fmax(hy, hz));
    launch_octant(oct_dev, nx, ny, nz, hx / hm, hy / hm, hz / hm, farq_dev, pbc, s);
    return (int)cudaGetLastError();
}

// ============================================================================ multilayer kernels
// Shifted kernels of the multilayered convolution (Boris/DemagKernelCollection_Calc.cpp):
//   regular cells (3D, or 2D with equal thickness)  Boris/DemagTFunc_Shifted.cpp:6,120,235,343
//   2D, source and destination thickness differ    Boris/DemagTFunc_Irregular.cpp:4,121
// evaluated per grid offset (i, j, k) in (-n, n) on each axis with the shift added, near field
// by exact Newell sums, far field (beyond 40 cells, measured with the shift) by this project's
// expansion. The irregular sums follow the reference's combination: xx, yy take z in
// {D-s, D, D+d, D+d-s}, zz, xy, xz, yz take z in {D-d, D, D+s, D+s-d} (D the shift, s and d the
// source and destination thickness); the irregular far field is the destination-cell
// expansion at z = D scaled by the source thickness, as the reference computes it.
struct MLTP {
    double hs[3], hd[3], sh[3];
    int irregular;
};

__device__ __forceinline__ double floor_r(double v) { return floor(v + 1e-4); }

// 36-point irregular sum for one component (c: 0 xx, 1 yy, 2 zz, 3 xy, 4 xz, 5 yz)
__device__ double ml_irregular(int c, double x, double y, double z, const MLTP &P)
{
    const double hx = P.hd[0], hy = P.hd[1], s = P.hs[2], d = P.hd[2];
    const bool setA = (c < 2);
    const double zq[4] = {setA ? z - s : z - d, z, setA ? z + d : z + s, setA ? z + d - s : z + s - d};
    const double wz[4] = {-1.0, 1.0, -1.0, 1.0};
    const double cw[3] = {-1.0, 2.0, -1.0};
    double v[36];
    int m = 0;
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int q = 0; q < 4; q++) {
                double w = cw[a + 1] * cw[b + 1] * wz[q], val;
                switch (c) {
                case 0: val = nf(x + a * hx, y + b * hy, zq[q]); break;
                case 1: val = nf(y + a * hy, x + b * hx, zq[q]); break;
                case 2: val = nf(zq[q], y + a * hy, x + b * hx); break;
                case 3: val = ng(x + a * hx, y + b * hy, zq[q]); break;
                case 4: val = ng(x + a * hx, zq[q], y + b * hy); break;
                default: val = ng(y + a * hy, zq[q], x + b * hx); break;
                }
                v[m++] = w * val;
            }
    return -csum_d(v, 36) / (4.0 * M_PI * hx * hy * d);
}

// D6[c * np + p] for the (2n-1)^3 box of offsets, p the position on the N grid
__global__ void k_ml_tensor(double *D6, long long np, MLTP P, int nx, int ny, int nz, int Nx, int Ny, int Nz,
                            const double *__restrict__ farq)
{
    const long long bx = 2 * nx - 1, by = 2 * ny - 1, bz = 2 * nz - 1;
    const long long nb = bx * by * bz;
    const bool two_d = (nz == 1);
    const double *h = P.irregular ? P.hd : P.hs;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb; t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t % bx) - (nx - 1);
        int j = (int)((t / bx) % by) - (ny - 1);
        int k = (int)(t / (bx * by)) - (nz - 1);
        double is = fabs(i + P.sh[0] / h[0]), js = fabs(j + P.sh[1] / h[1]), ks = fabs(k + P.sh[2] / h[2]);
        bool far = ((int)floor_r(is) >= BM_ASYMPT_DIST || (int)floor_r(js) >= BM_ASYMPT_DIST || (int)floor_r(ks) >= BM_ASYMPT_DIST ||
                    (int)floor_r(is * is + js * js + ks * ks) >= BM_ASYMPT_DIST * BM_ASYMPT_DIST);
        double x = i * h[0] + P.sh[0], y = j * h[1] + P.sh[1], z = k * h[2] + P.sh[2];
        double v[6];
        if (far) {
            double R = sqrt(x * x + y * y + z * z);
            double V = h[0] * h[1] * h[2] / (4.0 * M_PI);
            if (P.irregular) V *= P.hs[2];
            for (int c = 0; c < 6; c++) v[c] = V * far_eval(farq + c * BM_FARQ_PER_COMP, x / R, y / R, z / R, R);
        } else if (!P.irregular) {
            v[0] = -newellL<false>(x, y, z, h[0], h[1], h[2]);
            v[1] = -newellL<false>(y, x, z, h[1], h[0], h[2]);
            v[2] = -newellL<false>(z, y, x, h[2], h[1], h[0]);
            v[3] = -newellL<true>(x, y, z, h[0], h[1], h[2]);
            v[4] = -newellL<true>(x, z, y, h[0], h[2], h[1]);
            v[5] = -newellL<true>(y, z, x, h[1], h[2], h[0]);
        } else {
            for (int c = 0; c < 6; c++) v[c] = ml_irregular(c, x, y, z, P);
        }
        if (two_d && P.sh[0] == 0.0 && P.sh[1] == 0.0 && P.sh[2] == 0.0) { v[4] = 0.0; v[5] = 0.0; }
        long long p = (long long)((i + Nx) % Nx) + (long long)((j + Ny) % Ny) * Nx + (long long)((k + Nz) % Nz) * Nx * Ny;
        for (int c = 0; c < 6; c++) D6[c * np + p] = v[c];
    }
}

__global__ void k_ml_to_complex(cpx<double> *F, const double *__restrict__ D, long long np)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x)
        F[p] = mk<double>(D[p], 0.0);
}

// complex spectra of one component: z-shifted kernels keep ky <= Ny/2, kz <= Nz/2 (the rest
// follows from the x/y parity and the Hermitian symmetry); full kernels keep every ky, kz
template <typename T>
__global__ void k_ml_extract(cpx<T> *K, const cpx<double> *__restrict__ F, int kind, int Nx, int Ny, int Nz)
{
    const int Kx1 = Nx / 2 + 1;
    const int ny = (kind == BM_MLK_ZSHIFT) ? Ny / 2 + 1 : Ny;
    const int nzk = (kind == BM_MLK_ZSHIFT) ? Nz / 2 + 1 : Nz;
    const long long nk = (long long)Kx1 * ny * nzk;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nk; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q % Kx1);
        int j = (int)((q / Kx1) % ny);
        int k = (int)(q / ((long long)Kx1 * ny));
        cpx<double> v = F[(long long)i + (long long)j * Nx + (long long)k * Nx * Ny];
        K[q] = mk<T>((T)v.x, (T)v.y);
    }
}

template <typename T>
int build_ml_kernel_device(T *K, const MLKernelSpec &spec, const int *nc, const int *N, const double *farq_dev,
                           const cpx<double> *twx, const cpx<double> *twy, const cpx<double> *twz, cudaStream_t s)
{
    const int Nx = N[0], Ny = N[1], Nz = N[2];
    if (spec.kind == BM_MLK_SELF)
        return build_kernels_device<T>(K, nc[0], nc[1], nc[2], Nx, Ny, Nz, spec.hd[0], spec.hd[1], spec.hd[2], farq_dev, twx,
                                       twy, twz, s);
    const long long np = (long long)Nx * Ny * Nz;
    double *D6 = nullptr;
    cpx<double> *F = nullptr;
    if (cudaMalloc(&D6, sizeof(double) * 6 * np) != cudaSuccess) return 2;
    if (cudaMalloc(&F, sizeof(cpx<double>) * np) != cudaSuccess) { cudaFree(D6); return 2; }
    cudaMemsetAsync(D6, 0, sizeof(double) * 6 * np, s);
    MLTP P;
    for (int a = 0; a < 3; a++) { P.hs[a] = spec.hs[a]; P.hd[a] = spec.hd[a]; P.sh[a] = spec.shift[a]; }
    P.irregular = spec.irregular;
    long long nb = (long long)(2 * nc[0] - 1) * (2 * nc[1] - 1) * (2 * nc[2] - 1);
    k_ml_tensor<<<grid_for(nb), 256, 0, s>>>(D6, np, P, nc[0], nc[1], nc[2], Nx, Ny, Nz, farq_dev);
    FFTPlan px, py, pz;
    bm_make_plan(Nx, px); bm_make_plan(Ny, py); bm_make_plan(Nz, pz);
    const int Kx1 = Nx / 2 + 1;
    const long long nk = (spec.kind == BM_MLK_ZSHIFT) ? (long long)Kx1 * (Ny / 2 + 1) * (Nz / 2 + 1) : (long long)Kx1 * Ny * Nz;
    int rc = 0;
    for (int c = 0; c < 6 && !rc; c++) {
        k_ml_to_complex<<<grid_for(np), 256, 0, s>>>(F, D6 + c * np, np);
        if (Nx > 1) rc |= launch_fft_strided<double>(F, px, twx, 1, Nx, Ny * Nz, 0, 1, false, s);
        if (Ny > 1) rc |= launch_fft_strided<double>(F, py, twy, Nx, 1, Nx, (long long)Nx * Ny, Nz, false, s);
        if (Nz > 1) rc |= launch_fft_strided<double>(F, pz, twz, (long long)Nx * Ny, 1, Nx * Ny, 0, 1, false, s);
        k_ml_extract<T><<<grid_for(nk), 256, 0, s>>>(reinterpret_cast<cpx<T> *>(K) + c * nk, F, spec.kind, Nx, Ny, Nz);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(D6);
    cudaFree(F);
    if (e != cudaSuccess) return 3;
    return rc ? 4 : (int)cudaGetLastError();
}

template int build_ml_kernel_device<float>(float *, const MLKernelSpec &, const int *, const int *, const double *,
                                           const cpx<double> *, const cpx<double> *, const cpx<double> *, cudaStream_t);
template int build_ml_kernel_device<double>(double *, const MLKernelSpec &, const int *, const int *, const double *,
                                            const cpx<double> *, const cpx<double> *, const cpx<double> *, cudaStream_t);
