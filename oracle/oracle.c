/*
 * Oracle (test infrastructure only; never linked into the product path).
 *
 * FP64 CPU restatement of the reference's per-step micromagnetic path:
 *   Newell demag tensor        Boris/DemagTFunc_fg.cpp:10,45 (f, g), Boris/DemagTFunc_L.cpp:8,59
 *                              (27-point second differences), Boris/DemagTFunc.cpp:21,95,172,237
 *                              (octant fill with parity), Boris/DemagTFunc_Self.cpp:6
 *   far field                  the reference switches to an asymptotic expansion at
 *                              ASYMPTOTIC_DISTANCE = 40 cells (Boris/DemagTFunc_Defs.h:9,
 *                              DemagTFunc.cpp:57). The expansion here is derived for this
 *                              project: the Newell tensor is the double cell average of
 *                              -(1/4pi) d_i d_j (1/R); the average over two boxes is the
 *                              operator prod_k (sinh(a_k)/a_k)^2, a_k = h_k d_k / 2, whose
 *                              Taylor series 1 + h^2 d^2/12 + h^4 d^4/360 + h^6 d^6/20160 is
 *                              applied to d_i d_j (1/R) up to total order 8.
 *   kernel spectra             Boris/DemagKernel.cpp:171,317: real parts of the 3D DFT of the
 *                              tensor on the (Nx/2+1)(Ny/2+1)(Nz/2+1) octant
 *   convolution                Boris/Convolution.h:262,659 with the 3x3 product and mirror
 *                              signs of DemagKernel.cpp:42,85 (Kxy odd in x,y; Kxz odd in x,z;
 *                              Kyz odd in y,z)
 *   exchange                   Boris/Exchange.cpp:108 with BorisLib/VEC_VC_Del.h:10 (delsq_neu)
 *   interfacial DMI            Boris/iDMExchange.cpp:97 with BorisLib/VEC_VC_Del.h:141 (delsq_nneu),
 *                              BorisLib/VEC_VC_Grad.h:10,139 (grad_neu, grad_nneu)
 *   uniaxial anisotropy        Boris/Anisotropy.cpp:82
 *   Zeeman                     Boris/Zeeman.cpp:164 (sets Heff, first in the module list,
 *                              evaluated at the step start time: GetStageTime)
 *   LLG                        Boris/DiffEqFM_Equations.cpp:12
 *   RK4                        Boris/DiffEqFM_Evals_RK4.cpp:13-298, Boris/DiffEq_CommonBase_Iterate.cpp:576
 *   RKDP54                     Boris/DiffEqFM_Evals_RKDP54.cpp:9-260,
 *                              Boris/DiffEq_CommonBase_Iterate.cpp:1214 (FSAL, prime/restore)
 *   step control               Boris/DiffEq_CommonBase_Iterate.cpp:15 (SetAdaptiveTimeStep)
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

double *bm_fft_table(int n);
void bm_fft_table_free(double *tw);
void bm_fft_exec(int n, const double *tw, double *data, int sign, double *scratch);

#define ASYMPT_DIST 40

/* ------------------------------------------------------------------ sums */

/* Neumaier compensated sum of v[0..n) */
static double csum(const double *v, int n)
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

/* ------------------------------------------------------------------ Newell f, g */

/* Newell, Williams & Dunlop (1993) eq. 27; asinh written directly (odd symmetric). */
double orc_newell_f(double x, double y, double z)
{
    double x2 = x * x, y2 = y * y, z2 = z * z;
    double R = sqrt(x2 + y2 + z2);
    double t[4] = {0, 0, 0, 0};
    t[0] = (2.0 * x2 - y2 - z2) * R / 6.0;
    double rxz = sqrt(x2 + z2), rxy = sqrt(x2 + y2);
    if (rxz > 0.0) t[1] = 0.5 * y * (z2 - x2) * asinh(y / rxz);
    if (rxy > 0.0) t[2] = 0.5 * z * (y2 - x2) * asinh(z / rxy);
    if (x != 0.0 && R > 0.0) t[3] = -x * y * z * atan(y * z / (x * R));
    return csum(t, 4);
}

double orc_newell_g(double x, double y, double z)
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
    return csum(t, 7);
}

/* 27-point second difference with weights c(0)=2, c(+-1)=-1 per axis
 * (the combination of Newell's F/G functions, DemagTFunc_L.cpp:8-57) */
static double newell_L(double (*fn)(double, double, double), double x, double y, double z,
                       double hx, double hy, double hz)
{
    double v[27];
    int m = 0;
    static const double cw[3] = {-1.0, 2.0, -1.0};
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++)
                v[m++] = cw[a + 1] * cw[b + 1] * cw[c + 1] * fn(x + a * hx, y + b * hy, z + c * hz);
    return csum(v, 27) / (4.0 * M_PI * hx * hy * hz);
}

void orc_selfdemag(double hx, double hy, double hz, double *out3)
{
    /* DemagTFunc_Self.cpp:6,48: minus sign gives D = -N */
    out3[0] = -newell_L(orc_newell_f, 0, 0, 0, hx, hy, hz);
    out3[1] = -newell_L(orc_newell_f, 0, 0, 0, hy, hx, hz);
    out3[2] = -newell_L(orc_newell_f, 0, 0, 0, hz, hy, hx);
}

/* ------------------------------------------------------------------ far field */

/* Derivatives of 1/R: d^p_x d^q_y d^r_z (1/R) = P_pqr(x,y,z) / R^(2n+1), n = p+q+r, where P is
 * a homogeneous integer polynomial of degree n obtained from
 *   P_{p+1,q,r} = R^2 dP/dx - (2n+1) x P   (and likewise for y, z).
 * Polynomials are stored densely as coef[i][j][k] of x^i y^j z^k. */
#define PD 9
typedef struct { double c[PD][PD][PD]; } poly3;

static void poly_step(const poly3 *P, int n, int axis, poly3 *out)
{
    memset(out, 0, sizeof(*out));
    for (int i = 0; i < PD; i++)
        for (int j = 0; j < PD; j++)
            for (int k = 0; k < PD; k++) {
                double c = P->c[i][j][k];
                if (c == 0.0) continue;
                int e[3] = {i, j, k};
                /* derivative along axis times R^2 = x^2 + y^2 + z^2 */
                if (e[axis] > 0) {
                    int d[3] = {i, j, k};
                    d[axis] -= 1;
                    double dc = c * e[axis];
                    for (int s = 0; s < 3; s++) {
                        int f[3] = {d[0], d[1], d[2]};
                        f[s] += 2;
                        if (f[0] < PD && f[1] < PD && f[2] < PD) out->c[f[0]][f[1]][f[2]] += dc;
                    }
                }
                /* -(2n+1) x_axis P */
                int g[3] = {i, j, k};
                g[axis] += 1;
                if (g[0] < PD && g[1] < PD && g[2] < PD) out->c[g[0]][g[1]][g[2]] -= (2.0 * n + 1.0) * c;
            }
}

/* evaluate homogeneous polynomial at unit vector (u,v,w) */
static double poly_eval(const poly3 *P, double u, double v, double w)
{
    double pu[PD], pv[PD], pw[PD];
    pu[0] = pv[0] = pw[0] = 1.0;
    for (int i = 1; i < PD; i++) { pu[i] = pu[i - 1] * u; pv[i] = pv[i - 1] * v; pw[i] = pw[i - 1] * w; }
    double t[PD * PD * PD];
    int m = 0;
    for (int i = 0; i < PD; i++)
        for (int j = 0; j < PD; j++)
            for (int k = 0; k < PD; k++)
                if (P->c[i][j][k] != 0.0) t[m++] = P->c[i][j][k] * pu[i] * pv[j] * pw[k];
    return csum(t, m);
}

/* P_pqr for all p+q+r <= 8, built once */
static poly3 *g_dpoly = 0;
static int dpoly_index(int p, int q, int r) { return (p * PD + q) * PD + r; }

static void build_dpoly(void)
{
    if (g_dpoly) return;
    poly3 *T = (poly3 *)calloc((size_t)PD * PD * PD, sizeof(poly3));
    T[dpoly_index(0, 0, 0)].c[0][0][0] = 1.0;
    for (int p = 0; p < PD; p++)
        for (int q = 0; q < PD; q++)
            for (int r = 0; r < PD; r++) {
                int n = p + q + r;
                if (n > 8 || n == 0) continue;
                if (r > 0) poly_step(&T[dpoly_index(p, q, r - 1)], n - 1, 2, &T[dpoly_index(p, q, r)]);
                else if (q > 0) poly_step(&T[dpoly_index(p, q - 1, 0)], n - 1, 1, &T[dpoly_index(p, q, 0)]);
                else poly_step(&T[dpoly_index(p - 1, 0, 0)], n - 1, 0, &T[dpoly_index(p, 0, 0)]);
            }
    g_dpoly = T;
}

void orc_asymptotic(double hx, double hy, double hz, double x, double y, double z, double *out6)
{
#pragma omp critical(orc_dpoly)
    build_dpoly();
    static const double C[4] = {1.0, 1.0 / 12.0, 1.0 / 360.0, 1.0 / 20160.0};
    static const int comp[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    double R = sqrt(x * x + y * y + z * z);
    double u = x / R, v = y / R, w = z / R;
    double V = hx * hy * hz;
    for (int c = 0; c < 6; c++) {
        double terms[64];
        int m = 0;
        for (int a = 0; a <= 3; a++)
            for (int b = 0; a + b <= 3; b++)
                for (int cc = 0; a + b + cc <= 3; cc++) {
                    int e[3] = {2 * a, 2 * b, 2 * cc};
                    e[comp[c][0]] += 1;
                    e[comp[c][1]] += 1;
                    int n = e[0] + e[1] + e[2];
                    double coef = C[a] * C[b] * C[cc] * pow(hx, 2 * a) * pow(hy, 2 * b) * pow(hz, 2 * cc);
                    /* d^e (1/R) = P(u,v,w) / R^(n+1) */
                    terms[m++] = coef * poly_eval(&g_dpoly[dpoly_index(e[0], e[1], e[2])], u, v, w) / pow(R, n + 1);
                }
        out6[c] = V / (4.0 * M_PI) * csum(terms, m);
    }
}

/* ------------------------------------------------------------------ tensor on the N grid */

static int use_asympt(int i, int j, int k)
{
    return (i >= ASYMPT_DIST || j >= ASYMPT_DIST || k >= ASYMPT_DIST ||
            (long)i * i + (long)j * j + (long)k * k >= (long)ASYMPT_DIST * ASYMPT_DIST);
}

int orc_tensor(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
               double *diag, double *odiag)
{
    double hm = hx;
    if (hy > hm) hm = hy;
    if (hz > hm) hm = hz;
    hx /= hm; hy /= hm; hz /= hm;
    size_t np = (size_t)Nx * Ny * Nz;
    memset(diag, 0, sizeof(double) * 3 * np);
    memset(odiag, 0, sizeof(double) * 3 * np);
    int two_d = (nz == 1);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                double dv[3], ov[3];
                double x = i * hx, y = j * hy, z = k * hz;
                if (use_asympt(i, j, k)) {
                    double a[6];
                    orc_asymptotic(hx, hy, hz, x, y, z, a);
                    dv[0] = a[0]; dv[1] = a[1]; dv[2] = a[2];
                    ov[0] = a[3]; ov[1] = a[4]; ov[2] = a[5];
                } else {
                    /* D = -N; Nyy, Nzz by permuting f's arguments (DemagTFunc.cpp:59-62) */
                    dv[0] = -newell_L(orc_newell_f, x, y, z, hx, hy, hz);
                    dv[1] = -newell_L(orc_newell_f, y, x, z, hy, hx, hz);
                    dv[2] = -newell_L(orc_newell_f, z, y, x, hz, hy, hx);
                    ov[0] = -newell_L(orc_newell_g, x, y, z, hx, hy, hz);
                    ov[1] = -newell_L(orc_newell_g, x, z, y, hx, hz, hy);
                    ov[2] = -newell_L(orc_newell_g, y, z, x, hy, hz, hx);
                }
                if (two_d) { ov[1] = 0.0; ov[2] = 0.0; }
                for (int sx = -1; sx <= 1; sx += 2)
                    for (int sy = -1; sy <= 1; sy += 2)
                        for (int sz = -1; sz <= 1; sz += 2) {
                            int ii = ((sx * i) % Nx + Nx) % Nx;
                            int jj = ((sy * j) % Ny + Ny) % Ny;
                            int kk = ((sz * k) % Nz + Nz) % Nz;
                            size_t p = (size_t)ii + (size_t)jj * Nx + (size_t)kk * Nx * Ny;
                            diag[3 * p + 0] = dv[0]; diag[3 * p + 1] = dv[1]; diag[3 * p + 2] = dv[2];
                            /* xy odd in x,y; xz odd in x,z; yz odd in y,z */
                            odiag[3 * p + 0] = ov[0] * sx * sy;
                            odiag[3 * p + 1] = ov[1] * sx * sz;
                            odiag[3 * p + 2] = ov[2] * sy * sz;
                        }
            }
    return 0;
}

/* ------------------------------------------------------------------ 3D DFT helpers */

/* in-place complex 3D DFT of c[Nx*Ny*Nz] (interleaved re,im), all three axes */
static void dft3(double *c, int Nx, int Ny, int Nz, int sign)
{
    int dims[3] = {Nx, Ny, Nz};
    size_t strides[3] = {1, (size_t)Nx, (size_t)Nx * Ny};
    for (int ax = 0; ax < 3; ax++) {
        int L = dims[ax];
        if (L == 1) continue;
        double *tw = bm_fft_table(L);
        size_t nlines = (size_t)Nx * Ny * Nz / L;
#pragma omp parallel
        {
            double *line = (double *)malloc(sizeof(double) * 2 * L);
            double *scr = (double *)malloc(sizeof(double) * 4 * L);
#pragma omp for
            for (long li = 0; li < (long)nlines; li++) {
                /* decompose line index into the two other coordinates */
                size_t base;
                if (ax == 0) base = (size_t)li * Nx;
                else if (ax == 1) base = ((size_t)li % Nx) + ((size_t)li / Nx) * Nx * Ny;
                else base = (size_t)li;
                for (int t = 0; t < L; t++) {
                    line[2 * t] = c[2 * (base + t * strides[ax])];
                    line[2 * t + 1] = c[2 * (base + t * strides[ax]) + 1];
                }
                bm_fft_exec(L, tw, line, sign, scr);
                for (int t = 0; t < L; t++) {
                    c[2 * (base + t * strides[ax])] = line[2 * t];
                    c[2 * (base + t * strides[ax]) + 1] = line[2 * t + 1];
                }
            }
            free(line); free(scr);
        }
        bm_fft_table_free(tw);
    }
}

int orc_kernels(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
                double *kdiag, double *kodiag)
{
    size_t np = (size_t)Nx * Ny * Nz;
    double *dg = (double *)malloc(sizeof(double) * 3 * np);
    double *od = (double *)malloc(sizeof(double) * 3 * np);
    double *c = (double *)malloc(sizeof(double) * 2 * np);
    orc_tensor(nx, ny, nz, Nx, Ny, Nz, hx, hy, hz, dg, od);
    int Kx = Nx / 2 + 1, Ky = Ny / 2 + 1, Kz = Nz / 2 + 1;
    for (int comp = 0; comp < 6; comp++) {
        const double *src = comp < 3 ? dg : od;
        int cc = comp % 3;
        for (size_t p = 0; p < np; p++) { c[2 * p] = src[3 * p + cc]; c[2 * p + 1] = 0.0; }
        dft3(c, Nx, Ny, Nz, -1);
        double *dst = comp < 3 ? kdiag : kodiag;
        for (int k = 0; k < Kz; k++)
            for (int j = 0; j < Ky; j++)
                for (int i = 0; i < Kx; i++) {
                    size_t p = (size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny;
                    size_t q = (size_t)i + (size_t)j * Kx + (size_t)k * Kx * Ky;
                    dst[3 * q + cc] = c[2 * p];
                }
    }
    free(dg); free(od); free(c);
    return 0;
}

/* ------------------------------------------------------------------ convolution */

struct orc_demag {
    int nx, ny, nz, Nx, Ny, Nz;
    double *kd, *ko;   /* octant kernels */
};

orc_demag *orc_demag_create(int nx, int ny, int nz, double hx, double hy, double hz, int Nx, int Ny, int Nz)
{
    orc_demag *d = (orc_demag *)calloc(1, sizeof(orc_demag));
    d->nx = nx; d->ny = ny; d->nz = nz; d->Nx = Nx; d->Ny = Ny; d->Nz = Nz;
    size_t nk = (size_t)(Nx / 2 + 1) * (Ny / 2 + 1) * (Nz / 2 + 1);
    d->kd = (double *)malloc(sizeof(double) * 3 * nk);
    d->ko = (double *)malloc(sizeof(double) * 3 * nk);
    orc_kernels(nx, ny, nz, Nx, Ny, Nz, hx, hy, hz, d->kd, d->ko);
    return d;
}

void orc_demag_destroy(orc_demag *d)
{
    if (!d) return;
    free(d->kd); free(d->ko); free(d);
}

double orc_demag_apply(orc_demag *d, const double *M, double *H, int add)
{
    int nx = d->nx, ny = d->ny, nz = d->nz, Nx = d->Nx, Ny = d->Ny, Nz = d->Nz;
    size_t np = (size_t)Nx * Ny * Nz;
    double *F[3];
    for (int c = 0; c < 3; c++) {
        F[c] = (double *)calloc(2 * np, sizeof(double));
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    size_t p = (size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny;
                    F[c][2 * p] = M[3 * ((size_t)i + (size_t)j * nx + (size_t)k * nx * ny) + c];
                }
        dft3(F[c], Nx, Ny, Nz, -1);
    }
    int Kx = Nx / 2 + 1, Ky = Ny / 2 + 1;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++) {
                int ai = i <= Nx / 2 ? i : Nx - i, sx = i <= Nx / 2 ? 1 : -1;
                int aj = j <= Ny / 2 ? j : Ny - j, sy = j <= Ny / 2 ? 1 : -1;
                int ak = k <= Nz / 2 ? k : Nz - k, sz = k <= Nz / 2 ? 1 : -1;
                size_t q = (size_t)ai + (size_t)aj * Kx + (size_t)ak * Kx * Ky;
                double kxx = d->kd[3 * q], kyy = d->kd[3 * q + 1], kzz = d->kd[3 * q + 2];
                double kxy = d->ko[3 * q] * sx * sy, kxz = d->ko[3 * q + 1] * sx * sz, kyz = d->ko[3 * q + 2] * sy * sz;
                size_t p = (size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny;
                for (int ri = 0; ri < 2; ri++) {
                    double mx = F[0][2 * p + ri], my = F[1][2 * p + ri], mz = F[2][2 * p + ri];
                    F[0][2 * p + ri] = kxx * mx + kxy * my + kxz * mz;
                    F[1][2 * p + ri] = kxy * mx + kyy * my + kyz * mz;
                    F[2][2 * p + ri] = kxz * mx + kyz * my + kzz * mz;
                }
            }
    double inv = 1.0 / (double)np;
    double dot = 0.0;
    for (int c = 0; c < 3; c++) {
        dft3(F[c], Nx, Ny, Nz, +1);
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    size_t p = (size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny;
                    size_t cell = (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
                    double h = F[c][2 * p] * inv;
                    dot += M[3 * cell + c] * h;
                    if (add) H[3 * cell + c] += h;
                    else H[3 * cell + c] = h;
                }
        free(F[c]);
    }
    return dot;
}

/* ------------------------------------------------------------------ field terms */

static double ms_at(const double *Ms_cell, size_t i) { return Ms_cell[i]; }

/* one axis of delsq_nneu / grad_nneu (VEC_VC_Del.h:141-200, VEC_VC_Grad.h:139-183) for a
 * full rectangular mesh without PBC; bd = boundary differential along this axis (0 = neu) */
static void axis_terms(const double *M, size_t idx, int coord, int ncoord, size_t stride, double h,
                       const double *bd, double *d2, double *g)
{
    int has_p = coord + 1 < ncoord, has_m = coord > 0;
    for (int c = 0; c < 3; c++) {
        double q = M[3 * idx + c];
        if (has_p && has_m) {
            double qp = M[3 * (idx + stride) + c], qm = M[3 * (idx - stride) + c];
            d2[c] = (qp + qm - 2.0 * q) / (h * h);
            g[c] = (qp - qm) / (2.0 * h);
        } else if (has_p) {
            double qp = M[3 * (idx + stride) + c];
            d2[c] = ((qp - q) - bd[c] * h) / (h * h);
            g[c] = 0.5 * ((qp - q) / h + bd[c]);
        } else if (has_m) {
            double qm = M[3 * (idx - stride) + c];
            d2[c] = ((qm - q) + bd[c] * h) / (h * h);
            g[c] = 0.5 * ((q - qm) / h + bd[c]);
        } else {
            d2[c] = 0.0;
            g[c] = 0.0;
        }
    }
}

void orc_field_exchange(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                        double A, const double *Ms_cell, double *H)
{
    static const double zero[3] = {0, 0, 0};
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
                double dx[3], dy[3], dz[3], g[3];
                axis_terms(M, idx, i, nx, 1, hx, zero, dx, g);
                axis_terms(M, idx, j, ny, nx, hy, zero, dy, g);
                axis_terms(M, idx, k, nz, (size_t)nx * ny, hz, zero, dz, g);
                double Ms = ms_at(Ms_cell, idx);
                double cst = 2.0 * A / (ORC_MU0 * Ms * Ms);
                for (int c = 0; c < 3; c++) H[3 * idx + c] += cst * (dx[c] + dy[c] + dz[c]);
            }
}

void orc_field_idmi(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                    double A, double D, const double *Ms_cell, double *H)
{
    static const double zero[3] = {0, 0, 0};
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
                const double *m = M + 3 * idx;
                double r = D / (2.0 * A);
                double bx[3] = {r * m[2], 0.0, -r * m[0]};
                double by[3] = {0.0, r * m[2], -r * m[1]};
                double dx[3], dy[3], dz[3], gx[3], gy[3], gz[3];
                axis_terms(M, idx, i, nx, 1, hx, bx, dx, gx);
                axis_terms(M, idx, j, ny, nx, hy, by, dy, gy);
                axis_terms(M, idx, k, nz, (size_t)nx * ny, hz, zero, dz, gz);
                double Ms = ms_at(Ms_cell, idx);
                double Ac = 2.0 * A / (ORC_MU0 * Ms * Ms);
                double Dc = -2.0 * D / (ORC_MU0 * Ms * Ms);
                double hd[3] = {gx[2], gy[2], -gx[0] - gy[1]};
                for (int c = 0; c < 3; c++) H[3 * idx + c] += Ac * (dx[c] + dy[c] + dz[c]) + Dc * hd[c];
            }
}

void orc_field_aniuni(int n, const double *M, const double *Ms_cell, const double *K1_cell, double K2,
                      const double *ea, double *H)
{
#pragma omp parallel for
    for (int i = 0; i < n; i++) {
        double Ms = Ms_cell[i], K1 = K1_cell[i];
        const double *m = M + 3 * (size_t)i;
        double dp = (m[0] * ea[0] + m[1] * ea[1] + m[2] * ea[2]) / Ms;
        double s = (2.0 / (ORC_MU0 * Ms)) * dp * (K1 + 2.0 * K2 * (1.0 - dp * dp));
        for (int c = 0; c < 3; c++) H[3 * (size_t)i + c] += s * ea[c];
    }
}

/* ------------------------------------------------------------------ solver */

typedef struct {
    orc_mesh_desc d;
    int n;
    double *Ms, *K1;         /* per-cell */
    double *M, *H, *sM1, *sEval[6];
    orc_demag *dm;
} orc_mesh;

struct orc_solver {
    int nmesh;
    orc_mesh *m;
    int eval;
    double dT, tol, dT_incr, dT_min, dT_max;
    double time, stagetime;
    int primed;
    long accepted, rejected, evals;
    double last_lte;
};

static int fft_size(int n) { return n > 1 ? 2 * n : 1; }

orc_solver *orc_solver_create(int nmesh, const orc_mesh_desc *desc, int eval, double dt, double tol,
                              double dT_incr, double dT_min, double dT_max)
{
    orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
    s->nmesh = nmesh;
    s->m = (orc_mesh *)calloc(nmesh, sizeof(orc_mesh));
    s->eval = eval;
    s->dT = dt; s->tol = tol; s->dT_incr = dT_incr; s->dT_min = dT_min; s->dT_max = dT_max;
    for (int q = 0; q < nmesh; q++) {
        orc_mesh *m = &s->m[q];
        m->d = desc[q];
        m->n = desc[q].nx * desc[q].ny * desc[q].nz;
        size_t n3 = 3 * (size_t)m->n;
        m->Ms = (double *)malloc(sizeof(double) * m->n);
        m->K1 = (double *)malloc(sizeof(double) * m->n);
        for (int i = 0; i < m->n; i++) {
            m->Ms[i] = desc[q].Ms_map ? desc[q].Ms_map[i] : desc[q].Ms;
            m->K1[i] = desc[q].K1_map ? desc[q].K1_map[i] : desc[q].K1;
        }
        m->M = (double *)calloc(n3, sizeof(double));
        m->H = (double *)calloc(n3, sizeof(double));
        m->sM1 = (double *)calloc(n3, sizeof(double));
        for (int e = 0; e < 6; e++) m->sEval[e] = (double *)calloc(n3, sizeof(double));
        if (desc[q].modules & ORC_DEMAG)
            m->dm = orc_demag_create(desc[q].nx, desc[q].ny, desc[q].nz, desc[q].hx, desc[q].hy, desc[q].hz,
                                     fft_size(desc[q].nx), fft_size(desc[q].ny), fft_size(desc[q].nz));
    }
    return s;
}

void orc_solver_destroy(orc_solver *s)
{
    if (!s) return;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        free(m->Ms); free(m->K1); free(m->M); free(m->H); free(m->sM1);
        for (int e = 0; e < 6; e++) free(m->sEval[e]);
        orc_demag_destroy(m->dm);
    }
    free(s->m);
    free(s);
}

int orc_set_m(orc_solver *s, int q, const double *M)
{
    memcpy(s->m[q].M, M, sizeof(double) * 3 * s->m[q].n);
    s->primed = 0;
    return 0;
}

int orc_get_m(orc_solver *s, int q, double *M)
{
    memcpy(M, s->m[q].M, sizeof(double) * 3 * s->m[q].n);
    return 0;
}

static void applied_field(const orc_mesh_desc *d, double t, double *Ha)
{
    Ha[0] = Ha[1] = Ha[2] = 0.0;
    if (!(d->modules & ORC_ZEEMAN) || !d->Ha || d->nHa <= 0) return;
    int idx = 0;
    if (d->nHa > 1 && d->Ha_tspan > 0.0) {
        idx = (int)floor(t / d->Ha_tspan * d->nHa);
        if (idx < 0) idx = 0;
        if (idx >= d->nHa) idx = d->nHa - 1;
    }
    Ha[0] = d->Ha[3 * idx]; Ha[1] = d->Ha[3 * idx + 1]; Ha[2] = d->Ha[3 * idx + 2];
}

/* module order Zeeman (sets) -> Demag -> Exchange/iDMI -> Anisotropy (MeshModules.cpp:131,
 * Mesh_Ferromagnetic.h:152) */
static void update_fields(orc_solver *s, orc_mesh *m)
{
    const orc_mesh_desc *d = &m->d;
    size_t n = (size_t)m->n;
    double Ha[3];
    applied_field(d, s->stagetime, Ha);
    for (size_t i = 0; i < n; i++) { m->H[3 * i] = Ha[0]; m->H[3 * i + 1] = Ha[1]; m->H[3 * i + 2] = Ha[2]; }
    if (d->modules & ORC_DEMAG) orc_demag_apply(m->dm, m->M, m->H, 1);
    if (d->modules & ORC_IDMI) orc_field_idmi(d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, m->M, d->A, d->D, m->Ms, m->H);
    else if (d->modules & ORC_EXCH) orc_field_exchange(d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, m->M, d->A, m->Ms, m->H);
    if (d->modules & ORC_ANIUNI) orc_field_aniuni(m->n, m->M, m->Ms, m->K1, d->K2, d->ea, m->H);
}

static void update_all_fields(orc_solver *s)
{
    for (int q = 0; q < s->nmesh; q++) update_fields(s, &s->m[q]);
    s->evals++;
}

int orc_compute_heff(orc_solver *s, int q, double *H)
{
    update_fields(s, &s->m[q]);
    memcpy(H, s->m[q].H, sizeof(double) * 3 * s->m[q].n);
    return 0;
}

/* DiffEqFM_Equations.cpp:12 */
static inline void llg(const double *M, const double *H, double Ms, double alpha, double grel, double *out)
{
    double mxh[3] = {M[1] * H[2] - M[2] * H[1], M[2] * H[0] - M[0] * H[2], M[0] * H[1] - M[1] * H[0]};
    double mm[3] = {M[0] / Ms, M[1] / Ms, M[2] / Ms};
    double mmxh[3] = {mm[1] * mxh[2] - mm[2] * mxh[1], mm[2] * mxh[0] - mm[0] * mxh[2], mm[0] * mxh[1] - mm[1] * mxh[0]};
    double pre = -ORC_GAMMA * grel / (1.0 + alpha * alpha);
    for (int c = 0; c < 3; c++) out[c] = pre * (mxh[c] + alpha * mmxh[c]);
}

static inline void renorm(double *M, double Ms)
{
    double nrm = sqrt(M[0] * M[0] + M[1] * M[1] + M[2] * M[2]);
    double f = Ms / nrm;
    M[0] *= f; M[1] *= f; M[2] *= f;
}

/* SetAdaptiveTimeStep (DiffEq_CommonBase_Iterate.cpp:15); returns 1 to accept */
static int adaptive_dt(orc_solver *s, double lte)
{
    if (s->dT_min == s->dT_max) return 1;
    int order = 5;
    if (lte > s->tol && s->dT > s->dT_min) {
        s->time -= s->dT;
        s->stagetime -= s->dT;
        s->accepted--;
        double c = pow(s->tol * 0.8 / lte, 1.0 / (order + 1));
        if (c < 0.01) c = 0.01;
        s->dT *= c;
        if (s->dT < s->dT_min) s->dT = s->dT_min;
        return 0;
    } else if (lte > 0) {
        double c = pow(s->tol * 0.8 / lte, 1.0 / (order + 1));
        if (c > s->dT_incr) c = s->dT_incr;
        if (c < 0.01) c = 0.01;
        s->dT *= c;
        if (s->dT < s->dT_min) s->dT = s->dT_min;
        if (s->dT > s->dT_max) s->dT = s->dT_max;
    }
    return 1;
}

static void rk4_step(orc_solver *s)
{
    double dT = s->dT;
    for (int stage = 0; stage < 4; stage++) {
        update_all_fields(s);
        for (int q = 0; q < s->nmesh; q++) {
            orc_mesh *m = &s->m[q];
            const orc_mesh_desc *d = &m->d;
#pragma omp parallel for
            for (int i = 0; i < m->n; i++) {
                double *M = m->M + 3 * (size_t)i, *H = m->H + 3 * (size_t)i;
                double *M1 = m->sM1 + 3 * (size_t)i;
                double f[3];
                llg(M, H, m->Ms[i], d->alpha, d->grel, f);
                double *e0 = m->sEval[0] + 3 * (size_t)i, *e1 = m->sEval[1] + 3 * (size_t)i, *e2 = m->sEval[2] + 3 * (size_t)i;
                for (int c = 0; c < 3; c++) {
                    if (stage == 0) { M1[c] = M[c]; e0[c] = f[c]; M[c] += f[c] * (dT / 2); }
                    else if (stage == 1) { e1[c] = f[c]; M[c] = M1[c] + f[c] * (dT / 2); }
                    else if (stage == 2) { e2[c] = f[c]; M[c] = M1[c] + f[c] * dT; }
                    else M[c] = M1[c] + (e0[c] + 2 * e1[c] + 2 * e2[c] + f[c]) * (dT / 6);
                }
                if (stage == 3) renorm(M, m->Ms[i]);
            }
        }
    }
    s->time += dT;
    s->stagetime += dT;
    s->accepted++;
}

/* one RKDP54 attempt: returns 1 if a step was completed, 0 if the previous one was rejected */
static int rkdp_attempt(orc_solver *s)
{
    /* evalStep 0: FSAL rhs, 4th-order prediction, lte (DiffEqFM_Evals_RKDP54.cpp:52-88) */
    update_all_fields(s);
    double lte = 0.0;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        const orc_mesh_desc *d = &m->d;
        double dT = s->dT;
        double lmax = 0.0;
#pragma omp parallel for reduction(max:lmax)
        for (int i = 0; i < m->n; i++) {
            size_t o = 3 * (size_t)i;
            double f[3];
            llg(m->M + o, m->H + o, m->Ms[i], d->alpha, d->grel, f);
            double dd[3];
            for (int c = 0; c < 3; c++) {
                double pred = m->sM1[o + c] + (5179.0 * m->sEval[0][o + c] / 57600 + 7571.0 * m->sEval[2][o + c] / 16695 +
                                               393.0 * m->sEval[3][o + c] / 640 - 92097.0 * m->sEval[4][o + c] / 339200 +
                                               187.0 * m->sEval[5][o + c] / 2100 + f[c] / 40) * dT;
                dd[c] = m->M[o + c] - pred;
            }
            double mn = sqrt(m->M[o] * m->M[o] + m->M[o + 1] * m->M[o + 1] + m->M[o + 2] * m->M[o + 2]);
            double l = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]) / mn;
            if (l > lmax) lmax = l;
            for (int c = 0; c < 3; c++) m->sEval[0][o + c] = f[c];
        }
        if (lmax > lte) lte = lmax;
    }
    if (s->primed) {
        s->last_lte = lte;
        if (!adaptive_dt(s, lte)) {
            for (int q = 0; q < s->nmesh; q++) memcpy(s->m[q].M, s->m[q].sM1, sizeof(double) * 3 * s->m[q].n);
            s->primed = 0;
            s->rejected++;
            return 0;
        }
    } else s->primed = 1;
    double dT = s->dT;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        for (size_t o = 0; o < 3 * (size_t)m->n; o++) {
            m->sM1[o] = m->M[o];
            m->M[o] += m->sEval[0][o] * (dT / 5);
        }
    }
    static const double a[6][6] = {
        {0},
        {3.0 / 40, 9.0 / 40},
        {44.0 / 45, -56.0 / 15, 32.0 / 9},
        {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729},
        {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656},
        {35.0 / 384, 0.0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
    for (int st = 1; st <= 5; st++) {
        update_all_fields(s);
        for (int q = 0; q < s->nmesh; q++) {
            orc_mesh *m = &s->m[q];
            const orc_mesh_desc *d = &m->d;
#pragma omp parallel for
            for (int i = 0; i < m->n; i++) {
                size_t o = 3 * (size_t)i;
                double f[3];
                llg(m->M + o, m->H + o, m->Ms[i], d->alpha, d->grel, f);
                for (int c = 0; c < 3; c++) {
                    m->sEval[st][o + c] = f[c];
                    double acc = 0.0;
                    for (int e = 0; e <= st; e++) acc += a[st][e] * m->sEval[e][o + c];
                    m->M[o + c] = m->sM1[o + c] + acc * dT;
                }
                if (st == 5) renorm(m->M + o, m->Ms[i]);
            }
        }
    }
    s->time += dT;
    s->stagetime += dT;
    s->accepted++;
    return 1;
}

int orc_run(orc_solver *s, int steps, orc_stats *st)
{
    long target = s->accepted + steps;
    long guard = 0;
    while (s->accepted < target) {
        if (s->eval == ORC_RK4) rk4_step(s);
        else rkdp_attempt(s);
        if (++guard > 100L * steps + 1000) return 1;
    }
    if (st) {
        st->accepted = s->accepted; st->rejected = s->rejected; st->evals = s->evals;
        st->time = s->time; st->dT = s->dT; st->last_lte = s->last_lte;
    }
    return 0;
}
