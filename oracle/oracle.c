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
 *   evaluation speedup (RK4)   Boris/DemagCUDA.cpp:106-470, Boris/DemagCUDA.cu:29-265,
 *                              Boris/DiffEq_CommonBase_Iterate.cpp:1536,1639
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

/* cell loops run in parallel only above this many cells (thread start-up dominates small meshes) */
#define ORC_PAR_MIN 32768

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

/* DemagTFunc::SelfDemag (Boris/DemagTFunc_Self.cpp:6) on the cellsize in metres, as the reference's
 * evaluation speedup calls it (Boris/DemagCUDA.cpp:39): its Newell f (Boris/DemagTFunc_fg.cpp:10) leaves
 * out the log and atan terms whose squared lengths / coordinate are not above the zero threshold
 * (BorisLib/Funcs_Aux_base.h:9,35, 1e-12 as a float) */
static int ref_nz(double v) { const double e = (double)1e-12f; return v > e || v < -e; }

static double f_thresholded(double x, double y, double z)
{
    double xsq = x * x, ysq = y * y, zsq = z * z;
    double Rxy = xsq + ysq, Rxz = xsq + zsq, R = sqrt(xsq + ysq + zsq);
    double t[4] = {(2.0 * xsq - ysq - zsq) * R / 6.0, 0, 0, 0};
    if (ref_nz(Rxz)) {
        double arg = 2.0 * y * (y + R) / Rxz;
        if (arg > -1.0) t[1] = y * (zsq - xsq) * log1p(arg) / 4.0;
    }
    if (ref_nz(Rxy)) {
        double arg = 2.0 * z * (z + R) / Rxy;
        if (arg > -1.0) t[2] = z * (ysq - xsq) * log1p(arg) / 4.0;
    }
    if (ref_nz(x)) t[3] = -x * y * z * atan(y * z / (x * R));
    return csum(t, 4);
}

void orc_selfdemag_metres(double hx, double hy, double hz, double *out3)
{
    const double h3[3][3] = {{hx, hy, hz}, {hy, hx, hz}, {hz, hy, hx}};
    static const double cw[3] = {-1.0, 2.0, -1.0};
    for (int c = 0; c < 3; c++) {
        double v[27];
        int m = 0;
        for (int i = -1; i <= 1; i++)
            for (int j = -1; j <= 1; j++)
                for (int k = -1; k <= 1; k++)
                    v[m++] = cw[i + 1] * cw[j + 1] * cw[k + 1] * f_thresholded(i * h3[c][0], j * h3[c][1], k * h3[c][2]);
        out3[c] = -csum(v, 27) / (4.0 * M_PI * h3[c][0] * h3[c][1] * h3[c][2]);
    }
}

/* DemagTFunc::SelfDemag_PBC (Boris/DemagTFunc_Self.cpp:57): the cell's own D plus, for each image
 * period other than (0,0,0), the far-field D at that period's offset (|img * n| cells per axis). As
 * the reference does, the xx, yy and zz image terms all take the expansion of the (hx, hy, hz)
 * cell in its xx form, yy evaluated at the offset (y, x, z) and zz at (z, y, x). Cellsizes are
 * normalised by the largest (the product's choice for the self term; the expansion is scale free). */
static void selfdemag_pbc_core(double hx, double hy, double hz, const int *n3, const int *pbc, double *out3, int metres)
{
    /* the reference's loops run i_img from -images to images: a negative count on any axis leaves
       them empty, so the coefficient is zero (self term included) */
    if (pbc && (pbc[0] < 0 || pbc[1] < 0 || pbc[2] < 0)) { out3[0] = out3[1] = out3[2] = 0.0; return; }
    if (metres) orc_selfdemag_metres(hx, hy, hz, out3);
    double hm = hx;
    if (hy > hm) hm = hy;
    if (hz > hm) hm = hz;
    hx /= hm; hy /= hm; hz /= hm;
    if (!metres) orc_selfdemag(hx, hy, hz, out3);
    if (!pbc) return;
    int X = pbc[0], Y = pbc[1], Z = pbc[2];
    for (int a = -X; a <= X; a++)
        for (int b = -Y; b <= Y; b++)
            for (int c = -Z; c <= Z; c++) {
                if (!a && !b && !c) continue;
                double x = fabs((double)a * n3[0]) * hx, y = fabs((double)b * n3[1]) * hy, z = fabs((double)c * n3[2]) * hz;
                double v[6];
                orc_asymptotic(hx, hy, hz, x, y, z, v);
                out3[0] += v[0];
                orc_asymptotic(hx, hy, hz, y, x, z, v);
                out3[1] += v[0];
                orc_asymptotic(hx, hy, hz, z, y, x, v);
                out3[2] += v[0];
            }
}

void orc_selfdemag_pbc(double hx, double hy, double hz, const int *n3, const int *pbc, double *out3)
{
    selfdemag_pbc_core(hx, hy, hz, n3, pbc, out3, 0);
}

void orc_selfdemag_pbc_metres(double hx, double hy, double hz, const int *n3, const int *pbc, double *out3)
{
    selfdemag_pbc_core(hx, hy, hz, n3, pbc, out3, 1);
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

/* ------------------------------------------------------------------ periodic boundary conditions */

static int isgn(int v) { return (v > 0) - (v < 0); }   /* get_sign, BorisLib/Funcs_Math.h:103 */

/* D = -N on the N grid with PBC images (DemagTFunc::CalcDiagTens2D_PBC / CalcOffDiagTens2D_PBC,
 * Boris/DemagTFunc_PBC.cpp:5,97, and the 3D forms :185,:300): along a periodic axis N = n and every
 * index i0 in [0, N) holds the sum over images m in [-X, X] of the free tensor at m N + i0 (off-diagonal
 * components with the signs of the offsets, sign(0) = 0); along a non-periodic axis i0 runs over
 * [0, N/2) and the mirrors (N - i0) mod N are filled by parity. A one-cell-thick mesh (nz == 1) sums
 * its z images at k = k_img and has no xz, yz. */
int orc_tensor_pbc(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz, const int *pbc,
                   double *diag, double *odiag)
{
    double hm = hx;
    if (hy > hm) hm = hy;
    if (hz > hm) hm = hz;
    hx /= hm; hy /= hm; hz /= hm;
    const int X = abs(pbc[0]), Y = abs(pbc[1]), Z = abs(pbc[2]);
    const int two_d = (nz == 1);
    size_t np = (size_t)Nx * Ny * Nz;
    memset(diag, 0, sizeof(double) * 3 * np);
    memset(odiag, 0, sizeof(double) * 3 * np);
    const int ei = X ? Nx : Nx / 2, ej = Y ? Ny : Ny / 2, ek = two_d ? 1 : (Z ? Nz : Nz / 2);
    const int per[3] = {X != 0, Y != 0, two_d || Z != 0};
    const int Ng[3] = {Nx, Ny, Nz};
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k0 = 0; k0 < ek; k0++)
        for (int j0 = 0; j0 < ej; j0++)
            for (int i0 = 0; i0 < ei; i0++) {
                double dv[3] = {0, 0, 0}, ov[3] = {0, 0, 0};
                for (int ii = -X; ii <= X; ii++)
                    for (int jj = -Y; jj <= Y; jj++)
                        for (int kk = -Z; kk <= Z; kk++) {
                            int i = ii * Nx + i0, j = jj * Ny + j0, k = two_d ? kk : kk * Nz + k0;
                            int si = isgn(i), sj = isgn(j), sk = isgn(k);
                            i = abs(i); j = abs(j); k = abs(k);
                            double x = i * hx, y = j * hy, z = k * hz;
                            double a[6];
                            if (use_asympt(i, j, k)) orc_asymptotic(hx, hy, hz, x, y, z, a);
                            else {
                                a[0] = -newell_L(orc_newell_f, x, y, z, hx, hy, hz);
                                a[1] = -newell_L(orc_newell_f, y, x, z, hy, hx, hz);
                                a[2] = -newell_L(orc_newell_f, z, y, x, hz, hy, hx);
                                a[3] = -newell_L(orc_newell_g, x, y, z, hx, hy, hz);
                                a[4] = two_d ? 0.0 : -newell_L(orc_newell_g, x, z, y, hx, hz, hy);
                                a[5] = two_d ? 0.0 : -newell_L(orc_newell_g, y, z, x, hy, hz, hx);
                            }
                            dv[0] += a[0]; dv[1] += a[1]; dv[2] += a[2];
                            ov[0] += a[3] * si * sj;
                            if (!two_d) { ov[1] += a[4] * si * sk; ov[2] += a[5] * sj * sk; }
                        }
                const int q[3] = {i0, j0, k0};
                /* the point and, along non-periodic axes with a non-zero index, its mirrors */
                for (int f = 0; f < 8; f++) {
                    int r[3], sg[3] = {1, 1, 1}, ok = 1;
                    for (int ax = 0; ax < 3; ax++) {
                        if (f & (1 << ax)) {
                            if (per[ax] || q[ax] == 0) { ok = 0; break; }
                            r[ax] = (Ng[ax] - q[ax]) % Ng[ax];
                            sg[ax] = -1;
                        } else r[ax] = q[ax];
                    }
                    if (!ok) continue;
                    size_t p = (size_t)r[0] + (size_t)r[1] * Nx + (size_t)r[2] * Nx * Ny;
                    diag[3 * p] = dv[0]; diag[3 * p + 1] = dv[1]; diag[3 * p + 2] = dv[2];
                    odiag[3 * p] = ov[0] * sg[0] * sg[1];
                    odiag[3 * p + 1] = ov[1] * sg[0] * sg[2];
                    odiag[3 * p + 2] = ov[2] * sg[1] * sg[2];
                }
            }
    return 0;
}

/* in-place complex DFT of c[Nx*Ny*Nz] along one axis */
static void dft_axis(double *c, int Nx, int Ny, int Nz, int ax, int sign)
{
    int dims[3] = {Nx, Ny, Nz};
    size_t strides[3] = {1, (size_t)Nx, (size_t)Nx * Ny};
    int L = dims[ax];
    if (L == 1) return;
    double *tw = bm_fft_table(L);
    size_t nlines = (size_t)Nx * Ny * Nz / L;
#pragma omp parallel if (nlines * (size_t)L > ORC_PAR_MIN)
    {
        double *line = (double *)malloc(sizeof(double) * 2 * L);
        double *scr = (double *)malloc(sizeof(double) * 4 * L);
#pragma omp for
        for (long li = 0; li < (long)nlines; li++) {
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

/* Octant spectra from a tensor on the N grid the way DemagKernel builds them
 * (Boris/DemagKernel.cpp:171-300 2D, :317-470 3D): a real forward DFT along x, y, z in turn, after
 * each of which only the real part (even along that axis) or the imaginary part (odd along it) is
 * kept as the next input: xx, yy, zz Re Re Re; xy Im Im, then -Re along z; xz Im, Re, -Im; yz Re, Im,
 * -Im (2D: xy Im along x, -Im along y). Same layout as orc_kernels. */
int orc_kernels_from_tensor(const double *dg, const double *od, int nz, int Nx, int Ny, int Nz, double *kdiag,
                            double *kodiag)
{
    size_t np = (size_t)Nx * Ny * Nz;
    double *c = (double *)malloc(sizeof(double) * 2 * np);
    int Kx = Nx / 2 + 1, Ky = Ny / 2 + 1, Kz = Nz / 2 + 1;
    /* part kept after each axis: 0 Re, 1 Im; final sign */
    static const int keep[6][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    for (int comp = 0; comp < 6; comp++) {
        const double *src = comp < 3 ? dg : od;
        int cc = comp % 3;
        double *dst = comp < 3 ? kdiag : kodiag;
        if (nz == 1 && comp >= 4) {
            for (size_t q = 0; q < (size_t)Kx * Ky * Kz; q++) dst[3 * q + cc] = 0.0;
            continue;
        }
        for (size_t p = 0; p < np; p++) { c[2 * p] = src[3 * p + cc]; c[2 * p + 1] = 0.0; }
        int dims[3] = {Nx, Ny, Nz};
        int last = (Nz > 1) ? 2 : 1;
        double sgn = comp < 3 ? 1.0 : -1.0;
        for (int ax = 0; ax <= last; ax++) {
            if (dims[ax] > 1) dft_axis(c, Nx, Ny, Nz, ax, -1);
            int part = keep[comp][ax];
            for (size_t p = 0; p < np; p++) { c[2 * p] = c[2 * p + part]; c[2 * p + 1] = 0.0; }
        }
        for (int k = 0; k < Kz; k++)
            for (int j = 0; j < Ky; j++)
                for (int i = 0; i < Kx; i++) {
                    size_t p = (size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny;
                    size_t q = (size_t)i + (size_t)j * Kx + (size_t)k * Kx * Ky;
                    dst[3 * q + cc] = sgn * c[2 * p];
                }
    }
    free(c);
    return 0;
}

/* FFT sizes of ConvolutionData::SetConvolutionDimensions (Boris/ConvolutionData.cpp:115-145):
 * n along a periodic axis, 2n otherwise, 1 along z for a one-cell-thick mesh */
void orc_pbc_dims(int nx, int ny, int nz, const int *pbc, int *N3)
{
    N3[0] = (pbc && pbc[0]) ? nx : 2 * nx;
    N3[1] = (pbc && pbc[1]) ? ny : 2 * ny;
    N3[2] = nz > 1 ? ((pbc && pbc[2]) ? nz : 2 * nz) : 1;
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

/* demag with PBC images per axis (pbc NULL or all zero: the plain convolution with N = 2n) */
orc_demag *orc_demag_create_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc)
{
    int N3[3];
    orc_pbc_dims(nx, ny, nz, pbc, N3);
    if (!pbc || !(pbc[0] || pbc[1] || pbc[2])) return orc_demag_create(nx, ny, nz, hx, hy, hz, N3[0], N3[1], N3[2]);
    orc_demag *d = (orc_demag *)calloc(1, sizeof(orc_demag));
    d->nx = nx; d->ny = ny; d->nz = nz; d->Nx = N3[0]; d->Ny = N3[1]; d->Nz = N3[2];
    size_t np = (size_t)N3[0] * N3[1] * N3[2];
    size_t nk = (size_t)(N3[0] / 2 + 1) * (N3[1] / 2 + 1) * (N3[2] / 2 + 1);
    d->kd = (double *)malloc(sizeof(double) * 3 * nk);
    d->ko = (double *)malloc(sizeof(double) * 3 * nk);
    double *dg = (double *)malloc(sizeof(double) * 3 * np), *od = (double *)malloc(sizeof(double) * 3 * np);
    orc_tensor_pbc(nx, ny, nz, N3[0], N3[1], N3[2], hx, hy, hz, pbc, dg, od);
    orc_kernels_from_tensor(dg, od, nz, N3[0], N3[1], N3[2], d->kd, d->ko);
    free(dg); free(od);
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

/* ------------------------------------------------------------------ multilayered convolution */

/* Geometry of the multilayered convolution (SDemag multilayer mode):
 *   n_common        SDemag::set_default_n_common (Boris/SDemag.cpp:173), Set_n_common (:362),
 *                   Set_2D_Multilayered_Convolution (:341)
 *   layer rects     SDemag::set_Rect_collection (Boris/SDemag.cpp:215), Rect::get_zlayer
 *                   (BorisLib/Types_Rect.h:485) in 2D-layered mode
 *   h_max           SDemag::get_maximum_cellsize (Boris/SDemag.cpp:297): the meshes' own cellsizes
 *   transfer        SDemag_Demag::Initialize (Boris/SDemag_Demag.cpp:349-361) and the weighted
 *                   mesh transfer of BorisLib/VEC_MeshTransfer.h (:306 build_meshcells_weights,
 *                   :396 build_supermeshcells_weights, :901 initialize_transfer_in_weighted,
 *                   :1221 initialize_transfer_out)
 *   kernels         DemagKernelCollection::Calculate_Demag_Kernels and KernelAlreadyComputed
 *                   (Boris/DemagKernelCollection_Calc.cpp:9,114); tensors from
 *                   DemagTFunc_Shifted.cpp (3D and regular 2D) and DemagTFunc_Irregular.cpp
 *                   (2D with source and destination thickness differing), including the
 *                   thickness roles and far-field scaling those functions use
 *   evaluation      SDemag::UpdateField multilayer branch (Boris/SDemag.cpp:786-900)
 * Spectra here are plain full complex 3D DFTs of the real-space tensors (no symmetry storage). */

#define ML_EPS 1e-12          /* BorisLib/Funcs_Aux_base.h:9 EPSILON_POSITIVE */
#define ML_EPS_ROUND 1e-4     /* BorisLib/Funcs_Aux_base.h:13 EPSILON_ROUNDING */

typedef struct { double x, y, z; } d3;
typedef struct { d3 s, e; } rect3;

static int isz(double v) { return v < ML_EPS && v > -ML_EPS; }
static int iszop(double v) { return v > 0 || isz(v); }
static int d3eq(d3 a, d3 b) { return isz(a.x - b.x) && isz(a.y - b.y) && isz(a.z - b.z); }
static d3 d3m(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static d3 d3sub(d3 a, d3 b) { return d3m(a.x - b.x, a.y - b.y, a.z - b.z); }
static d3 d3add(d3 a, d3 b) { return d3m(a.x + b.x, a.y + b.y, a.z + b.z); }
static double d3norm(d3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static d3 rsize(rect3 r) { return d3sub(r.e, r.s); }
static int recteq(rect3 a, rect3 b) { return d3eq(a.s, b.s) && d3eq(a.e, b.e); }
static double floor_eps(double v) { return floor(v + ML_EPS_ROUND); }
static double ceil_eps(double v) { return ceil(v - ML_EPS_ROUND); }

/* Rect::get_intersection and intersects (BorisLib/Types_Rect.h:494,361) */
static int rect_intersection(rect3 a, rect3 b, rect3 *out)
{
    d3 st = d3m(b.s.x > a.s.x ? b.s.x : a.s.x, b.s.y > a.s.y ? b.s.y : a.s.y, b.s.z > a.s.z ? b.s.z : a.s.z);
    d3 en = d3m(b.e.x < a.e.x ? b.e.x : a.e.x, b.e.y < a.e.y ? b.e.y : a.e.y, b.e.z < a.e.z ? b.e.z : a.e.z);
    rect3 r = {{0, 0, 0}, {0, 0, 0}};
    if (iszop(en.x - st.x) && iszop(en.y - st.y) && iszop(en.z - st.z)) { r.s = st; r.e = en; }
    *out = r;
    /* intersects: the intersection differs from the null rect */
    return !(isz(r.s.x) && isz(r.s.y) && isz(r.s.z) && isz(r.e.x) && isz(r.e.y) && isz(r.e.z));
}
static int rect_isplane(rect3 r)
{
    double dx = r.s.x - r.e.x, dy = r.s.y - r.e.y, dz = r.s.z - r.e.z;
    return (isz(dx) && !isz(dy) && !isz(dz)) || (isz(dy) && !isz(dx) && !isz(dz)) || (isz(dz) && !isz(dx) && !isz(dy));
}
static int rect_ispoint(rect3 r) { return d3eq(r.s, r.e); }

typedef struct { int n; int *idx; double *w; } wlist;   /* one cell's contributions */

static void wl_push(wlist *l, int idx, double w)
{
    l->idx = (int *)realloc(l->idx, sizeof(int) * (l->n + 1));
    l->w = (double *)realloc(l->w, sizeof(double) * (l->n + 1));
    l->idx[l->n] = idx; l->w[l->n] = w; l->n++;
}

/* cells of grid (n, h, origin rs) within the index box of rect rc, with reciprocal-distance weights */
static double recip_weights(wlist *l, rect3 rc, const int n[3], d3 h, d3 rs)
{
    d3 coord = d3sub(d3m((rc.e.x + rc.s.x) / 2, (rc.e.y + rc.s.y) / 2, (rc.e.z + rc.s.z) / 2), rs);
    d3 pll = d3sub(rc.s, rs), pur = d3sub(rc.e, rs);
    int ll[3] = {(int)floor_eps(pll.x / h.x), (int)floor_eps(pll.y / h.y), (int)floor_eps(pll.z / h.z)};
    int ur[3] = {(int)ceil_eps(pur.x / h.x), (int)ceil_eps(pur.y / h.y), (int)ceil_eps(pur.z / h.z)};
    d3 sz = rsize(rc);
    double dmax = d3norm(d3m(sz.x / 2 + h.x / 2, sz.y / 2 + h.y / 2, sz.z / 2 + h.z / 2));
    double tot = 0.0;
    for (int ii = ll[0] >= 0 ? ll[0] : 0; ii < (ur[0] < n[0] ? ur[0] : n[0]); ii++)
        for (int jj = ll[1] >= 0 ? ll[1] : 0; jj < (ur[1] < n[1] ? ur[1] : n[1]); jj++)
            for (int kk = ll[2] >= 0 ? ll[2] : 0; kk < (ur[2] < n[2] ? ur[2] : n[2]); kk++) {
                d3 cc = d3m((ii + 0.5) * h.x, (jj + 0.5) * h.y, (kk + 0.5) * h.z);
                double dr = dmax - d3norm(d3sub(cc, coord));
                tot += dr;
                wl_push(l, ii + jj * n[0] + kk * n[0] * n[1], dr);
            }
    return tot;
}

typedef struct {
    int type;       /* 0 regular (same cellsize), 1 irregular 2D (source / destination thickness differ) */
    d3 hs, hd, shift;   /* normalised by h_max */
    double *F;      /* 6 full complex spectra, component-major, each Nx*Ny*Nz complex */
} ml_kernel;

typedef struct {
    int mesh, transfer;
    rect3 rect;
    d3 hc;                      /* convolution cellsize (rect / n_common) */
    wlist *tin;                 /* per common cell */
    wlist *tout;                /* per mesh cell */
    int *kidx, *kinv;           /* per source: kernel index, inverse z-shift flag */
    int *kkind;                 /* per source: 1 self, 2 z-shifted, 3 inverse z-shifted, 4 full */
} ml_layer;

struct orc_ml {
    int nmesh, L;
    int (*mn)[3];
    d3 *mh;
    rect3 *mrect;
    size_t *moff;               /* first cell of each mesh in the concatenated arrays */
    int nc[3], N[3], force2d;
    double h_max;
    ml_layer *lay;
    ml_kernel *ker;
    int nker;
    /* evaluation speedup (SDemagCUDA::UpdateField, Boris/SDemagCUDA.cpp:587-930): per slot, every
       layer's common-grid field minus its self term [slot][layer][3 ncell], and the layers' self
       coefficients SelfDemag_PBC(h_common, n_common) (Boris/SDemag_Demag.cpp:328) */
    double *es_H[6];
    double *es_self;
    int es_metres;   /* self coefficients on the cellsize in metres (the reference's computation) */
};

/* one tensor point D = -N (xx,yy,zz,xy,xz,yz) at grid offset (i,j,k) for a kernel */
static void ml_tensor_point(const ml_kernel *K, int i, int j, int k, int two_d, double out[6])
{
    const d3 h = (K->type == 1) ? K->hd : K->hs;
    const d3 sh = K->shift;
    double is = fabs(i + sh.x / h.x), js = fabs(j + sh.y / h.y), ks = fabs(k + sh.z / h.z);
    int far = ((int)floor_eps(is) >= ASYMPT_DIST || (int)floor_eps(js) >= ASYMPT_DIST || (int)floor_eps(ks) >= ASYMPT_DIST ||
               (int)floor_eps(is * is + js * js + ks * ks) >= ASYMPT_DIST * ASYMPT_DIST);
    double x = i * h.x + sh.x, y = j * h.y + sh.y, z = k * h.z + sh.z;
    if (far) {
        orc_asymptotic(h.x, h.y, h.z, x, y, z, out);
        /* irregular: the reference scales the destination-cell expansion by the source thickness
         * (DemagTFunc_Irregular.cpp:52-56) */
        if (K->type == 1) for (int c = 0; c < 6; c++) out[c] *= K->hs.z;
    } else if (K->type == 0) {
        out[0] = -newell_L(orc_newell_f, x, y, z, h.x, h.y, h.z);
        out[1] = -newell_L(orc_newell_f, y, x, z, h.y, h.x, h.z);
        out[2] = -newell_L(orc_newell_f, z, y, x, h.z, h.y, h.x);
        out[3] = -newell_L(orc_newell_g, x, y, z, h.x, h.y, h.z);
        out[4] = -newell_L(orc_newell_g, x, z, y, h.x, h.z, h.y);
        out[5] = -newell_L(orc_newell_g, y, z, x, h.y, h.z, h.x);
    } else {
        /* 36-point sums: (-1,2,-1) along the two in-plane axes, four z points along the axis
         * carrying the shift. xx, yy use z in {D-s, D, D+d, D+d-s}; zz, xy, xz, yz use
         * z in {D-d, D, D+s, D+s-d} (D the shift, s / d the source / destination thickness),
         * as fill_f_vals_zshifted_irregular / fill_g_vals_zshifted_irregular
         * (DemagTFunc_fg.cpp:507,560) and DemagTFunc_L.cpp:377-814 combine them. */
        const double s = K->hs.z, d = K->hd.z;
        const double zA[4] = {z - s, z, z + d, z + d - s}, zB[4] = {z - d, z, z + s, z + s - d};
        const double wz[4] = {-1.0, 1.0, -1.0, 1.0};
        const double cw[3] = {-1.0, 2.0, -1.0};
        const double tau = h.x * h.y * h.z;
        for (int c = 0; c < 6; c++) {
            double v[36];
            int m = 0;
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++)
                    for (int q = 0; q < 4; q++) {
                        double w = cw[a + 1] * cw[b + 1] * wz[q], val;
                        switch (c) {
                        case 0: val = orc_newell_f(x + a * h.x, y + b * h.y, zA[q]); break;
                        case 1: val = orc_newell_f(y + a * h.y, x + b * h.x, zA[q]); break;
                        case 2: val = orc_newell_f(zB[q], y + a * h.y, x + b * h.x); break;
                        case 3: val = orc_newell_g(x + a * h.x, y + b * h.y, zB[q]); break;
                        case 4: val = orc_newell_g(x + a * h.x, zB[q], y + b * h.y); break;
                        default: val = orc_newell_g(y + a * h.y, zB[q], x + b * h.x); break;
                        }
                        v[m++] = w * val;
                    }
            out[c] = -csum(v, 36) / (4.0 * M_PI * tau);
        }
    }
    /* 2D self kernel: only Dxy is computed off the diagonal (CalcOffDiagTens2D) */
    if (two_d && sh.x == 0.0 && sh.y == 0.0 && sh.z == 0.0) { out[4] = 0.0; out[5] = 0.0; }
}

static void ml_build_kernel(const struct orc_ml *s, ml_kernel *K)
{
    const int Nx = s->N[0], Ny = s->N[1], Nz = s->N[2];
    const int nx = s->nc[0], ny = s->nc[1], nz = s->nc[2];
    const int two_d = (nz == 1);
    size_t np = (size_t)Nx * Ny * Nz;
    K->F = (double *)calloc(6 * 2 * np, sizeof(double));
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int k = -nz + 1; k < nz; k++)
        for (int j = -ny + 1; j < ny; j++)
            for (int i = -nx + 1; i < nx; i++) {
                double v[6];
                ml_tensor_point(K, i, j, k, two_d, v);
                size_t p = (size_t)((i + Nx) % Nx) + (size_t)((j + Ny) % Ny) * Nx + (size_t)((k + Nz) % Nz) * Nx * Ny;
                for (int c = 0; c < 6; c++) K->F[2 * (c * np + p)] = v[c];
            }
    for (int c = 0; c < 6; c++) dft3(K->F + 2 * c * np, Nx, Ny, Nz, -1);
}

void orc_ml_destroy(orc_ml *s)
{
    if (!s) return;
    for (int l = 0; l < s->L; l++) {
        ml_layer *y = &s->lay[l];
        if (y->tin) {
            size_t ncell = (size_t)s->nc[0] * s->nc[1] * s->nc[2];
            for (size_t i = 0; i < ncell; i++) { free(y->tin[i].idx); free(y->tin[i].w); }
            free(y->tin);
        }
        if (y->tout) {
            int m = y->mesh;
            size_t n = (size_t)s->mn[m][0] * s->mn[m][1] * s->mn[m][2];
            for (size_t i = 0; i < n; i++) { free(y->tout[i].idx); free(y->tout[i].w); }
            free(y->tout);
        }
        free(y->kidx); free(y->kinv); free(y->kkind);
    }
    for (int q = 0; q < s->nker; q++) free(s->ker[q].F);
    for (int k = 0; k < 6; k++) free(s->es_H[k]);
    free(s->es_self);
    free(s->ker); free(s->lay); free(s->mn); free(s->mh); free(s->mrect); free(s->moff);
    free(s);
}

orc_ml *orc_ml_create(int nmesh, const int *n3, const double *h3, const double *o3, int mode, const int *ncommon)
{
    orc_ml *s = (orc_ml *)calloc(1, sizeof(orc_ml));
    s->nmesh = nmesh;
    s->mn = calloc(nmesh, sizeof(*s->mn));
    s->mh = (d3 *)calloc(nmesh, sizeof(d3));
    s->mrect = (rect3 *)calloc(nmesh, sizeof(rect3));
    s->moff = (size_t *)calloc(nmesh + 1, sizeof(size_t));
    for (int m = 0; m < nmesh; m++) {
        for (int a = 0; a < 3; a++) s->mn[m][a] = n3[3 * m + a];
        s->mh[m] = d3m(h3[3 * m], h3[3 * m + 1], h3[3 * m + 2]);
        s->mrect[m].s = d3m(o3[3 * m], o3[3 * m + 1], o3[3 * m + 2]);
        s->mrect[m].e = d3add(s->mrect[m].s, d3m(s->mh[m].x * s->mn[m][0], s->mh[m].y * s->mn[m][1], s->mh[m].z * s->mn[m][2]));
        s->moff[m + 1] = s->moff[m] + (size_t)s->mn[m][0] * s->mn[m][1] * s->mn[m][2];
    }
    /* n_common and the 2D mode */
    int force2d = mode;
    if (ncommon) {
        for (int a = 0; a < 3; a++) s->nc[a] = ncommon[a];
        if (force2d == 0 && s->nc[2] == 1) force2d = 1;
    } else {
        int all2d = 1;
        s->nc[0] = s->nc[1] = s->nc[2] = 1;
        for (int m = 0; m < nmesh; m++) {
            if (s->mn[m][2] != 1) all2d = 0;
            for (int a = 0; a < 3; a++) if (s->nc[a] < s->mn[m][a]) s->nc[a] = s->mn[m][a];
        }
        if (all2d) s->nc[2] = 1;
    }
    if (force2d) s->nc[2] = 1;
    s->force2d = force2d;
    for (int a = 0; a < 3; a++) s->N[a] = s->nc[a] > 1 ? 2 * s->nc[a] : 1;
    /* layers and the raw rect collection */
    int L = 0;
    for (int m = 0; m < nmesh; m++) L += (force2d == 2) ? s->mn[m][2] : 1;
    s->L = L;
    s->lay = (ml_layer *)calloc(L, sizeof(ml_layer));
    int li = 0;
    for (int m = 0; m < nmesh; m++) {
        int nl = (force2d == 2) ? s->mn[m][2] : 1;
        for (int q = 0; q < nl; q++, li++) {
            rect3 r = s->mrect[m];
            if (force2d == 2) {
                double t = s->mh[m].z;
                /* Rect::get_zlayer */
                if (!(q * t < 0 || (q + 1) * t > (r.e.z - r.s.z))) { r.s.z = s->mrect[m].s.z + q * t; r.e.z = s->mrect[m].s.z + (q + 1) * t; }
            }
            s->lay[li].mesh = m;
            s->lay[li].rect = r;
        }
    }
    /* enlarge to common sizes */
    d3 mx = d3m(0, 0, 0);
    double minx = s->lay[0].rect.s.x, miny = s->lay[0].rect.s.y, minz = s->lay[0].rect.s.z;
    for (int l = 0; l < L; l++) {
        d3 sz = rsize(s->lay[l].rect);
        if (mx.x < sz.x) mx.x = sz.x;
        if (mx.y < sz.y) mx.y = sz.y;
        if (mx.z < sz.z) mx.z = sz.z;
        if (s->lay[l].rect.s.x < minx) minx = s->lay[l].rect.s.x;
        if (s->lay[l].rect.s.y < miny) miny = s->lay[l].rect.s.y;
        if (s->lay[l].rect.s.z < minz) minz = s->lay[l].rect.s.z;
    }
    for (int l = 0; l < L; l++) {
        rect3 *r = &s->lay[l].rect;
        if (r->e.x - mx.x < minx) { r->s.x = minx; r->e.x = r->s.x + mx.x; } else r->s.x = r->e.x - mx.x;
        if (r->e.y - mx.y < miny) { r->s.y = miny; r->e.y = r->s.y + mx.y; } else r->s.y = r->e.y - mx.y;
        if (s->nc[2] != 1) {
            if (r->e.z - mx.z < minz) { r->s.z = minz; r->e.z = r->s.z + mx.z; } else r->s.z = r->e.z - mx.z;
        }
    }
    s->h_max = 0.0;
    for (int l = 0; l < L; l++) {
        d3 h = s->mh[s->lay[l].mesh];
        double hm = h.x > h.y ? h.x : h.y;
        if (h.z > hm) hm = h.z;
        if (s->h_max < hm) s->h_max = hm;
    }
    for (int l = 0; l < L; l++) {
        ml_layer *y = &s->lay[l];
        d3 sz = rsize(y->rect);
        y->hc = d3m(sz.x / s->nc[0], sz.y / s->nc[1], sz.z / s->nc[2]);
    }
    /* kernels: dedup by (shift, h_src, h_dst); in 2D a kernel computed for the opposite z shift
     * is reused with the xz, yz signs flipped */
    s->ker = (ml_kernel *)calloc(L * L, sizeof(ml_kernel));
    typedef struct { d3 shift, hs, hd; int computed; } kdesc;
    kdesc *kd = (kdesc *)calloc(L * L, sizeof(kdesc));
    int *slot = (int *)malloc(sizeof(int) * L * L);   /* per (dest, src): index into s->ker or -1 */
    for (int i = 0; i < L * L; i++) slot[i] = -1;
    for (int l = 0; l < L; l++) {
        ml_layer *y = &s->lay[l];
        y->kidx = (int *)calloc(L, sizeof(int));
        y->kinv = (int *)calloc(L, sizeof(int));
        y->kkind = (int *)calloc(L, sizeof(int));
    }
    for (int d = 0; d < L; d++) {
        ml_layer *y = &s->lay[d];
        for (int q = 0; q < L; q++) {
            d3 shift = d3sub(y->rect.s, s->lay[q].rect.s);
            d3 hsrc = s->lay[q].hc, hdst = y->hc;
            int found = -1, inv = 0;
            /* search every collection in order, each over its kernels in order */
            for (int c2 = 0; c2 < L && found < 0; c2++)
                for (int k2 = 0; k2 < L && found < 0; k2++) {
                    int kk = slot[c2 * L + k2];
                    if (kk < 0 || !kd[kk].computed) continue;
                    if (!(d3eq(kd[kk].hs, hsrc) && d3eq(kd[kk].hd, hdst))) continue;
                    if (d3eq(kd[kk].shift, shift)) found = kk;
                    else if (s->N[2] == 1 && isz(shift.x) && isz(shift.y) && isz(kd[kk].shift.x) && isz(kd[kk].shift.y) &&
                             isz(shift.z + kd[kk].shift.z)) found = kk;
                }
            int self = recteq(s->lay[q].rect, y->rect);
            if (found >= 0) {
                if (isz(shift.x) && isz(shift.y) && !isz(shift.z) && isz(shift.z + kd[found].shift.z)) inv = 1;
                slot[d * L + q] = found;
            } else {
                int kk = s->nker++;
                ml_kernel *K = &s->ker[kk];
                if (self) {
                    kd[kk].shift = d3m(0, 0, 0); kd[kk].hs = hdst; kd[kk].hd = hdst;
                    K->type = 0;
                    K->hs = K->hd = d3m(hdst.x / s->h_max, hdst.y / s->h_max, hdst.z / s->h_max);
                    K->shift = d3m(0, 0, 0);
                } else {
                    kd[kk].shift = shift; kd[kk].hs = hsrc; kd[kk].hd = hdst;
                    K->shift = d3m(shift.x / s->h_max, shift.y / s->h_max, shift.z / s->h_max);
                    if (s->nc[2] == 1) {
                        /* 2D: irregular unless s * 1e-9 == d * 1e-9 (DemagTFunc_Irregular.cpp:12) */
                        d3 a = d3m(hsrc.x / s->h_max, hsrc.y / s->h_max, hsrc.z / s->h_max);
                        d3 b = d3m(hdst.x / s->h_max, hdst.y / s->h_max, hdst.z / s->h_max);
                        K->hs = a; K->hd = b;
                        K->type = d3eq(d3m(a.x * 1e-9, a.y * 1e-9, a.z * 1e-9), d3m(b.x * 1e-9, b.y * 1e-9, b.z * 1e-9)) ? 0 : 1;
                    } else {
                        /* 3D uses the destination cellsize for both (DemagKernelCollection_Calc.cpp:921) */
                        K->type = 0;
                        K->hs = K->hd = d3m(hdst.x / s->h_max, hdst.y / s->h_max, hdst.z / s->h_max);
                    }
                }
                kd[kk].computed = 1;
                slot[d * L + q] = kk;
                found = kk;
            }
            y->kidx[q] = found;
            y->kinv[q] = inv;
            if (self) y->kkind[q] = 1;
            else if (isz(kd[found].shift.x) && isz(kd[found].shift.y) && !isz(kd[found].shift.z)) y->kkind[q] = inv ? 3 : 2;
            else y->kkind[q] = recteq(s->lay[q].rect, y->rect) ? 1 : 4;
        }
    }
    free(kd); free(slot);
    for (int k = 0; k < s->nker; k++) ml_build_kernel(s, &s->ker[k]);
    /* transfers */
    size_t ncell = (size_t)s->nc[0] * s->nc[1] * s->nc[2];
    for (int l = 0; l < L; l++) {
        ml_layer *y = &s->lay[l];
        int m = y->mesh;
        y->transfer = !(recteq(y->rect, s->mrect[m]) && d3eq(y->hc, s->mh[m]));
        if (!y->transfer) continue;
        y->tin = (wlist *)calloc(ncell, sizeof(wlist));
        for (size_t c = 0; c < ncell; c++) {
            int ii = (int)(c % s->nc[0]), jj = (int)((c / s->nc[0]) % s->nc[1]), kk = (int)(c / ((size_t)s->nc[0] * s->nc[1]));
            rect3 rc;
            rc.s = d3add(y->rect.s, d3m(y->hc.x * ii, y->hc.y * jj, y->hc.z * kk));
            rc.e = d3add(rc.s, y->hc);
            rect3 ri;
            double tot = 0.0, cov = 0.0;
            if (rect_intersection(s->mrect[m], rc, &ri) && !rect_isplane(ri) && !rect_ispoint(ri)) {
                d3 si = rsize(ri), sc = rsize(rc);
                cov += (si.x / sc.x) * (si.y / sc.y) * (si.z / sc.z);
                tot += recip_weights(&y->tin[c], rc, s->mn[m], s->mh[m], s->mrect[m].s);
            }
            if (tot > 0) for (int q = 0; q < y->tin[c].n; q++) y->tin[c].w[q] *= cov / tot;
        }
        size_t n = (size_t)s->mn[m][0] * s->mn[m][1] * s->mn[m][2];
        y->tout = (wlist *)calloc(n, sizeof(wlist));
        for (size_t c = 0; c < n; c++) {
            int ii = (int)(c % s->mn[m][0]), jj = (int)((c / s->mn[m][0]) % s->mn[m][1]);
            int kk = (int)(c / ((size_t)s->mn[m][0] * s->mn[m][1]));
            rect3 rc;
            rc.s = d3add(s->mrect[m].s, d3m(s->mh[m].x * ii, s->mh[m].y * jj, s->mh[m].z * kk));
            rc.e = d3add(rc.s, s->mh[m]);
            double tot = recip_weights(&y->tout[c], rc, s->nc, y->hc, y->rect.s);
            if (tot > 0) for (int q = 0; q < y->tout[c].n; q++) y->tout[c].w[q] *= 1.0 / tot;
        }
    }
    return s;
}

int orc_ml_info(orc_ml *s, int *L, int *nc3, int *layer_mesh, int *do_transfer, double *rects6, int *kinds)
{
    if (L) *L = s->L;
    if (nc3) for (int a = 0; a < 3; a++) nc3[a] = s->nc[a];
    for (int l = 0; l < s->L; l++) {
        ml_layer *y = &s->lay[l];
        if (layer_mesh) layer_mesh[l] = y->mesh;
        if (do_transfer) do_transfer[l] = y->transfer;
        if (rects6) {
            rects6[6 * l] = y->rect.s.x; rects6[6 * l + 1] = y->rect.s.y; rects6[6 * l + 2] = y->rect.s.z;
            rects6[6 * l + 3] = y->rect.e.x; rects6[6 * l + 4] = y->rect.e.y; rects6[6 * l + 5] = y->rect.e.z;
        }
        if (kinds) for (int q = 0; q < s->L; q++) kinds[l * s->L + q] = y->kkind[q];
    }
    return 0;
}

/* the field of destination layer d on the common grid (tmp) into every mesh of that layer */
static void ml_transfer_out(orc_ml *s, int d, const double *tmp, double *H)
{
    ml_layer *y = &s->lay[d];
    double *Hm = H + 3 * s->moff[y->mesh];
    size_t n = s->moff[y->mesh + 1] - s->moff[y->mesh];
    if (y->transfer) {
        for (size_t c = 0; c < n; c++)
            for (int q = 0; q < y->tout[c].n; q++)
                for (int a = 0; a < 3; a++) Hm[3 * c + a] += tmp[3 * (size_t)y->tout[c].idx[q] + a] * y->tout[c].w[q];
    } else {
        for (size_t c = 0; c < 3 * n; c++) Hm[c] += tmp[c];
    }
}

/* Evaluation with the speedup (es_mode 0 plain, 1 compute and save into es_slot, 2 extrapolate with
 * the weights es_a of K saved fields), per layer on its common grid as SDemagCUDA::UpdateField does
 * (Boris/SDemagCUDA.cpp:587-930): a save keeps H - S Mc (SDemag_EvalSpeedup_SubSelf /
 * AddField_SubSelf), an extrapolation sets sum_k a_k (H_k - S Mc_k) + S Mc before the transfer out
 * (SDemag_EvalSpeedup_SetExtrapField_AddSelf / AddExtrapField_AddSelf); Mc is the layer's input on
 * the common grid (the mesh's M when the layer needs no transfer). */
int orc_ml_eval_es(orc_ml *s, const double *M, double *H, int es_mode, int es_slot, const double *es_a, int K)
{
    const int Nx = s->N[0], Ny = s->N[1], Nz = s->N[2];
    const int nx = s->nc[0], ny = s->nc[1], nz = s->nc[2];
    const size_t np = (size_t)Nx * Ny * Nz, ncell = (size_t)nx * ny * nz;
    const int L = s->L;
    double **F = (double **)calloc(L, sizeof(double *));
    double *tmp = (double *)malloc(sizeof(double) * 3 * ncell);
    double *Mcs = es_mode ? (double *)malloc(sizeof(double) * 3 * ncell * L) : NULL;
    if (es_mode && !s->es_self) {
        s->es_self = (double *)malloc(sizeof(double) * 3 * L);
        for (int l = 0; l < L; l++)
            selfdemag_pbc_core(s->lay[l].hc.x, s->lay[l].hc.y, s->lay[l].hc.z, s->nc, NULL, s->es_self + 3 * l,
                               s->es_metres);
    }
    if (es_mode == 1 && !s->es_H[es_slot]) s->es_H[es_slot] = (double *)calloc(3 * ncell * L, sizeof(double));
    memset(H, 0, sizeof(double) * 3 * s->moff[s->nmesh]);
    for (int l = 0; l < L; l++) {
        ml_layer *y = &s->lay[l];
        const double *Mm = M + 3 * s->moff[y->mesh];
        if (y->transfer) {
            for (size_t c = 0; c < ncell; c++) {
                double v[3] = {0, 0, 0};
                for (int q = 0; q < y->tin[c].n; q++)
                    for (int a = 0; a < 3; a++) v[a] += Mm[3 * (size_t)y->tin[c].idx[q] + a] * y->tin[c].w[q];
                for (int a = 0; a < 3; a++) tmp[3 * c + a] = v[a];
            }
        } else memcpy(tmp, Mm, sizeof(double) * 3 * ncell);
        if (Mcs) memcpy(Mcs + 3 * ncell * l, tmp, sizeof(double) * 3 * ncell);
        if (es_mode == 2) continue;
        F[l] = (double *)calloc(3 * 2 * np, sizeof(double));
        for (int a = 0; a < 3; a++) {
            double *Fa = F[l] + 2 * a * np;
            for (int k = 0; k < nz; k++)
                for (int j = 0; j < ny; j++)
                    for (int i = 0; i < nx; i++)
                        Fa[2 * ((size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny)] = tmp[3 * ((size_t)i + (size_t)j * nx + (size_t)k * nx * ny) + a];
            dft3(Fa, Nx, Ny, Nz, -1);
        }
    }
    if (es_mode == 2) {
        for (int d = 0; d < L; d++) {
            const double *Mc = Mcs + 3 * ncell * d, *S = s->es_self + 3 * d;
            for (size_t i = 0; i < 3 * ncell; i++) {
                double v = S[i % 3] * Mc[i];
                for (int k = 0; k < K; k++) v += es_a[k] * s->es_H[k][3 * ncell * d + i];
                tmp[i] = v;
            }
            ml_transfer_out(s, d, tmp, H);
        }
        free(F); free(tmp); free(Mcs);
        return 0;
    }
    double *O = (double *)malloc(sizeof(double) * 3 * 2 * np);
    static const int cmap[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    for (int d = 0; d < L; d++) {
        ml_layer *y = &s->lay[d];
        memset(O, 0, sizeof(double) * 3 * 2 * np);
        for (int q = 0; q < L; q++) {
            const ml_kernel *K = &s->ker[y->kidx[q]];
            const int inv = y->kinv[q];
#pragma omp parallel for if ((np) > ORC_PAR_MIN)
            for (long p = 0; p < (long)np; p++) {
                for (int a = 0; a < 3; a++) {
                    double re = 0.0, im = 0.0;
                    for (int b = 0; b < 3; b++) {
                        int c = cmap[a][b];
                        double sg = (inv && (c == 4 || c == 5)) ? -1.0 : 1.0;
                        double kr = sg * K->F[2 * (c * np + p)], ki = sg * K->F[2 * (c * np + p) + 1];
                        double mr = F[q][2 * (b * np + p)], mi = F[q][2 * (b * np + p) + 1];
                        re += kr * mr - ki * mi;
                        im += kr * mi + ki * mr;
                    }
                    O[2 * (a * np + p)] += re;
                    O[2 * (a * np + p) + 1] += im;
                }
            }
        }
        for (int a = 0; a < 3; a++) {
            double *Oa = O + 2 * a * np;
            dft3(Oa, Nx, Ny, Nz, +1);
            for (size_t c = 0; c < ncell; c++) {
                int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
                tmp[3 * c + a] = Oa[2 * ((size_t)i + (size_t)j * Nx + (size_t)k * Nx * Ny)] / (double)np;
            }
        }
        if (es_mode == 1) {
            const double *Mc = Mcs + 3 * ncell * d, *S = s->es_self + 3 * d;
            double *Hs = s->es_H[es_slot] + 3 * ncell * d;
            for (size_t i = 0; i < 3 * ncell; i++) Hs[i] = tmp[i] - S[i % 3] * Mc[i];
        }
        ml_transfer_out(s, d, tmp, H);
    }
    for (int l = 0; l < L; l++) free(F[l]);
    free(F); free(tmp); free(O); free(Mcs);
    return 0;
}

/* H_demag of every mesh (AoS, meshes concatenated) from M of every mesh */
int orc_ml_eval(orc_ml *s, const double *M, double *H)
{
    return orc_ml_eval_es(s, M, H, 0, 0, NULL, 0);
}

/* the transfer of one layer alone (tests): Mc = transfer_in(M), Hmesh = transfer_out(Hc) */
int orc_ml_transfer(orc_ml *s, int l, const double *M, double *Mc, const double *Hc, double *Hmesh)
{
    if (l < 0 || l >= s->L || !s->lay[l].transfer) return 1;
    ml_layer *y = &s->lay[l];
    const double *Mm = M + 3 * s->moff[y->mesh];
    size_t ncell = (size_t)s->nc[0] * s->nc[1] * s->nc[2];
    for (size_t c = 0; c < ncell; c++) {
        double v[3] = {0, 0, 0};
        for (int q = 0; q < y->tin[c].n; q++)
            for (int a = 0; a < 3; a++) v[a] += Mm[3 * (size_t)y->tin[c].idx[q] + a] * y->tin[c].w[q];
        for (int a = 0; a < 3; a++) Mc[3 * c + a] = v[a];
    }
    size_t n = s->moff[y->mesh + 1] - s->moff[y->mesh];
    for (size_t c = 0; c < n; c++) {
        double v[3] = {0, 0, 0};
        for (int q = 0; q < y->tout[c].n; q++)
            for (int a = 0; a < 3; a++) v[a] += Hc[3 * (size_t)y->tout[c].idx[q] + a] * y->tout[c].w[q];
        for (int a = 0; a < 3; a++) Hmesh[3 * c + a] = v[a];
    }
    return 0;
}

/* ------------------------------------------------------------------ supermesh demag */

/* SDemag with the multilayered convolution off (Boris/SDemag.cpp:737-760): M of every mesh moved onto
 * the ferromagnetic supermesh by the weighted mesh transfer, one demag convolution there (with the
 * supermesh's PBC images), the field moved back into every mesh.
 *   rectangle, cells  SuperMesh::UpdateConfiguration (Boris/SuperMeshControl.cpp:22-44): the bounding
 *                     box of the meshes (Rect::operator+=, BorisLib/Types_Rect.h:290), n = round(size /
 *                     h_request) per axis (at least 1), h = size / n
 *   transfer in       initialize_transfer_in_weighted over every input mesh (BorisLib/VEC_MeshTransfer.h:
 *                     901): per supermesh cell the covered-volume ratios and reciprocal-distance weights
 *                     summed over every overlapping mesh, then one normalisation
 *   transfer out      initialize_transfer_out (VEC_MeshTransfer.h:1221), reciprocal-distance weights
 *   non-empty cells   supermesh cells that a mesh covers (VEC::get_nonempty_cells after transfer_in,
 *                     SDemag.cpp:574-576, for a magnetisation without zero cells) */
struct orc_sm {
    int nmesh;
    int (*mn)[3];
    size_t *moff;
    int n[3];
    d3 h;
    rect3 rect;
    long nonempty;
    wlist **tin;      /* per mesh, per supermesh cell */
    wlist **tout;     /* per mesh, per mesh cell */
    orc_demag *dm;
};

orc_sm *orc_sm_create(int nmesh, const int *n3, const double *h3, const double *o3, const double *h_request,
                      const int *pbc)
{
    if (nmesh < 1) return NULL;
    orc_sm *s = (orc_sm *)calloc(1, sizeof(orc_sm));
    s->nmesh = nmesh;
    s->mn = (int (*)[3])calloc(nmesh, sizeof(int[3]));
    s->moff = (size_t *)calloc(nmesh + 1, sizeof(size_t));
    d3 *mh = (d3 *)calloc(nmesh, sizeof(d3));
    rect3 *mr = (rect3 *)calloc(nmesh, sizeof(rect3));
    for (int m = 0; m < nmesh; m++) {
        for (int a = 0; a < 3; a++) s->mn[m][a] = n3[3 * m + a];
        mh[m] = d3m(h3[3 * m], h3[3 * m + 1], h3[3 * m + 2]);
        mr[m].s = d3m(o3[3 * m], o3[3 * m + 1], o3[3 * m + 2]);
        mr[m].e = d3add(mr[m].s, d3m(mh[m].x * n3[3 * m], mh[m].y * n3[3 * m + 1], mh[m].z * n3[3 * m + 2]));
        s->moff[m + 1] = s->moff[m] + (size_t)n3[3 * m] * n3[3 * m + 1] * n3[3 * m + 2];
        if (m == 0) s->rect = mr[0];
        else {
            if (mr[m].s.x < s->rect.s.x) s->rect.s.x = mr[m].s.x;
            if (mr[m].s.y < s->rect.s.y) s->rect.s.y = mr[m].s.y;
            if (mr[m].s.z < s->rect.s.z) s->rect.s.z = mr[m].s.z;
            if (mr[m].e.x > s->rect.e.x) s->rect.e.x = mr[m].e.x;
            if (mr[m].e.y > s->rect.e.y) s->rect.e.y = mr[m].e.y;
            if (mr[m].e.z > s->rect.e.z) s->rect.e.z = mr[m].e.z;
        }
    }
    d3 sz = rsize(s->rect);
    double szv[3] = {sz.x, sz.y, sz.z}, hv[3];
    for (int a = 0; a < 3; a++) {
        double c = round(szv[a] / h_request[a]);
        s->n[a] = c < 1 ? 1 : (int)c;
        hv[a] = szv[a] / s->n[a];
    }
    s->h = d3m(hv[0], hv[1], hv[2]);
    size_t ncell = (size_t)s->n[0] * s->n[1] * s->n[2];
    s->tin = (wlist **)calloc(nmesh, sizeof(wlist *));
    s->tout = (wlist **)calloc(nmesh, sizeof(wlist *));
    for (int m = 0; m < nmesh; m++) s->tin[m] = (wlist *)calloc(ncell, sizeof(wlist));
    for (size_t c = 0; c < ncell; c++) {
        int ii = (int)(c % s->n[0]), jj = (int)((c / s->n[0]) % s->n[1]), kk = (int)(c / ((size_t)s->n[0] * s->n[1]));
        rect3 rc;
        rc.s = d3add(s->rect.s, d3m(s->h.x * ii, s->h.y * jj, s->h.z * kk));
        rc.e = d3add(rc.s, s->h);
        double tot = 0.0, cov = 0.0;
        for (int m = 0; m < nmesh; m++) {
            rect3 ri;
            if (rect_intersection(mr[m], rc, &ri) && !rect_isplane(ri) && !rect_ispoint(ri)) {
                d3 si = rsize(ri), sc = rsize(rc);
                cov += (si.x / sc.x) * (si.y / sc.y) * (si.z / sc.z);
                tot += recip_weights(&s->tin[m][c], rc, s->mn[m], mh[m], mr[m].s);
            }
        }
        if (cov > 0) s->nonempty++;
        if (tot > 0)
            for (int m = 0; m < nmesh; m++)
                for (int q = 0; q < s->tin[m][c].n; q++) s->tin[m][c].w[q] *= cov / tot;
    }
    for (int m = 0; m < nmesh; m++) {
        size_t n = s->moff[m + 1] - s->moff[m];
        s->tout[m] = (wlist *)calloc(n, sizeof(wlist));
        for (size_t c = 0; c < n; c++) {
            int ii = (int)(c % s->mn[m][0]), jj = (int)((c / s->mn[m][0]) % s->mn[m][1]);
            int kk = (int)(c / ((size_t)s->mn[m][0] * s->mn[m][1]));
            rect3 rc;
            rc.s = d3add(mr[m].s, d3m(mh[m].x * ii, mh[m].y * jj, mh[m].z * kk));
            rc.e = d3add(rc.s, mh[m]);
            double tot = recip_weights(&s->tout[m][c], rc, s->n, s->h, s->rect.s);
            if (tot > 0) for (int q = 0; q < s->tout[m][c].n; q++) s->tout[m][c].w[q] *= 1.0 / tot;
        }
    }
    s->dm = orc_demag_create_pbc(s->n[0], s->n[1], s->n[2], s->h.x, s->h.y, s->h.z, pbc);
    free(mh); free(mr);
    return s;
}

void orc_sm_destroy(orc_sm *s)
{
    if (!s) return;
    size_t ncell = (size_t)s->n[0] * s->n[1] * s->n[2];
    for (int m = 0; m < s->nmesh; m++) {
        for (size_t c = 0; c < ncell; c++) { free(s->tin[m][c].idx); free(s->tin[m][c].w); }
        size_t n = s->moff[m + 1] - s->moff[m];
        for (size_t c = 0; c < n; c++) { free(s->tout[m][c].idx); free(s->tout[m][c].w); }
        free(s->tin[m]); free(s->tout[m]);
    }
    free(s->tin); free(s->tout); free(s->mn); free(s->moff);
    orc_demag_destroy(s->dm);
    free(s);
}

int orc_sm_info(orc_sm *s, int *n3, double *h3, double *rect6, long *nonempty)
{
    for (int a = 0; a < 3; a++) {
        if (n3) n3[a] = s->n[a];
    }
    if (h3) { h3[0] = s->h.x; h3[1] = s->h.y; h3[2] = s->h.z; }
    if (rect6) {
        rect6[0] = s->rect.s.x; rect6[1] = s->rect.s.y; rect6[2] = s->rect.s.z;
        rect6[3] = s->rect.e.x; rect6[4] = s->rect.e.y; rect6[5] = s->rect.e.z;
    }
    if (nonempty) *nonempty = s->nonempty;
    return 0;
}

/* H_demag of every mesh (AoS, meshes concatenated) from M of every mesh; returns the reference's
 * supermesh energy density -mu0 / (2 non_empty_cells) sum_supermesh M . H */
double orc_sm_eval(orc_sm *s, const double *M, double *H)
{
    size_t ncell = (size_t)s->n[0] * s->n[1] * s->n[2];
    double *Ms = (double *)calloc(3 * ncell, sizeof(double));
    double *Hs = (double *)calloc(3 * ncell, sizeof(double));
    for (int m = 0; m < s->nmesh; m++) {
        const double *Mm = M + 3 * s->moff[m];
        for (size_t c = 0; c < ncell; c++)
            for (int q = 0; q < s->tin[m][c].n; q++)
                for (int a = 0; a < 3; a++) Ms[3 * c + a] += Mm[3 * (size_t)s->tin[m][c].idx[q] + a] * s->tin[m][c].w[q];
    }
    double dot = orc_demag_apply(s->dm, Ms, Hs, 0);
    for (int m = 0; m < s->nmesh; m++) {
        double *Hm = H + 3 * s->moff[m];
        size_t n = s->moff[m + 1] - s->moff[m];
        for (size_t c = 0; c < n; c++) {
            double v[3] = {0, 0, 0};
            for (int q = 0; q < s->tout[m][c].n; q++)
                for (int a = 0; a < 3; a++) v[a] += Hs[3 * (size_t)s->tout[m][c].idx[q] + a] * s->tout[m][c].w[q];
            for (int a = 0; a < 3; a++) Hm[3 * c + a] = v[a];
        }
    }
    free(Ms); free(Hs);
    return s->nonempty ? -ORC_MU0 * dot / (2.0 * (double)s->nonempty) : 0.0;
}

/* ------------------------------------------------------------------ field terms */

static double ms_at(const double *Ms_cell, size_t i) { return Ms_cell[i]; }

/* one axis of delsq_nneu / grad_nneu (VEC_VC_Del.h:141-200, VEC_VC_Grad.h:139-183) for a
 * full rectangular mesh; bd = boundary differential along this axis (0 = neu); wrap = 0, or the
 * sign (+1 / -1) of a periodic axis, whose missing neighbour is the cell on the far side times wrap
 * (the NF_PBC branches there; a one-cell axis has no neighbour either way) */
static void axis_terms_w(const double *M, size_t idx, int coord, int ncoord, size_t stride, double h,
                         const double *bd, int wrap, double *d2, double *g)
{
    int has_p = coord + 1 < ncoord, has_m = coord > 0;
    size_t ip = idx + stride, im = idx - stride;
    double sp = 1.0, sm = 1.0;
    if (wrap && ncoord > 1) {
        if (!has_p) { has_p = 1; ip = idx - (size_t)(ncoord - 1) * stride; sp = wrap; }
        if (!has_m) { has_m = 1; im = idx + (size_t)(ncoord - 1) * stride; sm = wrap; }
    }
    for (int c = 0; c < 3; c++) {
        double q = M[3 * idx + c];
        if (has_p && has_m) {
            double qp = sp * M[3 * ip + c], qm = sm * M[3 * im + c];
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

static void axis_terms(const double *M, size_t idx, int coord, int ncoord, size_t stride, double h,
                       const double *bd, double *d2, double *g)
{
    axis_terms_w(M, idx, coord, ncoord, stride, h, bd, 0, d2, g);
}

static int wrap_of(const int *pbc, int ax) { return pbc ? isgn(pbc[ax]) : 0; }

void orc_field_exchange_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                            double A, const double *Ms_cell, const int *pbc, double *H)
{
    static const double zero[3] = {0, 0, 0};
#pragma omp parallel for collapse(2) if (((long)nx * ny * nz) > ORC_PAR_MIN)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
                double dx[3], dy[3], dz[3], g[3];
                axis_terms_w(M, idx, i, nx, 1, hx, zero, wrap_of(pbc, 0), dx, g);
                axis_terms_w(M, idx, j, ny, nx, hy, zero, wrap_of(pbc, 1), dy, g);
                axis_terms_w(M, idx, k, nz, (size_t)nx * ny, hz, zero, wrap_of(pbc, 2), dz, g);
                double Ms = ms_at(Ms_cell, idx);
                double cst = 2.0 * A / (ORC_MU0 * Ms * Ms);
                for (int c = 0; c < 3; c++) H[3 * idx + c] += cst * (dx[c] + dy[c] + dz[c]);
            }
}

void orc_field_exchange(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                        double A, const double *Ms_cell, double *H)
{
    orc_field_exchange_pbc(nx, ny, nz, hx, hy, hz, M, A, Ms_cell, NULL, H);
}

void orc_field_idmi_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                        double A, double D, const double *Ms_cell, const int *pbc, double *H)
{
    static const double zero[3] = {0, 0, 0};
#pragma omp parallel for collapse(2) if (((long)nx * ny * nz) > ORC_PAR_MIN)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
                const double *m = M + 3 * idx;
                double r = D / (2.0 * A);
                double bx[3] = {r * m[2], 0.0, -r * m[0]};
                double by[3] = {0.0, r * m[2], -r * m[1]};
                double dx[3], dy[3], dz[3], gx[3], gy[3], gz[3];
                axis_terms_w(M, idx, i, nx, 1, hx, bx, wrap_of(pbc, 0), dx, gx);
                axis_terms_w(M, idx, j, ny, nx, hy, by, wrap_of(pbc, 1), dy, gy);
                axis_terms_w(M, idx, k, nz, (size_t)nx * ny, hz, zero, wrap_of(pbc, 2), dz, gz);
                double Ms = ms_at(Ms_cell, idx);
                double Ac = 2.0 * A / (ORC_MU0 * Ms * Ms);
                double Dc = -2.0 * D / (ORC_MU0 * Ms * Ms);
                double hd[3] = {gx[2], gy[2], -gx[0] - gy[1]};
                for (int c = 0; c < 3; c++) H[3 * idx + c] += Ac * (dx[c] + dy[c] + dz[c]) + Dc * hd[c];
            }
}

void orc_field_idmi(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                    double A, double D, const double *Ms_cell, double *H)
{
    orc_field_idmi_pbc(nx, ny, nz, hx, hy, hz, M, A, D, Ms_cell, NULL, H);
}

void orc_field_aniuni(int n, const double *M, const double *Ms_cell, const double *K1_cell, double K2,
                      const double *ea, double *H)
{
#pragma omp parallel for if ((n) > ORC_PAR_MIN)
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
    double *Hs[6];           /* evaluation speedup: saved demag fields minus the self term */
    double self[3];          /* self-demag coefficients (-N) */
    orc_field_fn hook;       /* caller's demag + exchange/iDMI terms, or NULL */
    void *hook_user;
} orc_mesh;

struct orc_solver {
    int nmesh;
    orc_mesh *m;
    orc_ml *ml;          /* multilayered convolution over the meshes with demag, or NULL */
    orc_sm *sm;          /* supermesh demag over the meshes with demag, or NULL */
    int *ml_mesh;        /* solver mesh of each multilayer mesh */
    int ml_nmesh;
    double *ml_M, *ml_H; /* concatenated M and H_demag of the multilayer meshes */
    int eval;
    double dT, tol, dT_incr, dT_min, dT_max;
    double time, stagetime;
    int primed;
    long accepted, rejected, evals;
    double last_lte;
    /* evaluation speedup (DemagCUDA::UpdateField, Boris/DemagCUDA.cpp:106): level K = number of
       saved fields, es_mode of the current evaluation (0 full, 1 full + save, 2 extrapolate) */
    int es_level, es_saved, es_mode, es_slot;
    double es_t[6], es_a[6];
    int es_available;    /* the reference's ODECommon_Base::available: the previous step completed */
    int es_metres;       /* the speedup's self term on cellsizes in metres (DemagCUDA.cpp:39 as is) */
    /* torque and dm/dt diagnostics (ODECommon_Base::Get_mxh / Get_dmdt, DiffEq_CommonBase_Get.cpp:7,19):
       a request makes the next step compute them, which clears the request */
    int calc_mxh, calc_dmdt;
    double mxh, dmdt;
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
            m->dm = orc_demag_create_pbc(desc[q].nx, desc[q].ny, desc[q].nz, desc[q].hx, desc[q].hy, desc[q].hz,
                                         desc[q].pbc);
    }
    return s;
}

/* Replace the per-mesh demag of every mesh with ORC_DEMAG by one multilayered convolution
 * (SDemag in multilayer mode); origins give the meshes' positions. */
int orc_solver_set_multilayer(orc_solver *s, const double *o3, int mode, const int *ncommon)
{
    int cnt = 0;
    for (int q = 0; q < s->nmesh; q++) if (s->m[q].d.modules & ORC_DEMAG) cnt++;
    if (!cnt) return 1;
    int *n3 = (int *)malloc(sizeof(int) * 3 * cnt);
    double *h3 = (double *)malloc(sizeof(double) * 3 * cnt), *oo = (double *)malloc(sizeof(double) * 3 * cnt);
    s->ml_mesh = (int *)malloc(sizeof(int) * cnt);
    size_t tot = 0;
    int k = 0;
    for (int q = 0; q < s->nmesh; q++) {
        const orc_mesh_desc *d = &s->m[q].d;
        if (!(d->modules & ORC_DEMAG)) continue;
        n3[3 * k] = d->nx; n3[3 * k + 1] = d->ny; n3[3 * k + 2] = d->nz;
        h3[3 * k] = d->hx; h3[3 * k + 1] = d->hy; h3[3 * k + 2] = d->hz;
        for (int a = 0; a < 3; a++) oo[3 * k + a] = o3[3 * q + a];
        s->ml_mesh[k++] = q;
        tot += (size_t)s->m[q].n;
    }
    s->ml_nmesh = cnt;
    s->ml = orc_ml_create(cnt, n3, h3, oo, mode, ncommon);
    s->ml_M = (double *)calloc(3 * tot, sizeof(double));
    s->ml_H = (double *)calloc(3 * tot, sizeof(double));
    free(n3); free(h3); free(oo);
    return s->ml ? 0 : 2;
}

/* Replace the per-mesh demag of every mesh with ORC_DEMAG by one supermesh convolution (SDemag with
 * the multilayered convolution off); origins give the meshes' positions. */
int orc_solver_set_supermesh(orc_solver *s, const double *o3, const double *h_request, const int *pbc)
{
    int cnt = 0;
    for (int q = 0; q < s->nmesh; q++) if (s->m[q].d.modules & ORC_DEMAG) cnt++;
    if (!cnt || s->ml || s->sm) return 1;
    int *n3 = (int *)malloc(sizeof(int) * 3 * cnt);
    double *h3 = (double *)malloc(sizeof(double) * 3 * cnt), *oo = (double *)malloc(sizeof(double) * 3 * cnt);
    s->ml_mesh = (int *)malloc(sizeof(int) * cnt);
    size_t tot = 0;
    int k = 0;
    for (int q = 0; q < s->nmesh; q++) {
        const orc_mesh_desc *d = &s->m[q].d;
        if (!(d->modules & ORC_DEMAG)) continue;
        n3[3 * k] = d->nx; n3[3 * k + 1] = d->ny; n3[3 * k + 2] = d->nz;
        h3[3 * k] = d->hx; h3[3 * k + 1] = d->hy; h3[3 * k + 2] = d->hz;
        for (int a = 0; a < 3; a++) oo[3 * k + a] = o3[3 * q + a];
        s->ml_mesh[k++] = q;
        tot += (size_t)s->m[q].n;
    }
    s->ml_nmesh = cnt;
    s->sm = orc_sm_create(cnt, n3, h3, oo, h_request, pbc);
    s->ml_M = (double *)calloc(3 * tot, sizeof(double));
    s->ml_H = (double *)calloc(3 * tot, sizeof(double));
    free(n3); free(h3); free(oo);
    return s->sm ? 0 : 2;
}

void orc_solver_destroy(orc_solver *s)
{
    if (!s) return;
    if (s->sm) { orc_sm_destroy(s->sm); free(s->ml_mesh); free(s->ml_M); free(s->ml_H); }
    if (s->ml) { orc_ml_destroy(s->ml); free(s->ml_mesh); free(s->ml_M); free(s->ml_H); }
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        free(m->Ms); free(m->K1); free(m->M); free(m->H); free(m->sM1);
        for (int e = 0; e < 6; e++) { free(m->sEval[e]); free(m->Hs[e]); }
        orc_demag_destroy(m->dm);
    }
    free(s->m);
    free(s);
}

int orc_set_m(orc_solver *s, int q, const double *M)
{
    memcpy(s->m[q].M, M, sizeof(double) * 3 * s->m[q].n);
    s->primed = 0;
    /* a new state drops the fields saved for the evaluation speedup */
    s->es_saved = 0;
    s->es_available = 1;
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
/* multilayered convolution of all multilayer meshes into s->ml_H */
static void update_ml(orc_solver *s)
{
    size_t off = 0;
    for (int k = 0; k < s->ml_nmesh; k++) {
        orc_mesh *m = &s->m[s->ml_mesh[k]];
        memcpy(s->ml_M + 3 * off, m->M, sizeof(double) * 3 * m->n);
        off += (size_t)m->n;
    }
    if (s->sm) orc_sm_eval(s->sm, s->ml_M, s->ml_H);
    else orc_ml_eval_es(s->ml, s->ml_M, s->ml_H, s->es_mode, s->es_slot, s->es_a, s->es_level);
}

static void update_fields(orc_solver *s, orc_mesh *m)
{
    const orc_mesh_desc *d = &m->d;
    size_t n = (size_t)m->n;
    double Ha[3];
    applied_field(d, s->stagetime, Ha);
#pragma omp parallel for if ((n) > ORC_PAR_MIN)
    for (long i = 0; i < (long)n; i++) { m->H[3 * i] = Ha[0]; m->H[3 * i + 1] = Ha[1]; m->H[3 * i + 2] = Ha[2]; }
    if (m->hook) {
        m->hook(m->hook_user, m->M, m->H);
        if (d->modules & ORC_ANIUNI) orc_field_aniuni(m->n, m->M, m->Ms, m->K1, d->K2, d->ea, m->H);
        return;
    }
    if ((d->modules & ORC_DEMAG) && (s->ml || s->sm)) {
        size_t off = 0;
        for (int k = 0; k < s->ml_nmesh; k++) {
            orc_mesh *mk = &s->m[s->ml_mesh[k]];
            if (mk == m) { for (size_t i = 0; i < 3 * n; i++) m->H[i] += s->ml_H[3 * off + i]; break; }
            off += (size_t)mk->n;
        }
    } else if ((d->modules & ORC_DEMAG) && s->es_mode == 1) {
        /* Demag_EvalSpeedup_AddField_SubSelf (Boris/DemagCUDA.cu:46): add the new field, keep it
           minus the self term */
        double *Hs = m->Hs[s->es_slot];
        memset(Hs, 0, sizeof(double) * 3 * n);
        orc_demag_apply(m->dm, m->M, Hs, 1);
        for (size_t i = 0; i < 3 * n; i++) { m->H[i] += Hs[i]; Hs[i] -= m->self[i % 3] * m->M[i]; }
    } else if ((d->modules & ORC_DEMAG) && s->es_mode == 2) {
        /* Demag_EvalSpeedup_AddExtrapField_AddSelf (Boris/DemagCUDA.cu:64-265) */
        for (size_t i = 0; i < 3 * n; i++) {
            double v = m->self[i % 3] * m->M[i];
            for (int k = 0; k < s->es_level; k++) v += s->es_a[k] * m->Hs[k][i];
            m->H[i] += v;
        }
    } else if (d->modules & ORC_DEMAG) orc_demag_apply(m->dm, m->M, m->H, 1);
    if (d->modules & ORC_IDMI)
        orc_field_idmi_pbc(d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, m->M, d->A, d->D, m->Ms, d->pbc, m->H);
    else if (d->modules & ORC_EXCH)
        orc_field_exchange_pbc(d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, m->M, d->A, m->Ms, d->pbc, m->H);
    if (d->modules & ORC_ANIUNI) orc_field_aniuni(m->n, m->M, m->Ms, m->K1, d->K2, d->ea, m->H);
}

static void update_all_fields(orc_solver *s)
{
    if (s->ml || s->sm) update_ml(s);
    for (int q = 0; q < s->nmesh; q++) update_fields(s, &s->m[q]);
    s->evals++;
}

int orc_solver_set_field_hook(orc_solver *s, int q, orc_field_fn fn, void *user)
{
    if (q < 0 || q >= s->nmesh || s->ml || s->sm || s->es_level) return 1;
    s->m[q].hook = fn;
    s->m[q].hook_user = user;
    return 0;
}

int orc_compute_heff(orc_solver *s, int q, double *H)
{
    if (s->ml || s->sm) update_ml(s);
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

/* |M x H| / |M|^2 of one cell (DiffEqFM_Evals_RK4.cpp:78-79, DiffEqFM_EvalsCUDA_RKDP54.cu:31-32) */
static inline double cell_mxh(const double *M, const double *H)
{
    double x[3] = {M[1] * H[2] - M[2] * H[1], M[2] * H[0] - M[0] * H[2], M[0] * H[1] - M[1] * H[0]};
    double m2 = M[0] * M[0] + M[1] * M[1] + M[2] * M[2];
    return sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) / m2;
}

/* |M - M1| / (dT GAMMA |M|^2) of one cell after the step's last stage (DiffEqFM_Evals_RK4.cpp:191-199,
   DiffEqFM_EvalsCUDA_RKDP54.cu:215-217) */
static inline double cell_dmdt(const double *M, const double *M1, double dT)
{
    double d[3] = {M[0] - M1[0], M[1] - M1[1], M[2] - M1[2]};
    double m2 = M[0] * M[0] + M[1] * M[1] + M[2] * M[2];
    return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / (dT * ORC_GAMMA * m2);
}

/* the maximum over the meshes whose grel is non-zero of cell_mxh at the current M and H (the
   stage-0 reduction of the RK4 and RKDP54 evaluators) */
static double max_mxh(orc_solver *s)
{
    double v = 0.0;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        if (m->d.grel == 0.0) continue;
        for (int i = 0; i < m->n; i++) {
            double c = cell_mxh(m->M + 3 * (size_t)i, m->H + 3 * (size_t)i);
            if (c > v) v = c;
        }
    }
    return v;
}

/* the maximum over the meshes whose grel is non-zero of cell_dmdt after the last stage */
static double max_dmdt(orc_solver *s, double dT)
{
    double v = 0.0;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        if (m->d.grel == 0.0) continue;
        for (int i = 0; i < m->n; i++) {
            double c = cell_dmdt(m->M + 3 * (size_t)i, m->sM1 + 3 * (size_t)i, dT);
            if (c > v) v = c;
        }
    }
    return v;
}

int orc_solver_get_mxh(orc_solver *s, double *v)
{
    s->calc_mxh = 1;
    if (v) *v = s->mxh;
    return 0;
}

int orc_solver_get_dmdt(orc_solver *s, double *v)
{
    s->calc_dmdt = 1;
    if (v) *v = s->dmdt;
    return 0;
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

/* Evaluation speedup for one RK4 evaluation (DemagCUDA::UpdateField, Boris/DemagCUDA.cpp:106-470,
   with ODECommon_Base::Check_Step_Update / Get_EvalStep_Time, Boris/DiffEq_CommonBase_Iterate.cpp:
   1536,1639, dTspeedup linked to dT): the first evaluation of a step computes the field and saves it
   (into the next free slot, then into the slot holding the earliest time); the others compute it in
   full until `level` fields are saved, then extrapolate with the Lagrange polynomial through the
   saved times. */
/* the slot the next saved field goes to (Boris/DemagCUDA.cpp:158-280): the next free one while fewer
   than K are saved; then the first when the saved times increase, else the first slot whose time is
   below its predecessor's, else the last */
static int es_slot_rule(const orc_solver *s)
{
    int K = s->es_level;
    if (s->es_saved < K) return s->es_saved;
    if (K == 1) return 0;
    int inc = 1;
    for (int k = 1; k < K; k++) inc = inc && (s->es_t[k] > s->es_t[k - 1]);
    if (inc) return 0;
    for (int j = 1; j < K - 1; j++)
        if (s->es_t[j - 1] > s->es_t[j]) return j;
    return K - 1;
}

/* save the field of this evaluation (time t) into the slot of the rule; a save at a time already
   saved replaces that slot instead (deviation: under RKDP54 the last stage and the next step's first
   evaluation share the time t + dT, and the reference's rule would then keep two fields at one time,
   a zero Lagrange denominator at level 6) */
static void es_save_at(orc_solver *s, double t)
{
    for (int k = 0; k < s->es_saved; k++)
        if (s->es_t[k] == t) {
            s->es_slot = k;
            s->es_mode = 1;
            return;
        }
    int slot = es_slot_rule(s);
    /* a level-1 (step) save keeps its time once cycling (Boris/DemagCUDA.cpp:276) */
    if (!(s->es_level == 1 && s->es_saved >= 1)) s->es_t[slot] = t;
    if (s->es_saved < s->es_level) s->es_saved++;
    s->es_slot = slot;
    s->es_mode = 1;
}

static void es_weights(orc_solver *s, double t)
{
    int K = s->es_level;
    for (int k = 0; k < K; k++) {
        double a = 1.0;
        for (int j = 0; j < K; j++)
            if (j != k) a *= (t - s->es_t[j]) / (s->es_t[k] - s->es_t[j]);
        s->es_a[k] = a;
    }
    s->es_mode = 2;
}

static void es_prepare(orc_solver *s, int stage)
{
    static const double c_rk4[4] = {0.0, 0.5, 0.5, 1.0};
    s->es_mode = 0;
    if (!s->es_level) return;
    int K = s->es_level;
    double t = s->time + s->dT * c_rk4[stage];
    if (stage == 0) es_save_at(s, t);
    else if (s->es_saved >= K) es_weights(s, t);
}

/* RKDP54 (DemagCUDA::UpdateField, Boris/DemagCUDA.cpp:139-144, with Check_Step_Update returning
   `available` and Get_EvalStep_Time at the Dormand-Prince nodes, Boris/DiffEq_CommonBase_Iterate.cpp:
   1562,1656): compute and save when the previous step completed and this is the attempt's first
   evaluation, or while fewer than K are saved; extrapolate otherwise */
static void es_prepare_dp(orc_solver *s, int eval)
{
    static const double c_dp[6] = {0.0, 0.2, 0.3, 0.8, 8.0 / 9, 1.0};
    s->es_mode = 0;
    if (!s->es_level) return;
    double t = s->time + s->dT * c_dp[eval];
    if ((eval == 0 && s->es_available) || s->es_saved < s->es_level) es_save_at(s, t);
    else es_weights(s, t);
}

/* the speedup's self term: 0 on normalised cellsizes, 1 on cellsizes in metres as the reference computes
   it; takes effect at the next orc_solver_set_evalspeedup */
int orc_solver_set_evalspeedup_self(orc_solver *s, int metres)
{
    s->es_metres = metres != 0;
    if (s->ml) {
        s->ml->es_metres = s->es_metres;
        free(s->ml->es_self);
        s->ml->es_self = NULL;
    }
    return 0;
}

int orc_solver_set_evalspeedup(orc_solver *s, int level)
{
    if (level < 0 || level > 6 || s->sm) return 1;
    s->es_level = level;
    s->es_saved = 0;
    s->es_available = 1;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        {
            const int n3[3] = {m->d.nx, m->d.ny, m->d.nz};
            selfdemag_pbc_core(m->d.hx, m->d.hy, m->d.hz, n3, m->d.pbc, m->self, s->es_metres);
        }
        for (int k = 0; k < 6; k++) {
            free(m->Hs[k]);
            m->Hs[k] = k < level ? (double *)calloc(3 * (size_t)m->n, sizeof(double)) : NULL;
        }
    }
    return 0;
}

static void rk4_step(orc_solver *s)
{
    double dT = s->dT;
    for (int stage = 0; stage < 4; stage++) {
        es_prepare(s, stage);
        update_all_fields(s);
        if (stage == 0 && s->calc_mxh) {
            s->mxh = max_mxh(s);
            s->calc_mxh = 0;
        }
        for (int q = 0; q < s->nmesh; q++) {
            orc_mesh *m = &s->m[q];
            const orc_mesh_desc *d = &m->d;
#pragma omp parallel for if ((m->n) > ORC_PAR_MIN)
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
    if (s->calc_dmdt) {
        s->dmdt = max_dmdt(s, dT);
        s->calc_dmdt = 0;
    }
    s->time += dT;
    s->stagetime += dT;
    s->accepted++;
}

/* one RKDP54 attempt: returns 1 if a step was completed, 0 if the previous one was rejected */
static int rkdp_attempt(orc_solver *s)
{
    /* evalStep 0: FSAL rhs, 4th-order prediction, lte (DiffEqFM_Evals_RKDP54.cpp:52-88) */
    es_prepare_dp(s, 0);
    update_all_fields(s);
    if (s->calc_mxh) {
        s->mxh = max_mxh(s);
        s->calc_mxh = 0;
    }
    double lte = 0.0;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
        const orc_mesh_desc *d = &m->d;
        double dT = s->dT;
        double lmax = 0.0;
#pragma omp parallel for reduction(max:lmax) if ((m->n) > ORC_PAR_MIN)
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
            s->es_available = 0;   /* failed - must repeat (SetAdaptiveTimeStep) */
            return 0;
        }
    } else s->primed = 1;
    double dT = s->dT;
    for (int q = 0; q < s->nmesh; q++) {
        orc_mesh *m = &s->m[q];
#pragma omp parallel for if ((m->n) > ORC_PAR_MIN)
        for (long o = 0; o < 3 * (long)m->n; o++) {
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
        es_prepare_dp(s, st);
        update_all_fields(s);
        for (int q = 0; q < s->nmesh; q++) {
            orc_mesh *m = &s->m[q];
            const orc_mesh_desc *d = &m->d;
#pragma omp parallel for if ((m->n) > ORC_PAR_MIN)
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
    if (s->calc_dmdt) {
        s->dmdt = max_dmdt(s, dT);
        s->calc_dmdt = 0;
    }
    s->time += dT;
    s->stagetime += dT;
    s->accepted++;
    s->es_available = 1;   /* done for this step (the reference's `available = true`) */
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

/* ------------------------------------------------------------------ discrete adjoint of RK4 */
/* Forward: the solver's RK4 step (DiffEqFM_Evals_RK4.cpp, renormalisation to Ms; the Zeeman sample
 * is the one at the step start time, as the solver takes it), modules demag + exchange + uniaxial
 * anisotropy (K2 = 0) + Zeeman, per-cell Ms and K1; the initial state is M0 = Ms m0.
 * Loss: L = (1/n) sum_i |M_i(T)/Ms_i - target_i|^2.
 * Backward: reverse mode through every stage of every step, the renormalisation and the field terms
 * (the project's own derivation; the reference has no adjoint). The demag operator D and the
 * Neumann Laplacian L are symmetric, so their transposes are themselves. States of every step are
 * kept (test sizes); each step's stages are recomputed in the backward sweep. */

typedef struct {
    const orc_mesh_desc *d;
    orc_demag *dm;
    int n;
    const double *Ms, *K1;
    double *tmp;
} adj_ctx;

static void adj_fields(adj_ctx *a, const double *X, const double *Ha, double *H)
{
    const orc_mesh_desc *d = a->d;
    for (int i = 0; i < a->n; i++) { H[3 * i] = Ha[0]; H[3 * i + 1] = Ha[1]; H[3 * i + 2] = Ha[2]; }
    if (d->modules & ORC_DEMAG) orc_demag_apply(a->dm, X, H, 1);
    if (d->modules & ORC_EXCH) orc_field_exchange_pbc(d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, X, d->A, a->Ms, d->pbc, H);
    if (d->modules & ORC_ANIUNI) orc_field_aniuni(a->n, X, a->Ms, a->K1, 0.0, d->ea, H);
}

/* out = L V per component (Neumann: only existing neighbours) */
static void adj_lap(const orc_mesh_desc *d, const double *V, double *out)
{
    static const double zero[3] = {0, 0, 0};
    int nx = d->nx, ny = d->ny, nz = d->nz;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)i + (size_t)j * nx + (size_t)k * nx * ny;
                double dx[3], dy[3], dz[3], g[3];
                axis_terms_w(V, idx, i, nx, 1, d->hx, zero, wrap_of(d->pbc, 0), dx, g);
                axis_terms_w(V, idx, j, ny, nx, d->hy, zero, wrap_of(d->pbc, 1), dy, g);
                axis_terms_w(V, idx, k, nz, (size_t)nx * ny, d->hz, zero, wrap_of(d->pbc, 2), dz, g);
                for (int c = 0; c < 3; c++) out[3 * idx + c] = dx[c] + dy[c] + dz[c];
            }
}

/* one RK4 step from M0 at time t; stage inputs X[0..3], fields H[0..3], pre-normalisation Y */
static void adj_step(adj_ctx *a, const double *M0, double t, double dt, double *X[4], double *H[4], double *Y, double *Mout)
{
    const orc_mesh_desc *d = a->d;
    const int n = a->n;
    double Ha[3];
    applied_field(d, t, Ha);
    double *k = a->tmp;   /* 4 x 3n */
    static const double cx[4] = {0.0, 0.5, 0.5, 1.0};
    for (int s = 0; s < 4; s++) {
        if (s == 0) memcpy(X[0], M0, sizeof(double) * 3 * n);
        else
            for (int i = 0; i < 3 * n; i++) X[s][i] = M0[i] + cx[s] * dt * k[(size_t)(s - 1) * 3 * n + i];
        adj_fields(a, X[s], Ha, H[s]);
        for (int i = 0; i < n; i++) llg(X[s] + 3 * i, H[s] + 3 * i, a->Ms[i], d->alpha, d->grel, k + (size_t)s * 3 * n + 3 * i);
    }
    for (int i = 0; i < 3 * n; i++)
        Y[i] = M0[i] + (k[i] + 2 * k[3 * n + i] + 2 * k[6 * n + i] + k[9 * n + i]) * (dt / 6);
    for (int i = 0; i < n; i++) {
        double *y = Y + 3 * i, nr = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
        for (int c = 0; c < 3; c++) Mout[3 * i + c] = a->Ms[i] * y[c] / nr;
    }
}

/* gX = (d f / d X)^T mu for f = LLG(X, H(X)) at one stage; accumulates the parameter gradients */
static void adj_vjp(adj_ctx *a, const double *X, const double *H, const double *mu, double t, double *gX, double *gMs,
                    double *gK1, double *gHa)
{
    const orc_mesh_desc *d = a->d;
    const int n = a->n;
    double *gH = a->tmp + 12 * (size_t)n, *w = a->tmp + 15 * (size_t)n, *lx = a->tmp + 18 * (size_t)n;
    const double al = d->alpha, pre = -ORC_GAMMA * d->grel / (1.0 + al * al);
    for (int i = 0; i < n; i++) {
        const double *x = X + 3 * i, *h = H + 3 * i, *m = mu + 3 * i;
        const double Ms = a->Ms[i], b = pre * al / Ms;
        double xh = x[0] * h[0] + x[1] * h[1] + x[2] * h[2];
        double mx = m[0] * x[0] + m[1] * x[1] + m[2] * x[2];
        double mh = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
        double xx = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        double hxm[3] = {h[1] * m[2] - h[2] * m[1], h[2] * m[0] - h[0] * m[2], h[0] * m[1] - h[1] * m[0]};
        double mxx[3] = {m[1] * x[2] - m[2] * x[1], m[2] * x[0] - m[0] * x[2], m[0] * x[1] - m[1] * x[0]};
        for (int c = 0; c < 3; c++) {
            gX[3 * i + c] = pre * hxm[c] + b * (xh * m[c] + mx * h[c] - 2.0 * mh * x[c]);
            gH[3 * i + c] = pre * mxx[c] + b * (mx * x[c] - xx * m[c]);
        }
        /* d/dMs of (alpha/Ms) X x (X x H): mu . (X (X.H) - H |X|^2) times -alpha pre / Ms^2 */
        gMs[i] += -pre * al / (Ms * Ms) * (mx * xh - mh * xx);
    }
    /* Zeeman */
    if ((d->modules & ORC_ZEEMAN) && d->Ha && d->nHa > 0) {
        int idx = 0;
        if (d->nHa > 1 && d->Ha_tspan > 0.0) {
            idx = (int)floor(t / d->Ha_tspan * d->nHa);
            if (idx < 0) idx = 0;
            if (idx >= d->nHa) idx = d->nHa - 1;
        }
        for (int i = 0; i < n; i++)
            for (int c = 0; c < 3; c++) gHa[3 * idx + c] += gH[3 * i + c];
    }
    /* demag: D is symmetric */
    if (d->modules & ORC_DEMAG) {
        orc_demag_apply(a->dm, gH, w, 0);
        for (int i = 0; i < 3 * n; i++) gX[i] += w[i];
    }
    /* exchange: H = c (L X), c_i = 2 A / (mu0 Ms_i^2) */
    if (d->modules & ORC_EXCH) {
        for (int i = 0; i < n; i++) {
            double ci = 2.0 * d->A / (ORC_MU0 * a->Ms[i] * a->Ms[i]);
            for (int c = 0; c < 3; c++) w[3 * i + c] = ci * gH[3 * i + c];
        }
        adj_lap(d, w, lx);
        for (int i = 0; i < 3 * n; i++) gX[i] += lx[i];
        adj_lap(d, X, lx);
        for (int i = 0; i < n; i++) {
            double ci = 2.0 * d->A / (ORC_MU0 * a->Ms[i] * a->Ms[i]);
            double dot = gH[3 * i] * lx[3 * i] + gH[3 * i + 1] * lx[3 * i + 1] + gH[3 * i + 2] * lx[3 * i + 2];
            gMs[i] += dot * (-2.0 * ci / a->Ms[i]);
        }
    }
    /* uniaxial anisotropy: H = kappa (X.e) e, kappa_i = 2 K1_i / (mu0 Ms_i^2) */
    if (d->modules & ORC_ANIUNI) {
        const double *e = d->ea;
        for (int i = 0; i < n; i++) {
            double Ms = a->Ms[i], kap = 2.0 * a->K1[i] / (ORC_MU0 * Ms * Ms);
            double xe = X[3 * i] * e[0] + X[3 * i + 1] * e[1] + X[3 * i + 2] * e[2];
            double ge = gH[3 * i] * e[0] + gH[3 * i + 1] * e[1] + gH[3 * i + 2] * e[2];
            for (int c = 0; c < 3; c++) gX[3 * i + c] += kap * ge * e[c];
            gK1[i] += xe * ge * 2.0 / (ORC_MU0 * Ms * Ms);
            gMs[i] += xe * ge * (-2.0 * kap / Ms);
        }
    }
}

int orc_adjoint_rk4(const orc_mesh_desc *d, const double *m0, const double *target, int steps, double dt,
                    double *loss, double *gMs, double *gK1, double *gHa)
{
    adj_ctx a;
    a.d = d;
    a.n = d->nx * d->ny * d->nz;
    const int n = a.n;
    double *Ms = (double *)malloc(sizeof(double) * n), *K1 = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) {
        Ms[i] = d->Ms_map ? d->Ms_map[i] : d->Ms;
        K1[i] = d->K1_map ? d->K1_map[i] : d->K1;
    }
    a.Ms = Ms; a.K1 = K1;
    a.dm = (d->modules & ORC_DEMAG) ? orc_demag_create_pbc(d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, d->pbc) : 0;
    a.tmp = (double *)calloc(21 * (size_t)n, sizeof(double));
    size_t v3 = 3 * (size_t)n;
    double *Ms_hist = (double *)malloc(sizeof(double) * v3 * (steps + 1));
    double *tm = (double *)malloc(sizeof(double) * (steps + 1));
    double *X[4], *H[4];
    for (int s = 0; s < 4; s++) { X[s] = (double *)malloc(sizeof(double) * v3); H[s] = (double *)malloc(sizeof(double) * v3); }
    double *Y = (double *)malloc(sizeof(double) * v3);
    /* forward */
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) Ms_hist[3 * i + c] = Ms[i] * m0[3 * i + c];
    tm[0] = 0.0;
    for (int st = 0; st < steps; st++) {
        adj_step(&a, Ms_hist + st * v3, tm[st], dt, X, H, Y, Ms_hist + (st + 1) * v3);
        tm[st + 1] = tm[st] + dt;
    }
    /* loss and its gradient at the final state */
    for (int i = 0; i < n; i++) gMs[i] = 0.0, gK1[i] = 0.0;
    if (gHa && d->nHa > 0) memset(gHa, 0, sizeof(double) * 3 * d->nHa);
    double *lam = (double *)malloc(sizeof(double) * v3), *lY = (double *)malloc(sizeof(double) * v3);
    double *mu = (double *)malloc(sizeof(double) * v3), *gX = (double *)malloc(sizeof(double) * v3);
    const double *MT = Ms_hist + steps * v3;
    double L = 0.0;
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) {
            double m = MT[3 * i + c] / Ms[i], r = m - target[3 * i + c];
            L += r * r;
            lam[3 * i + c] = 2.0 / n * r / Ms[i];
            gMs[i] += 2.0 / n * r * (-m / Ms[i]);
        }
    *loss = L / n;
    double dummyHa[3 * 256];
    double *gHa_use = gHa ? gHa : dummyHa;
    /* backward */
    for (int st = steps - 1; st >= 0; st--) {
        adj_step(&a, Ms_hist + st * v3, tm[st], dt, X, H, Y, gX);   /* recompute the stages */
        for (int i = 0; i < n; i++) {
            double *y = Y + 3 * i, nr = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
            double yl = (y[0] * lam[3 * i] + y[1] * lam[3 * i + 1] + y[2] * lam[3 * i + 2]) / nr;
            gMs[i] += yl;
            for (int c = 0; c < 3; c++) lY[3 * i + c] = Ms[i] / nr * (lam[3 * i + c] - yl * y[c] / nr);
        }
        /* lam <- dL/dM_st */
        memcpy(lam, lY, sizeof(double) * v3);
        for (int i = 0; i < (int)v3; i++) mu[i] = dt / 6 * lY[i];
        adj_vjp(&a, X[3], H[3], mu, tm[st], gX, gMs, gK1, gHa_use);
        for (int i = 0; i < (int)v3; i++) { lam[i] += gX[i]; mu[i] = dt / 3 * lY[i] + dt * gX[i]; }
        adj_vjp(&a, X[2], H[2], mu, tm[st], gX, gMs, gK1, gHa_use);
        for (int i = 0; i < (int)v3; i++) { lam[i] += gX[i]; mu[i] = dt / 3 * lY[i] + dt / 2 * gX[i]; }
        adj_vjp(&a, X[1], H[1], mu, tm[st], gX, gMs, gK1, gHa_use);
        for (int i = 0; i < (int)v3; i++) { lam[i] += gX[i]; mu[i] = dt / 6 * lY[i] + dt / 2 * gX[i]; }
        adj_vjp(&a, X[0], H[0], mu, tm[st], gX, gMs, gK1, gHa_use);
        for (int i = 0; i < (int)v3; i++) lam[i] += gX[i];
    }
    /* initial state M0 = Ms m0 */
    for (int i = 0; i < n; i++)
        gMs[i] += m0[3 * i] * lam[3 * i] + m0[3 * i + 1] * lam[3 * i + 1] + m0[3 * i + 2] * lam[3 * i + 2];
    for (int s = 0; s < 4; s++) { free(X[s]); free(H[s]); }
    free(Y); free(lam); free(lY); free(mu); free(gX); free(Ms_hist); free(tm); free(a.tmp); free(Ms); free(K1);
    orc_demag_destroy(a.dm);
    return 0;
}
