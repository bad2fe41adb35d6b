/*
 * Oracle test infrastructure (CPU, FP64). Not part of the product path.
 *
 * A small FP64 FFT written for this project, exposed under the subset of the
 * FFTW3 API that the reference's demag code calls, so that the reference's own
 * sources can be compiled and run here without FFTW:
 *   - ConvolutionData.cpp:180-208   fftw_plan_many_dft_r2c / _dft / _dft_c2r
 *   - DemagKernel.cpp:225-243,348-361 fftw_plan_many_dft_r2c
 *   - Convolution.h (all fftw_execute calls)
 * FFTW itself is a third-party dependency that is not vendored in the
 * reference (only its header Boris/fftw3.h, version unpinned). The transform it
 * computes is the plain DFT, X[k] = sum_n x[n] exp(sign * 2 pi i n k / N),
 * unnormalised in both directions; that definition is what this file restates.
 *
 * Algorithm: recursive mixed-radix decimation in time over the prime factors
 * of N (radix 2, 3, 5 and a direct DFT for any other prime factor), with
 * twiddles taken from a per-plan table of exp(-2 pi i m / N) computed with
 * sin/cos of reduced arguments. The oracle's own restatement (oracle.c) uses
 * the same entry point through bm_oracle_fft().
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef double fftw_complex[2];

typedef struct fftw_plan_s {
    int kind;          /* 0 = c2c, 1 = r2c, 2 = c2r */
    int n, howmany;
    int istride, idist, ostride, odist;
    int sign;
    void *in, *out;
    double *tw;        /* 2*n: exp(-2 pi i m / n) */
    double *work;      /* 4*n scratch */
} *fftw_plan;

static double *make_twiddles(int n)
{
    double *tw = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    for (int m = 0; m < n; m++) {
        /* reduce to the first octant-ish by symmetry for accuracy */
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        tw[2 * m + 0] = (double)cosl(a);
        tw[2 * m + 1] = (double)-sinl(a);
    }
    return tw;
}

static int smallest_factor(int n)
{
    if (n % 2 == 0) return 2;
    if (n % 3 == 0) return 3;
    if (n % 5 == 0) return 5;
    for (int p = 7; p * p <= n; p += 2) if (n % p == 0) return p;
    return n;
}

/* out[k*os] = sum_j in[j*is] w^(j k); w = exp(sign 2 pi i / n) via table of full length N
 * (tw_step = N / n). tmp has room for 2*n doubles. */
static void fft_rec(int n, const double *in, int is, double *out, int os,
                    int sign, const double *tw, int tw_step, double *tmp)
{
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    int p = smallest_factor(n);
    int m = n / p;
    /* sub-transforms of length m on decimated inputs, written contiguously to out */
    for (int r = 0; r < p; r++)
        fft_rec(m, in + 2 * (size_t)r * is, is * p, out + 2 * (size_t)r * m * os, os, sign, tw, tw_step * p, tmp);
    /* combine: X[k + q m] = sum_r w_n^{r (k + q m)} S_r[k] */
    for (int k = 0; k < m; k++) {
        double s[2 * 64];
        double *sv = (p <= 64) ? s : (double *)malloc(sizeof(double) * 2 * p);
        for (int r = 0; r < p; r++) {
            sv[2 * r] = out[2 * ((size_t)(r * m + k)) * os];
            sv[2 * r + 1] = out[2 * ((size_t)(r * m + k)) * os + 1];
        }
        for (int q = 0; q < p; q++) {
            double ar = 0.0, ai = 0.0;
            for (int r = 0; r < p; r++) {
                long e = ((long)r * (long)(k + q * m)) % n;
                double wr = tw[2 * (e * tw_step)];
                double wi = tw[2 * (e * tw_step) + 1];
                if (sign > 0) wi = -wi;
                ar += sv[2 * r] * wr - sv[2 * r + 1] * wi;
                ai += sv[2 * r] * wi + sv[2 * r + 1] * wr;
            }
            tmp[2 * (k + q * m)] = ar;
            tmp[2 * (k + q * m) + 1] = ai;
        }
        if (sv != s) free(sv);
    }
    for (int k = 0; k < n; k++) {
        out[2 * (size_t)k * os] = tmp[2 * k];
        out[2 * (size_t)k * os + 1] = tmp[2 * k + 1];
    }
}

/* complex DFT of length n, contiguous in/out (may alias is not allowed) */
static void cdft(int n, const double *in, double *out, int sign, const double *tw, double *tmp)
{
    fft_rec(n, in, 1, out, 1, sign, tw, 1, tmp);
}

/* exported helper for the oracle restatement: in-place complex DFT of length n, stride 1 */
void bm_oracle_fft(int n, double *data, int sign)
{
    double *tw = make_twiddles(n);
    double *a = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    memcpy(a, data, sizeof(double) * 2 * (size_t)n);
    cdft(n, a, data, sign, tw, tmp);
    free(a); free(tmp); free(tw);
}

/* reusable twiddle table + in-place transform with caller scratch (4n doubles);
 * safe to call from several threads on one table */
double *bm_fft_table(int n) { return make_twiddles(n); }
void bm_fft_table_free(double *tw) { free(tw); }
void bm_fft_exec(int n, const double *tw, double *data, int sign, double *scratch)
{
    double *a = scratch, *tmp = scratch + 2 * (size_t)n;
    memcpy(a, data, sizeof(double) * 2 * (size_t)n);
    cdft(n, a, data, sign, tw, tmp);
}

static fftw_plan new_plan(int kind, int n, int howmany, void *in, int istride, int idist,
                          void *out, int ostride, int odist, int sign)
{
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->kind = kind; p->n = n; p->howmany = howmany;
    p->in = in; p->out = out;
    p->istride = istride; p->idist = idist; p->ostride = ostride; p->odist = odist;
    p->sign = sign;
    p->tw = make_twiddles(n);
    p->work = (double *)malloc(sizeof(double) * 6 * (size_t)(n > 0 ? n : 1));
    return p;
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride, int odist,
                             int sign, unsigned flags)
{
    (void)rank; (void)inembed; (void)onembed; (void)flags;
    return new_plan(0, n[0], howmany, in, istride, idist, out, ostride, odist, sign);
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags)
{
    (void)rank; (void)inembed; (void)onembed; (void)flags;
    return new_plan(1, n[0], howmany, in, istride, idist, out, ostride, odist, -1);
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags)
{
    (void)rank; (void)inembed; (void)onembed; (void)flags;
    return new_plan(2, n[0], howmany, in, istride, idist, out, ostride, odist, +1);
}

void fftw_execute(const fftw_plan p)
{
    int n = p->n;
    double *a = p->work;           /* 2n */
    double *b = p->work + 2 * n;   /* 2n */
    double *t = p->work + 4 * n;   /* 2n */
    for (int h = 0; h < p->howmany; h++) {
        if (p->kind == 0) {
            const double *in = (const double *)p->in + 2 * (size_t)h * p->idist;
            double *out = (double *)p->out + 2 * (size_t)h * p->odist;
            for (int i = 0; i < n; i++) { a[2 * i] = in[2 * (size_t)i * p->istride]; a[2 * i + 1] = in[2 * (size_t)i * p->istride + 1]; }
            cdft(n, a, b, p->sign, p->tw, t);
            for (int i = 0; i < n; i++) { out[2 * (size_t)i * p->ostride] = b[2 * i]; out[2 * (size_t)i * p->ostride + 1] = b[2 * i + 1]; }
        } else if (p->kind == 1) {
            const double *in = (const double *)p->in + (size_t)h * p->idist;
            double *out = (double *)p->out + 2 * (size_t)h * p->odist;
            for (int i = 0; i < n; i++) { a[2 * i] = in[(size_t)i * p->istride]; a[2 * i + 1] = 0.0; }
            cdft(n, a, b, -1, p->tw, t);
            for (int i = 0; i < n / 2 + 1; i++) { out[2 * (size_t)i * p->ostride] = b[2 * i]; out[2 * (size_t)i * p->ostride + 1] = b[2 * i + 1]; }
        } else {
            const double *in = (const double *)p->in + 2 * (size_t)h * p->idist;
            double *out = (double *)p->out + (size_t)h * p->odist;
            /* rebuild the full Hermitian spectrum; FFTW ignores the imaginary parts of
             * the DC and (even n) Nyquist bins, so do the same */
            for (int i = 0; i < n / 2 + 1; i++) { a[2 * i] = in[2 * (size_t)i * p->istride]; a[2 * i + 1] = in[2 * (size_t)i * p->istride + 1]; }
            a[1] = 0.0;
            if (n % 2 == 0) a[2 * (n / 2) + 1] = 0.0;
            for (int i = n / 2 + 1; i < n; i++) { a[2 * i] = a[2 * (n - i)]; a[2 * i + 1] = -a[2 * (n - i) + 1]; }
            cdft(n, a, b, +1, p->tw, t);
            for (int i = 0; i < n; i++) out[(size_t)i * p->ostride] = b[2 * i];
        }
    }
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    free(p->tw); free(p->work); free(p);
}

double *fftw_alloc_real(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)calloc(n ? n : 1, sizeof(fftw_complex)); }
void fftw_free(void *p) { free(p); }
