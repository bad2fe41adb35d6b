/*
 * Oracle test infrastructure: a thin extern "C" harness over the reference's
 * own CPU demag/stencil sources, compiled in place from the reference tree by
 * oracle/Makefile into oracle/_ref/libborisref.so. Used only by tests and by the
 * CPU-baseline leg of bench.py, never by the product path.
 *
 * Entry points and the reference code each one runs:
 *   ref_selfdemag      DemagTFunc::SelfDemag                (Boris/DemagTFunc_Self.cpp:6)
 *   ref_tensor         DemagTFunc::CalcDiagTens{2D,3D},
 *                      CalcOffDiagTens{2D,3D}               (Boris/DemagTFunc.cpp:21,95,172,237)
 *   ref_kernels        DemagKernel::Calculate_Demag_Kernels (Boris/DemagKernel.cpp:171,317)
 *   ref_hdemag         Convolution<.,DemagKernel>::Convolute (Boris/Convolution.h:142,262,659)
 *   ref_exchange       VEC_VC<DBL3>::delsq_neu              (BorisLib/VEC_VC_Del.h:10)
 *                      with the field formula of Exch_6ngbr_Neu::UpdateField (Boris/Exchange.cpp:108)
 *   ref_idmi           VEC_VC<DBL3>::delsq_nneu/grad_nneu/grad_neu (BorisLib/VEC_VC_Del.h:141,
 *                      BorisLib/VEC_VC_Grad.h:10,139) with the field formula of
 *                      iDMExchange::UpdateField (Boris/iDMExchange.cpp:97)
 * All arrays are AoS (x,y,z per cell), cells ordered x fastest, then y, then z.
 */
#include "stdafx.h"
#include "DemagTFunc.h"
#include "DemagKernel.h"
#include "Convolution.h"

#include <vector>
#include <cstring>

namespace {

struct OracleDemag : public Convolution<OracleDemag, DemagKernel> {
    OracleDemag(INT3 n_, DBL3 h_) : Convolution<OracleDemag, DemagKernel>(n_, h_) {}
    BError calc(void) { return Calculate_Demag_Kernels(true); }
    SZ3 get_N(void) const { return N; }
    SZ3 get_n(void) const { return n; }
    bool create_failed(void) { return (bool)Convolution_Error_on_Create(); }
    double convolute(VEC<DBL3> &In, VEC<DBL3> &Out) { return Convolute(In, Out, true); }
};

}

extern "C" {

int ref_selfdemag(double hx, double hy, double hz, double *out3)
{
    DemagTFunc dtf;
    DBL3 s = dtf.SelfDemag(DBL3(hx, hy, hz), true);
    out3[0] = s.x; out3[1] = s.y; out3[2] = s.z;
    return 0;
}

/* Real-space tensor D = -N on the N grid (AoS doubles, 3 per point), as the reference
 * builds it before the FFT. 2D (nz == 1): odiag holds Dxy in component 0 only. */
int ref_tensor(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
               double *diag, double *odiag)
{
    DBL3 h(hx, hy, hz);
    double hm = maximum(hx, hy, hz);
    DemagTFunc dtf;
    VEC<DBL3> D;
    INT3 n(nx, ny, nz), N(Nx, Ny, Nz);
    if (!D.resize(SZ3(Nx, Ny, Nz))) return 1;
    size_t np = (size_t)Nx * Ny * Nz;
    if (nz == 1) {
        if (!dtf.CalcDiagTens2D(D, n, N, h / hm, true)) return 2;
        memcpy(diag, D.data(), sizeof(double) * 3 * np);
        std::vector<double> od(np, 0.0);
        if (!dtf.CalcOffDiagTens2D(od, n, N, h / hm)) return 3;
        for (size_t i = 0; i < np; i++) { odiag[3 * i] = od[i]; odiag[3 * i + 1] = 0; odiag[3 * i + 2] = 0; }
    }
    else {
        if (!dtf.CalcDiagTens3D(D, n, N, h / hm, true)) return 2;
        memcpy(diag, D.data(), sizeof(double) * 3 * np);
        if (!dtf.CalcOffDiagTens3D(D, n, N, h / hm)) return 3;
        memcpy(odiag, D.data(), sizeof(double) * 3 * np);
    }
    return 0;
}

/* FFT sizes the reference CPU build uses for this mesh (ConvolutionData.cpp:115-145). */
int ref_fft_dims(int nx, int ny, int nz, int *N3)
{
    N3[0] = 2 * nx; N3[1] = 2 * ny; N3[2] = (nz > 1) ? 2 * nz : 1;
    return 0;
}

/* Kernel spectra exactly as DemagKernel stores them.
 * 3D: kdiag, kodiag each (Nx/2+1)(Ny/2+1)(Nz/2+1) x 3 doubles.
 * 2D: kdiag (Nx/2+1)(Ny/2+1) x 3 doubles, kodiag (Nx/2+1)(Ny/2+1) doubles (Kxy). */
int ref_kernels(int nx, int ny, int nz, double hx, double hy, double hz, double *kdiag, double *kodiag)
{
    OracleDemag od(INT3(nx, ny, nz), DBL3(hx, hy, hz));
    if (od.create_failed()) return 1;
    if (od.calc()) return 2;
    if (nz == 1) {
        memcpy(kdiag, od.Kdiag.data(), sizeof(double) * 3 * od.Kdiag.linear_size());
        memcpy(kodiag, od.K2D_odiag.data(), sizeof(double) * od.K2D_odiag.size());
    }
    else {
        memcpy(kdiag, od.Kdiag.data(), sizeof(double) * 3 * od.Kdiag.linear_size());
        memcpy(kodiag, od.Kodiag.data(), sizeof(double) * 3 * od.Kodiag.linear_size());
    }
    return 0;
}

/* Persistent demag convolution object so repeated evaluations (CPU baseline timing)
 * do not rebuild kernels. */
struct ref_demag_s {
    OracleDemag *od;
    VEC<DBL3> In, Out;
    int n;
};

void *ref_demag_create(int nx, int ny, int nz, double hx, double hy, double hz)
{
    ref_demag_s *s = new ref_demag_s();
    s->od = new OracleDemag(INT3(nx, ny, nz), DBL3(hx, hy, hz));
    if (s->od->create_failed() || s->od->calc()) { delete s->od; delete s; return nullptr; }
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    s->In.resize(DBL3(hx, hy, hz), r);
    s->Out.resize(DBL3(hx, hy, hz), r);
    s->n = nx * ny * nz;
    return s;
}

/* H = D * M (Out cleared first); returns demag energy density -mu0/(2 n) sum M.H
 * (Demag.cpp:176-195), which is what Demag::UpdateField reports. */
double ref_demag_eval(void *h, const double *M, double *H)
{
    ref_demag_s *s = (ref_demag_s *)h;
    memcpy(s->In.data(), M, sizeof(double) * 3 * s->n);
    double dot = s->od->convolute(s->In, s->Out);
    memcpy(H, s->Out.data(), sizeof(double) * 3 * s->n);
    return -MU0 * dot / (2.0 * s->n);
}

void ref_demag_destroy(void *h)
{
    ref_demag_s *s = (ref_demag_s *)h;
    if (!s) return;
    delete s->od;
    delete s;
}

int ref_hdemag(int nx, int ny, int nz, double hx, double hy, double hz, const double *M, double *H, double *energy)
{
    void *s = ref_demag_create(nx, ny, nz, hx, hy, hz);
    if (!s) return 1;
    double e = ref_demag_eval(s, M, H);
    if (energy) *energy = e;
    ref_demag_destroy(s);
    return 0;
}

/* Exchange field 2A/(mu0 Ms^2) * delsq_neu(M) with per-cell A and Ms (Exchange.cpp:108-145, T = 0). */
int ref_exchange(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                 const double *A, const double *Ms, double *H)
{
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    VEC_VC<DBL3> V(DBL3(hx, hy, hz), r, DBL3(1, 0, 0));
    int n = nx * ny * nz;
    memcpy(V.data(), M, sizeof(double) * 3 * n);
    for (int i = 0; i < n; i++) {
        DBL3 d = V.delsq_neu(i);
        double c = 2 * A[i] / (MU0 * Ms[i] * Ms[i]);
        H[3 * i] = c * d.x; H[3 * i + 1] = c * d.y; H[3 * i + 2] = c * d.z;
    }
    return 0;
}

/* Exchange + interfacial DMI field of iDMExchange::UpdateField (iDMExchange.cpp:97-176, T = 0),
 * per-cell A, D and Ms. */
int ref_idmi(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
             const double *A, const double *D, const double *Ms, double *H)
{
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    VEC_VC<DBL3> V(DBL3(hx, hy, hz), r, DBL3(1, 0, 0));
    int n = nx * ny * nz;
    memcpy(V.data(), M, sizeof(double) * 3 * n);
    for (int idx = 0; idx < n; idx++) {
        double Aconst = 2 * A[idx] / (MU0 * Ms[idx] * Ms[idx]);
        double Dconst = -2 * D[idx] / (MU0 * Ms[idx] * Ms[idx]);
        DBL3 HA, HD;
        if (V.is_plane_interior(idx)) {
            HA = Aconst * V.delsq_neu(idx);
            DBL33 Md = V.grad_neu(idx);
            HD = Dconst * DBL3(Md.x.z, Md.y.z, -Md.x.x - Md.y.y);
        }
        else {
            DBL3 bx = (D[idx] / (2 * A[idx])) * DBL3(V[idx].z, 0, -V[idx].x);
            DBL3 by = (D[idx] / (2 * A[idx])) * DBL3(0, V[idx].z, -V[idx].y);
            DBL33 bnd(bx, by, DBL3());
            HA = Aconst * V.delsq_nneu(idx, bnd);
            DBL33 Md = V.grad_nneu(idx, bnd);
            HD = Dconst * DBL3(Md.x.z, Md.y.z, -Md.x.x - Md.y.y);
        }
        DBL3 Ht = HA + HD;
        H[3 * idx] = Ht.x; H[3 * idx + 1] = Ht.y; H[3 * idx + 2] = Ht.z;
    }
    return 0;
}

}
