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
 *   ref_film_fields_*  a persistent demag + exchange / iDMI field of one film for the CPU baseline:
 *                      Convolution<.,DemagKernel>::Convolute (Boris/Convolution.h:659) added into H,
 *                      then the stencils of ref_exchange / ref_idmi with uniform A, D, Ms over an
 *                      OpenMP loop as Exch_6ngbr_Neu / iDMExchange::UpdateField run theirs
 *                      (Boris/Exchange.cpp:108, Boris/iDMExchange.cpp:97)
 *   ref_tensor_shifted DemagTFunc::Calc{Diag,OffDiag}Tens3D_Shifted (Boris/DemagTFunc_Shifted.cpp:6,...)
 *                      and Calc{Diag,OffDiag}Tens2D_Shifted_Irregular (Boris/DemagTFunc_Irregular.cpp:4,121)
 *   ref_ml_*           the multilayered convolution: one Convolution<., DemagKernelCollection> per
 *                      layer with the rectangle rules of SDemag (Boris/SDemag.cpp:173,215,441), the
 *                      weighted mesh transfer of SDemag_Demag (Boris/SDemag_Demag.cpp:64,349) and the
 *                      evaluation order of SDemag::UpdateField (Boris/SDemag.cpp:786-900)
 *   ref_*_pbc          the same with periodic boundary conditions: DemagTFunc::Calc{Diag,OffDiag}Tens
 *                      {2D,3D}_PBC (Boris/DemagTFunc_PBC.cpp:5,97,185,300), the convolution set up by
 *                      SetDimensions(n, h, true, pbc_images) (Boris/Convolution.h:248,
 *                      Boris/ConvolutionData.cpp:100) as Demag::Initialize does (Boris/Demag.cpp:111),
 *                      the stencils on a VEC_VC with set_pbc (BorisLib/VEC_VC_flags.h:890), and
 *                      DemagTFunc::SelfDemag_PBC (Boris/DemagTFunc_Self.cpp:57)
 *   ref_sm_*           the supermesh demag of SDemag with the multilayered convolution off: the supermesh
 *                      rectangle and cells of SuperMesh::UpdateConfiguration (Boris/SuperMeshControl.cpp:
 *                      22-44), sm_Vals with Initialize_MeshTransfer(M of every mesh, Heff of every mesh,
 *                      MESHTRANSFERTYPE_WEIGHTED), transfer_in, Convolute, transfer_out and the energy of
 *                      SDemag::UpdateField (Boris/SDemag.cpp:566-576,737-760)
 *   ref_ovf2_read      OVF2::Read_OVF2_VEC                  (Boris/OVF2_Handlers.cpp:364)
 *   ref_ovf2_write     OVF2::Write_OVF2_VEC                 (Boris/OVF2_Handlers.cpp:701)
 *   ref_ovf2_load      the loadovf2mag command's data path (Boris/Commands.cpp:5025): read,
 *                      VEC::renormalize when the value is non-zero, VEC::resize(SZ3) to the mesh's
 *                      cell counts (BorisLib/VEC_mng.h:9,118)
 * All arrays are AoS (x,y,z per cell), cells ordered x fastest, then y, then z.
 */
#include "stdafx.h"
#include "DemagTFunc.h"
#include "DemagKernel.h"
#include "DemagKernelCollection.h"
#include "Convolution.h"
#include "OVF2_Handlers.h"

#include <vector>
#include <cstring>

namespace {

struct OracleDemag : public Convolution<OracleDemag, DemagKernel> {
    BError pbc_err;
    OracleDemag(INT3 n_, DBL3 h_) : Convolution<OracleDemag, DemagKernel>(n_, h_) {}
    /* with PBC images, set up as Demag::Initialize does (Boris/Demag.cpp:111) */
    OracleDemag(INT3 n_, DBL3 h_, INT3 pbc) : Convolution<OracleDemag, DemagKernel>()
    {
        pbc_err = SetDimensions(n_, h_, true, pbc);
    }
    BError calc(void) { return Calculate_Demag_Kernels(true); }
    SZ3 get_N(void) const { return N; }
    SZ3 get_n(void) const { return n; }
    bool create_failed(void) { return (bool)Convolution_Error_on_Create() || (bool)pbc_err; }
    double convolute(VEC<DBL3> &In, VEC<DBL3> &Out) { return Convolute(In, Out, true); }
};

/* one layer of the multilayered convolution (the Convolution part of SDemag_Demag) */
struct OracleMLConv : public Convolution<OracleMLConv, DemagKernelCollection> {
    OracleMLConv() : Convolution<OracleMLConv, DemagKernelCollection>() {}
    BError setdims(SZ3 n_, DBL3 h_) { return SetDimensions(n_, h_, false); }
    BError setrects(std::vector<Rect> &rc, Rect r, double hmax, int idx) { return Set_Rect_Collection(rc, r, hmax, idx); }
    BError calc(std::vector<DemagKernelCollection *> &kc) { return Calculate_Demag_Kernels(kc); }
    VEC<ReIm3> *in_space(void) { return Get_Input_Scratch_Space(); }
    void fwd(VEC<DBL3> &In) { ForwardFFT(In); }
    void mult(std::vector<VEC<ReIm3> *> &F) { KernelMultiplication_MultipleInputs(F); }
    double inv(VEC<DBL3> &In, VEC<DBL3> &Out, bool clear) { return InverseFFT(In, Out, clear); }
    SZ3 get_N(void) const { return N; }
    int kernel_kind(int idx)
    {
        std::shared_ptr<KerType> k = Get_Kernel(idx);
        if (!k) return -1;
        if (k->zshifted) return is_inverse_shifted(idx) ? 3 : 2;
        if (k->Kdiag_cmpl.linear_size()) return 4;
        return 1;
    }
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


/* The demag and exchange / iDMI terms of one film, kept across evaluations (kernels built once).
 * modules: bit 1 demag, 2 exchange, 4 iDMI (exchange + DMI). ref_film_fields_add adds the terms
 * into H for M (AoS), with the signature the oracle solver's field hook takes. */
struct ref_film_s {
    OracleDemag *od = nullptr;
    VEC<DBL3> In, Out;
    VEC_VC<DBL3> V;
    int n = 0, modules = 0;
    double A = 0, D = 0, Ms = 1;
};

void *ref_film_fields_create(int nx, int ny, int nz, double hx, double hy, double hz, int modules, double Ms, double A,
                             double D)
{
    ref_film_s *s = new ref_film_s();
    s->n = nx * ny * nz;
    s->modules = modules;
    s->A = A; s->D = D; s->Ms = Ms;
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    if (modules & 1) {
        s->od = new OracleDemag(INT3(nx, ny, nz), DBL3(hx, hy, hz));
        if (s->od->create_failed() || s->od->calc()) { delete s->od; delete s; return nullptr; }
        s->In.resize(DBL3(hx, hy, hz), r);
        s->Out.resize(DBL3(hx, hy, hz), r);
    }
    if (modules & 6) s->V.assign(DBL3(hx, hy, hz), r, DBL3(1, 0, 0));
    return s;
}

void ref_film_fields_add(void *h, const double *M, double *H)
{
    ref_film_s *s = (ref_film_s *)h;
    const int n = s->n;
    if (s->od) {
        memcpy(s->In.data(), M, sizeof(double) * 3 * n);
        s->od->convolute(s->In, s->Out);
        const double *o = (const double *)s->Out.data();
#pragma omp parallel for
        for (long i = 0; i < 3L * n; i++) H[i] += o[i];
    }
    if (!(s->modules & 6)) return;
    VEC_VC<DBL3> &V = s->V;
    memcpy(V.data(), M, sizeof(double) * 3 * n);
    const double Aconst = 2 * s->A / (MU0 * s->Ms * s->Ms);
    if (!(s->modules & 4)) {
#pragma omp parallel for
        for (int i = 0; i < n; i++) {
            DBL3 d = V.delsq_neu(i);
            H[3 * i] += Aconst * d.x; H[3 * i + 1] += Aconst * d.y; H[3 * i + 2] += Aconst * d.z;
        }
        return;
    }
    const double Dconst = -2 * s->D / (MU0 * s->Ms * s->Ms);
    const double rr = s->D / (2 * s->A);
#pragma omp parallel for
    for (int idx = 0; idx < n; idx++) {
        DBL3 HA, HD;
        if (V.is_plane_interior(idx)) {
            HA = Aconst * V.delsq_neu(idx);
            DBL33 Md = V.grad_neu(idx);
            HD = Dconst * DBL3(Md.x.z, Md.y.z, -Md.x.x - Md.y.y);
        }
        else {
            DBL3 bx = rr * DBL3(V[idx].z, 0, -V[idx].x);
            DBL3 by = rr * DBL3(0, V[idx].z, -V[idx].y);
            DBL33 bnd(bx, by, DBL3());
            HA = Aconst * V.delsq_nneu(idx, bnd);
            DBL33 Md = V.grad_nneu(idx, bnd);
            HD = Dconst * DBL3(Md.x.z, Md.y.z, -Md.x.x - Md.y.y);
        }
        H[3 * idx] += HA.x + HD.x; H[3 * idx + 1] += HA.y + HD.y; H[3 * idx + 2] += HA.z + HD.z;
    }
}

/* The demag field alone (H = D * M, H overwritten) of a film object built with the demag bit. */
int ref_film_fields_demag(void *h, const double *M, double *H)
{
    ref_film_s *s = (ref_film_s *)h;
    if (!s->od) return 1;
    memcpy(s->In.data(), M, sizeof(double) * 3 * s->n);
    s->od->convolute(s->In, s->Out);
    memcpy(H, s->Out.data(), sizeof(double) * 3 * s->n);
    return 0;
}

void ref_film_fields_destroy(void *h)
{
    ref_film_s *s = (ref_film_s *)h;
    if (!s) return;
    delete s->od;
    delete s;
}

/* ---- periodic boundary conditions: pbc = images per axis ---- */

/* D = -N on the PBC N grid (N = n along periodic axes, ConvolutionData.cpp:115-145), cellsizes
 * normalised by the largest as DemagKernel passes them; 2D: odiag holds Dxy in component 0 only. */
int ref_tensor_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc, double *diag, double *odiag,
                   int *N3)
{
    DBL3 h(hx, hy, hz);
    double hm = maximum(hx, hy, hz);
    INT3 N(pbc[0] ? nx : 2 * nx, pbc[1] ? ny : 2 * ny, nz > 1 ? (pbc[2] ? nz : 2 * nz) : 1);
    N3[0] = N.x; N3[1] = N.y; N3[2] = N.z;
    if (!diag) return 0;
    DemagTFunc dtf;
    VEC<DBL3> D;
    if (!D.resize(SZ3(N.x, N.y, N.z))) return 1;
    size_t np = (size_t)N.x * N.y * N.z;
    if (nz == 1) {
        if (!dtf.CalcDiagTens2D_PBC(D, N, h / hm, true, ASYMPTOTIC_DISTANCE, pbc[0], pbc[1], pbc[2])) return 2;
        memcpy(diag, D.data(), sizeof(double) * 3 * np);
        std::vector<double> od(np, 0.0);
        if (!dtf.CalcOffDiagTens2D_PBC(od, N, h / hm, true, ASYMPTOTIC_DISTANCE, pbc[0], pbc[1], pbc[2])) return 3;
        for (size_t i = 0; i < np; i++) { odiag[3 * i] = od[i]; odiag[3 * i + 1] = 0; odiag[3 * i + 2] = 0; }
    }
    else {
        if (!dtf.CalcDiagTens3D_PBC(D, N, h / hm, true, ASYMPTOTIC_DISTANCE, pbc[0], pbc[1], pbc[2])) return 2;
        memcpy(diag, D.data(), sizeof(double) * 3 * np);
        if (!dtf.CalcOffDiagTens3D_PBC(D, N, h / hm, true, ASYMPTOTIC_DISTANCE, pbc[0], pbc[1], pbc[2])) return 3;
        memcpy(odiag, D.data(), sizeof(double) * 3 * np);
    }
    return 0;
}

/* Kernel spectra of the PBC convolution as DemagKernel stores them (layouts as ref_kernels). */
int ref_kernels_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc, double *kdiag, double *kodiag)
{
    OracleDemag od(INT3(nx, ny, nz), DBL3(hx, hy, hz), INT3(pbc[0], pbc[1], pbc[2]));
    if (od.create_failed()) return 1;
    if (od.calc()) return 2;
    memcpy(kdiag, od.Kdiag.data(), sizeof(double) * 3 * od.Kdiag.linear_size());
    if (nz == 1) memcpy(kodiag, od.K2D_odiag.data(), sizeof(double) * od.K2D_odiag.size());
    else memcpy(kodiag, od.Kodiag.data(), sizeof(double) * 3 * od.Kodiag.linear_size());
    return 0;
}

/* H = D * M with PBC (Out cleared first); energy as ref_demag_eval. */
int ref_hdemag_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc, const double *M, double *H,
                   double *energy)
{
    OracleDemag od(INT3(nx, ny, nz), DBL3(hx, hy, hz), INT3(pbc[0], pbc[1], pbc[2]));
    if (od.create_failed()) return 1;
    if (od.calc()) return 2;
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    VEC<DBL3> In(DBL3(hx, hy, hz), r), Out(DBL3(hx, hy, hz), r);
    int n = nx * ny * nz;
    memcpy(In.data(), M, sizeof(double) * 3 * n);
    double dot = od.convolute(In, Out);
    memcpy(H, Out.data(), sizeof(double) * 3 * n);
    if (energy) *energy = -MU0 * dot / (2.0 * n);
    return 0;
}

/* exchange (modules 2) or exchange + iDMI (modules 4) field with PBC on the stencils, per-cell A, D, Ms
 * (D ignored for exchange); the formulas of ref_exchange / ref_idmi */
int ref_stencil_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc, int modules, const double *M,
                    const double *A, const double *D, const double *Ms, double *H)
{
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    VEC_VC<DBL3> V(DBL3(hx, hy, hz), r, DBL3(1, 0, 0));
    V.set_pbc(pbc[0], pbc[1], pbc[2]);
    int n = nx * ny * nz;
    memcpy(V.data(), M, sizeof(double) * 3 * n);
    for (int idx = 0; idx < n; idx++) {
        double Aconst = 2 * A[idx] / (MU0 * Ms[idx] * Ms[idx]);
        DBL3 Ht;
        if (modules & 4) {
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
            Ht = HA + HD;
        }
        else Ht = Aconst * V.delsq_neu(idx);
        H[3 * idx] = Ht.x; H[3 * idx + 1] = Ht.y; H[3 * idx + 2] = Ht.z;
    }
    return 0;
}

/* DemagTFunc::SelfDemag_PBC(h, n, pbc) as Demag.cpp:62 and DemagCUDA.cpp:39 call it */
int ref_selfdemag_pbc(double hx, double hy, double hz, int nx, int ny, int nz, const int *pbc, double *out3)
{
    DemagTFunc dtf;
    DBL3 s = dtf.SelfDemag_PBC(DBL3(hx, hy, hz), DBL3(nx, ny, nz), INT3(pbc[0], pbc[1], pbc[2]));
    out3[0] = s.x; out3[1] = s.y; out3[2] = s.z;
    return 0;
}

/* ---- supermesh demag ---- */
struct ref_sm_s {
    std::vector<VEC<DBL3> *> M, Heff;
    VEC<DBL3> sm_Vals;
    OracleDemag *od = nullptr;
    SZ3 n_fm;
    DBL3 h_fm;
    Rect rect;
    int non_empty = 0;
    std::vector<int> ncell;
};

void ref_sm_destroy(void *h)
{
    ref_sm_s *s = (ref_sm_s *)h;
    if (!s) return;
    for (auto p : s->M) delete p;
    for (auto p : s->Heff) delete p;
    delete s->od;
    delete s;
}

void *ref_sm_create(int nmesh, const int *n3, const double *h3, const double *o3, const double *h_request, const int *pbc)
{
    ref_sm_s *s = new ref_sm_s();
    Rect sMeshRect_fm;
    for (int m = 0; m < nmesh; m++) {
        DBL3 h(h3[3 * m], h3[3 * m + 1], h3[3 * m + 2]);
        DBL3 o(o3[3 * m], o3[3 * m + 1], o3[3 * m + 2]);
        Rect r(o, o + (h & DBL3(n3[3 * m], n3[3 * m + 1], n3[3 * m + 2])));
        VEC<DBL3> *M = new VEC<DBL3>(), *H = new VEC<DBL3>();
        M->resize(h, r);
        H->resize(h, r);
        s->M.push_back(M);
        s->Heff.push_back(H);
        s->ncell.push_back(n3[3 * m] * n3[3 * m + 1] * n3[3 * m + 2]);
        sMeshRect_fm += r;
    }
    /* SuperMesh::UpdateConfiguration (SuperMeshControl.cpp:40-44) */
    DBL3 h_fm(h_request[0], h_request[1], h_request[2]);
    s->n_fm = round(sMeshRect_fm / h_fm);
    if (s->n_fm.x == 0) s->n_fm.x = 1;
    if (s->n_fm.y == 0) s->n_fm.y = 1;
    if (s->n_fm.z == 0) s->n_fm.z = 1;
    if (!sMeshRect_fm.IsNull()) h_fm = sMeshRect_fm / s->n_fm;
    s->h_fm = h_fm;
    s->rect = sMeshRect_fm;
    /* SDemag::UpdateConfiguration / Initialize / Initialize_Mesh_Transfer (SDemag.cpp:451-454,566-576,659-661) */
    s->od = new OracleDemag(INT3(s->n_fm.x, s->n_fm.y, s->n_fm.z), h_fm,
                            pbc ? INT3(pbc[0], pbc[1], pbc[2]) : INT3());
    if (s->od->create_failed() || s->od->calc()) { ref_sm_destroy(s); return nullptr; }
    if (!s->sm_Vals.resize(h_fm, sMeshRect_fm)) { ref_sm_destroy(s); return nullptr; }
    if (!s->sm_Vals.Initialize_MeshTransfer(s->M, s->Heff, MESHTRANSFERTYPE_WEIGHTED)) { ref_sm_destroy(s); return nullptr; }
    return s;
}

int ref_sm_info(void *h, int *n3, double *h3, double *rect6)
{
    ref_sm_s *s = (ref_sm_s *)h;
    n3[0] = s->n_fm.x; n3[1] = s->n_fm.y; n3[2] = s->n_fm.z;
    h3[0] = s->h_fm.x; h3[1] = s->h_fm.y; h3[2] = s->h_fm.z;
    rect6[0] = s->rect.s.x; rect6[1] = s->rect.s.y; rect6[2] = s->rect.s.z;
    rect6[3] = s->rect.e.x; rect6[4] = s->rect.e.y; rect6[5] = s->rect.e.z;
    return 0;
}

/* H (meshes concatenated, AoS, overwritten) from M; returns the energy density of SDemag::UpdateField
 * with non_empty_cells counted after the first transfer in (SDemag.cpp:573-576) */
double ref_sm_eval(void *h, const double *M, double *H)
{
    ref_sm_s *s = (ref_sm_s *)h;
    size_t off = 0;
    for (size_t m = 0; m < s->M.size(); m++) {
        memcpy(s->M[m]->data(), M + 3 * off, sizeof(double) * 3 * s->ncell[m]);
        s->Heff[m]->set(DBL3());
        off += s->ncell[m];
    }
    s->sm_Vals.transfer_in();
    if (!s->non_empty) s->non_empty = s->sm_Vals.get_nonempty_cells();
    double energy = s->od->convolute(s->sm_Vals, s->sm_Vals);
    energy *= -MU0 / (2 * s->non_empty);
    s->sm_Vals.transfer_out();
    off = 0;
    for (size_t m = 0; m < s->M.size(); m++) {
        memcpy(H + 3 * off, s->Heff[m]->data(), sizeof(double) * 3 * s->ncell[m]);
        off += s->ncell[m];
    }
    return energy;
}

/* Shifted real-space tensors D = -N on the N grid (AoS, 3 doubles per point).
 * kind 0: Calc{Diag,OffDiag}Tens3D_Shifted(n, N, hs, shift)
 * kind 1: Calc{Diag,OffDiag}Tens2D_Shifted_Irregular(n, N, s = hs, d = hd, shift)
 * Cellsizes and shift are given already normalised (the reference divides them by h_max).
 * asympt is the asymptotic distance in cells (40 is the reference value; 0 uses the exact
 * Newell sums everywhere). */
int ref_tensor_shifted(int kind, int nx, int ny, int nz, int Nx, int Ny, int Nz, const double *hs, const double *hd,
                       const double *shift, int asympt, double *diag, double *odiag)
{
    DemagTFunc dtf;
    VEC<DBL3> D;
    INT3 n(nx, ny, nz), N(Nx, Ny, Nz);
    if (!D.resize(SZ3(Nx, Ny, Nz))) return 1;
    size_t np = (size_t)Nx * Ny * Nz;
    DBL3 s(hs[0], hs[1], hs[2]), d(hd[0], hd[1], hd[2]), sh(shift[0], shift[1], shift[2]);
    if (kind == 0) {
        if (!dtf.CalcDiagTens3D_Shifted(D, n, N, s, sh, true, asympt)) return 2;
        memcpy(diag, D.data(), sizeof(double) * 3 * np);
        if (!dtf.CalcOffDiagTens3D_Shifted(D, n, N, s, sh, true, asympt)) return 3;
        memcpy(odiag, D.data(), sizeof(double) * 3 * np);
    }
    else {
        if (!dtf.CalcDiagTens2D_Shifted_Irregular(D, n, N, s, d, sh, true, asympt)) return 2;
        memcpy(diag, D.data(), sizeof(double) * 3 * np);
        if (!dtf.CalcOffDiagTens2D_Shifted_Irregular(D, n, N, s, d, sh, true, asympt)) return 3;
        memcpy(odiag, D.data(), sizeof(double) * 3 * np);
    }
    return 0;
}

/* ---------------------------------------------------------------- multilayered convolution
 * Meshes are given by n, h and origin o (rect = [o, o + n h]); all are ferromagnetic with
 * demag. force2d follows SDemag::force_2d_convolution (0: 3D unless every mesh is one cell
 * thick, 1: 2D with each mesh one layer, 2: 2D with every z cell layer its own layer);
 * ncommon (optional) is the user's n_common (Set_n_common, SDemag.cpp:362); n_common.z is 1
 * whenever a 2D mode is on (Set_2D_Multilayered_Convolution, SDemag.cpp:341). */
struct ref_ml_s {
    int nmesh = 0, L = 0;
    std::vector<VEC<DBL3> *> M, Heff;
    std::vector<OracleMLConv *> conv;
    std::vector<VEC<DBL3> *> transfer;
    std::vector<int> layer_mesh;
    std::vector<int> do_transfer;
    std::vector<Rect> rects;
    std::vector<VEC<ReIm3> *> F;
    std::vector<DemagKernelCollection *> kc;
    SZ3 n_common;
    double h_max = 0.0;
};

void ref_ml_destroy(void *hp)
{
    ref_ml_s *s = (ref_ml_s *)hp;
    if (!s) return;
    for (auto p : s->conv) delete p;
    for (auto p : s->transfer) delete p;
    for (auto p : s->M) delete p;
    for (auto p : s->Heff) delete p;
    delete s;
}

void *ref_ml_create(int nmesh, const int *n3, const double *h3, const double *o3, int force2d, const int *ncommon)
{
    ref_ml_s *s = new ref_ml_s();
    s->nmesh = nmesh;
    std::vector<Rect> mrect(nmesh);
    std::vector<DBL3> mh(nmesh);
    std::vector<INT3> mn(nmesh);
    for (int m = 0; m < nmesh; m++) {
        mn[m] = INT3(n3[3 * m], n3[3 * m + 1], n3[3 * m + 2]);
        mh[m] = DBL3(h3[3 * m], h3[3 * m + 1], h3[3 * m + 2]);
        DBL3 o(o3[3 * m], o3[3 * m + 1], o3[3 * m + 2]);
        mrect[m] = Rect(o, o + (mh[m] & DBL3(mn[m].x, mn[m].y, mn[m].z)));
        VEC<DBL3> *M = new VEC<DBL3>(), *H = new VEC<DBL3>();
        M->resize(mh[m], mrect[m]);
        H->resize(mh[m], mrect[m]);
        s->M.push_back(M);
        s->Heff.push_back(H);
    }
    // n_common (SDemag::set_default_n_common, SDemag.cpp:173; Set_n_common, :362)
    SZ3 nc(1, 1, 1);
    if (ncommon) {
        nc = SZ3(ncommon[0], ncommon[1], ncommon[2]);
        if (force2d == 0 && nc.z == 1) force2d = 1;
    }
    else {
        bool all2d = true;
        for (int m = 0; m < nmesh; m++) if (mn[m].z != 1) all2d = false;
        for (int m = 0; m < nmesh; m++) {
            if (nc.x < mn[m].x) nc.x = mn[m].x;
            if (nc.y < mn[m].y) nc.y = mn[m].y;
            if (nc.z < mn[m].z) nc.z = mn[m].z;
        }
        if (all2d || force2d) nc.z = 1;
    }
    if (force2d) nc.z = 1;
    s->n_common = nc;
    // layers and the raw rectangle collection (SDemag::set_Rect_collection, SDemag.cpp:215)
    std::vector<Rect> rc;
    for (int m = 0; m < nmesh; m++) {
        int nl = (force2d == 2) ? mn[m].z : 1;
        for (int l = 0; l < nl; l++) {
            rc.push_back(force2d == 2 ? mrect[m].get_zlayer(l, mh[m].z) : mrect[m]);
            s->layer_mesh.push_back(m);
        }
    }
    DBL3 max_sizes;
    double min_x = rc[0].s.x, min_y = rc[0].s.y, min_z = rc[0].s.z;
    for (size_t i = 0; i < rc.size(); i++) {
        if (max_sizes.x < rc[i].size().x) max_sizes.x = rc[i].size().x;
        if (max_sizes.y < rc[i].size().y) max_sizes.y = rc[i].size().y;
        if (max_sizes.z < rc[i].size().z) max_sizes.z = rc[i].size().z;
        if (rc[i].s.x < min_x) min_x = rc[i].s.x;
        if (rc[i].s.y < min_y) min_y = rc[i].s.y;
        if (rc[i].s.z < min_z) min_z = rc[i].s.z;
    }
    for (size_t i = 0; i < rc.size(); i++) {
        if (rc[i].e.x - max_sizes.x < min_x) { rc[i].s.x = min_x; rc[i].e.x = rc[i].s.x + max_sizes.x; }
        else rc[i].s.x = rc[i].e.x - max_sizes.x;
        if (rc[i].e.y - max_sizes.y < min_y) { rc[i].s.y = min_y; rc[i].e.y = rc[i].s.y + max_sizes.y; }
        else rc[i].s.y = rc[i].e.y - max_sizes.y;
        if (nc.z != 1) {
            if (rc[i].e.z - max_sizes.z < min_z) { rc[i].s.z = min_z; rc[i].e.z = rc[i].s.z + max_sizes.z; }
            else rc[i].s.z = rc[i].e.z - max_sizes.z;
        }
    }
    s->rects = rc;
    s->L = (int)rc.size();
    // h_max over the meshes' own cellsizes (SDemag::get_maximum_cellsize, SDemag.cpp:297)
    for (int i = 0; i < s->L; i++) {
        double hm = mh[s->layer_mesh[i]].maxdim();
        if (s->h_max < hm) s->h_max = hm;
    }
    // convolution objects (SDemag::Initialize, SDemag.cpp:456-486)
    for (int i = 0; i < s->L; i++) {
        OracleMLConv *c = new OracleMLConv();
        DBL3 hconv = rc[i] / nc;
        if (c->setdims(nc, hconv)) { s->conv.push_back(c); ref_ml_destroy(s); return nullptr; }
        s->conv.push_back(c);
    }
    for (int i = 0; i < s->L; i++) {
        if (s->conv[i]->setrects(rc, rc[i], s->h_max, i)) { ref_ml_destroy(s); return nullptr; }
        s->kc.push_back(s->conv[i]);
        s->F.push_back(s->conv[i]->in_space());
    }
    // kernels and transfers (SDemag_Demag::Initialize, SDemag_Demag.cpp:306-366)
    for (int i = 0; i < s->L; i++) {
        if (s->conv[i]->calc(s->kc)) { ref_ml_destroy(s); return nullptr; }
        int m = s->layer_mesh[i];
        DBL3 hconv = rc[i] / nc;
        VEC<DBL3> *t = new VEC<DBL3>();
        s->transfer.push_back(t);
        if (rc[i] == mrect[m] && hconv == mh[m]) s->do_transfer.push_back(0);
        else {
            s->do_transfer.push_back(1);
            if (!t->resize(hconv, rc[i])) { ref_ml_destroy(s); return nullptr; }
            if (!t->Initialize_MeshTransfer({s->M[m]}, {s->Heff[m]}, MESHTRANSFERTYPE_WEIGHTED)) { ref_ml_destroy(s); return nullptr; }
        }
    }
    return s;
}

/* layer count, n_common, and per layer: mesh, transfer flag, rect (s, e), kernel kinds per
 * source (1 self/regular real, 2 z-shifted, 3 inverse z-shifted, 4 complex full) */
int ref_ml_info(void *hp, int *L, int *nc3, int *layer_mesh, int *do_transfer, double *rects6, int *kinds)
{
    ref_ml_s *s = (ref_ml_s *)hp;
    if (L) *L = s->L;
    if (nc3) { nc3[0] = s->n_common.x; nc3[1] = s->n_common.y; nc3[2] = s->n_common.z; }
    for (int i = 0; i < s->L; i++) {
        if (layer_mesh) layer_mesh[i] = s->layer_mesh[i];
        if (do_transfer) do_transfer[i] = s->do_transfer[i];
        if (rects6) {
            rects6[6 * i + 0] = s->rects[i].s.x; rects6[6 * i + 1] = s->rects[i].s.y; rects6[6 * i + 2] = s->rects[i].s.z;
            rects6[6 * i + 3] = s->rects[i].e.x; rects6[6 * i + 4] = s->rects[i].e.y; rects6[6 * i + 5] = s->rects[i].e.z;
        }
        if (kinds) for (int j = 0; j < s->L; j++) kinds[i * s->L + j] = s->conv[i]->kernel_kind(j);
    }
    return 0;
}

/* H_demag of every mesh from M of every mesh (AoS, meshes concatenated in order), as
 * SDemag::UpdateField computes it in multilayered mode (no evaluation speedup). */
int ref_ml_eval(void *hp, const double *M, double *H)
{
    ref_ml_s *s = (ref_ml_s *)hp;
    size_t off = 0;
    for (int m = 0; m < s->nmesh; m++) {
        size_t n = s->M[m]->linear_size();
        memcpy(s->M[m]->data(), M + 3 * off, sizeof(double) * 3 * n);
        s->Heff[m]->set(DBL3());
        off += n;
    }
    for (int i = 0; i < s->L; i++) {
        int m = s->layer_mesh[i];
        if (s->do_transfer[i]) {
            s->transfer[i]->transfer_in();
            s->conv[i]->fwd(*s->transfer[i]);
        }
        else s->conv[i]->fwd(*s->M[m]);
    }
    for (int i = s->L - 1; i >= 0; i--) s->conv[i]->mult(s->F);
    for (int i = 0; i < s->L; i++) {
        int m = s->layer_mesh[i];
        if (s->do_transfer[i]) {
            s->conv[i]->inv(*s->transfer[i], *s->transfer[i], true);
            s->transfer[i]->transfer_out();
        }
        else s->conv[i]->inv(*s->M[m], *s->Heff[m], false);
    }
    off = 0;
    for (int m = 0; m < s->nmesh; m++) {
        size_t n = s->Heff[m]->linear_size();
        memcpy(H + 3 * off, s->Heff[m]->data(), sizeof(double) * 3 * n);
        off += n;
    }
    return 0;
}

/* transfer only (tests of the mesh-transfer rules): for layer i, the common-grid input
 * transfer_in() builds from M (AoS, all meshes), and the mesh H that transfer_out() adds from
 * a given common-grid field Hc. */
int ref_ml_transfer(void *hp, int layer, const double *M, double *Mc, const double *Hc, double *Hmesh)
{
    ref_ml_s *s = (ref_ml_s *)hp;
    if (layer < 0 || layer >= s->L || !s->do_transfer[layer]) return 1;
    size_t off = 0;
    for (int m = 0; m < s->nmesh; m++) {
        size_t n = s->M[m]->linear_size();
        memcpy(s->M[m]->data(), M + 3 * off, sizeof(double) * 3 * n);
        s->Heff[m]->set(DBL3());
        off += n;
    }
    VEC<DBL3> &t = *s->transfer[layer];
    t.transfer_in();
    memcpy(Mc, t.data(), sizeof(double) * 3 * t.linear_size());
    memcpy(t.data(), Hc, sizeof(double) * 3 * t.linear_size());
    t.transfer_out();
    int m = s->layer_mesh[layer];
    memcpy(Hmesh, s->Heff[m]->data(), sizeof(double) * 3 * s->Heff[m]->linear_size());
    return 0;
}

/* Header of an OVF 2.0 file (n, h, rect) and, when data != NULL, its values; 0 on success,
 * 1 when the reference's reader returns an error. */
int ref_ovf2_read(const char *path, int *n3, double *h3, double *rect6, double *data)
{
    VEC<DBL3> v;
    OVF2 ovf2;
    BError err = ovf2.Read_OVF2_VEC(std::string(path), v);
    if (err) return 1;
    n3[0] = v.n.x; n3[1] = v.n.y; n3[2] = v.n.z;
    h3[0] = v.h.x; h3[1] = v.h.y; h3[2] = v.h.z;
    rect6[0] = v.rect.s.x; rect6[1] = v.rect.s.y; rect6[2] = v.rect.s.z;
    rect6[3] = v.rect.e.x; rect6[4] = v.rect.e.y; rect6[5] = v.rect.e.z;
    if (data) memcpy(data, v.data(), sizeof(double) * 3 * v.linear_size());
    return 0;
}

int ref_ovf2_write(const char *path, const int *n3, const double *h3, const double *origin3, const double *data,
                   const char *data_type, double norm)
{
    DBL3 h(h3[0], h3[1], h3[2]);
    DBL3 s(origin3[0], origin3[1], origin3[2]);
    Rect r(s, s + DBL3(n3[0] * h3[0], n3[1] * h3[1], n3[2] * h3[2]));
    VEC<DBL3> v(h, r);
    if (v.n.x != n3[0] || v.n.y != n3[1] || v.n.z != n3[2]) return 2;
    memcpy(v.data(), data, sizeof(double) * 3 * v.linear_size());
    OVF2 ovf2;
    BError err = ovf2.Write_OVF2_VEC(std::string(path), v, std::string(data_type), norm);
    return err ? 1 : 0;
}

int ref_ovf2_load(const char *path, double renormalize, const int *dst_n3, double *out)
{
    VEC<DBL3> v;
    OVF2 ovf2;
    BError err = ovf2.Read_OVF2_VEC(std::string(path), v);
    if (err) return 1;
    if (IsNZ(renormalize)) v.renormalize(renormalize);
    if (!v.resize(SZ3(dst_n3[0], dst_n3[1], dst_n3[2]))) return 2;
    memcpy(out, v.data(), sizeof(double) * 3 * v.linear_size());
    return 0;
}

}
