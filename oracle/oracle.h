/*
 * Oracle (test infrastructure only; never linked into the product path).
 * FP64 CPU restatement of the reference's demag + field + LLG + RK4/RKDP54 path.
 * Every function names the reference file:line it follows. Arrays are AoS
 * (x, y, z per cell), cells x fastest, then y, then z.
 */
#ifndef BORIS_ORACLE_H
#define BORIS_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MU0 1.256637061435916e-6   /* BorisLib/Funcs_Math_base.h:9 */
#define ORC_GAMMA 2.212761569e5        /* BorisLib/Funcs_Math_base.h:16 */

/* module bits (same values as the product's BM_* flags) */
#define ORC_DEMAG   1
#define ORC_EXCH    2
#define ORC_IDMI    4
#define ORC_ANIUNI  8
#define ORC_ZEEMAN 16

/* ---- Newell tensor ---- */
double orc_newell_f(double x, double y, double z);
double orc_newell_g(double x, double y, double z);
void orc_selfdemag(double hx, double hy, double hz, double *out3);
/* far-field expansion of D = -N at normalised offset (x,y,z) for cell (hx,hy,hz): out6 = xx,yy,zz,xy,xz,yz */
void orc_asymptotic(double hx, double hy, double hz, double x, double y, double z, double *out6);
/* D = -N on the N grid, same layout as the reference (ref_tensor). */
int orc_tensor(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
               double *diag, double *odiag);
/* octant kernel spectra (Nx/2+1)(Ny/2+1)(Nz/2+1) x 3 each; kodiag = (xy, xz, yz) */
int orc_kernels(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
                double *kdiag, double *kodiag);

/* ---- periodic boundary conditions (pbc: images per axis) ---- */
/* D = -N on the N grid with images (DemagTFunc_PBC.cpp); N from orc_pbc_dims */
int orc_tensor_pbc(int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz, const int *pbc,
                   double *diag, double *odiag);
/* octant spectra of a tensor on the N grid, built axis by axis as DemagKernel does */
int orc_kernels_from_tensor(const double *diag, const double *odiag, int nz, int Nx, int Ny, int Nz, double *kdiag,
                            double *kodiag);
/* FFT sizes: n along a periodic axis, 2n otherwise (ConvolutionData.cpp:115-145) */
void orc_pbc_dims(int nx, int ny, int nz, const int *pbc, int *N3);
/* SelfDemag_PBC (DemagTFunc_Self.cpp:57) on normalised cellsizes */
void orc_selfdemag_pbc(double hx, double hy, double hz, const int *n3, const int *pbc, double *out3);
/* DemagTFunc::SelfDemag on the cellsize in metres, with the reference's zero thresholds in f */
void orc_selfdemag_metres(double hx, double hy, double hz, double *out3);
void orc_selfdemag_pbc_metres(double hx, double hy, double hz, const int *n3, const int *pbc, double *out3);

/* ---- demag convolution ---- */
typedef struct orc_demag orc_demag;
orc_demag *orc_demag_create(int nx, int ny, int nz, double hx, double hy, double hz, int Nx, int Ny, int Nz);
/* H = D * M; if add, H += instead of H =. Returns sum_i M_i . Hdemag_i */
double orc_demag_apply(orc_demag *d, const double *M, double *H, int add);
void orc_demag_destroy(orc_demag *d);
/* with PBC images per axis (NULL / zeros: as orc_demag_create with N = 2n) */
orc_demag *orc_demag_create_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc);

/* ---- field terms (add into H) ---- */
void orc_field_exchange(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                        double A, const double *Ms_cell, double *H);
void orc_field_idmi(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                    double A, double D, const double *Ms_cell, double *H);
void orc_field_exchange_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                            double A, const double *Ms_cell, const int *pbc, double *H);
void orc_field_idmi_pbc(int nx, int ny, int nz, double hx, double hy, double hz, const double *M,
                        double A, double D, const double *Ms_cell, const int *pbc, double *H);
void orc_field_aniuni(int n, const double *M, const double *Ms_cell, const double *K1_cell, double K2,
                      const double *ea, double *H);

/* ---- solver over one or more meshes with a common time step ---- */
typedef struct {
    int nx, ny, nz;
    double hx, hy, hz;
    double Ms, A, D, alpha, grel, K1, K2;
    double ea[3];
    const double *Ms_map;  /* per-cell Ms (absolute), or NULL */
    const double *K1_map;  /* per-cell K1 (absolute), or NULL */
    int modules;
    const double *Ha;      /* 3 * nHa piecewise-constant applied-field samples over [0, Ha_tspan) */
    int nHa;
    double Ha_tspan;
    int pbc[3];            /* periodic images per axis (0: none; the sign is the stencils' wrap sign) */
} orc_mesh_desc;

typedef struct {
    long accepted, rejected, evals;
    double time, dT, last_lte;
} orc_stats;

typedef struct orc_ml orc_ml;
typedef struct orc_solver orc_solver;
#define ORC_RK4 0
#define ORC_RKDP54 1
orc_solver *orc_solver_create(int nmesh, const orc_mesh_desc *desc, int eval, double dt, double tol,
                              double dT_incr, double dT_min, double dT_max);
int orc_set_m(orc_solver *s, int mesh, const double *M);
int orc_get_m(orc_solver *s, int mesh, double *M);
/* one multilayered convolution (orc_ml, below) replaces the per-mesh demag of every mesh with
 * ORC_DEMAG; o3 = origin of every solver mesh (3 per mesh) */
int orc_solver_set_multilayer(orc_solver *s, const double *o3, int mode, const int *ncommon);
/* Evaluation speedup (level 0 off, 1 step .. 6 quintic): demag extrapolated from saved fields, per
 * mesh or, with the multilayered convolution, per layer on the common grid. */
int orc_solver_set_evalspeedup(orc_solver *s, int level);
/* the speedup's self term: 0 normalised cellsizes (default), 1 metres as the reference computes it;
   call before orc_solver_set_evalspeedup */
int orc_solver_set_evalspeedup_self(orc_solver *s, int metres);
/* Replace the demag and exchange / iDMI terms of one mesh by a caller's function that adds them
 * into H (3n doubles) for the mesh's M; Zeeman, anisotropy, LLG and the stages stay the solver's.
 * Used to drive the reference's own compiled field code (oracle/ref_harness.cpp) with this
 * integrator for the CPU baseline. fn NULL restores the solver's own terms. */
typedef void (*orc_field_fn)(void *user, const double *M, double *H);
int orc_solver_set_field_hook(orc_solver *s, int mesh, orc_field_fn fn, void *user);
/* effective field at the current M and time; H has 3n doubles */
int orc_compute_heff(orc_solver *s, int mesh, double *H);
/* advance until `steps` more steps are accepted */
int orc_run(orc_solver *s, int steps, orc_stats *st);
/* ODECommon_Base::Get_mxh / Get_dmdt (DiffEq_CommonBase_Get.cpp:7,19): the value of the last step
 * that computed it (0 before any), and a request that the next step computes it: max over cells of
 * |M x Heff| / |M|^2 at the step's first evaluation, and of |M - M_step_start| / (dT GAMMA |M|^2)
 * after its last stage, over the meshes with grel != 0 */
int orc_solver_get_mxh(orc_solver *s, double *v);
int orc_solver_get_dmdt(orc_solver *s, double *v);
void orc_solver_destroy(orc_solver *s);

/* ---- multilayered convolution (SDemag multilayer mode) ----
 * meshes: n3, h3 (cellsize), o3 (origin), 3 per mesh; mode 0: 3D (2D when every mesh is one cell
 * thick or ncommon[2] == 1), 1: 2D, 2: 2D with every z cell layer its own layer; ncommon: NULL for
 * the largest n of the meshes per axis. */
orc_ml *orc_ml_create(int nmesh, const int *n3, const double *h3, const double *o3, int mode, const int *ncommon);
/* layer count, n_common, per layer: mesh, transfer flag, rect (s, e), kernel kind per source
 * (1 self, 2 z-shifted, 3 inverse z-shifted, 4 full complex) */
int orc_ml_info(orc_ml *s, int *L, int *nc3, int *layer_mesh, int *do_transfer, double *rects6, int *kinds);
/* H_demag of every mesh (AoS, meshes concatenated in order) from M of every mesh */
int orc_ml_eval(orc_ml *s, const double *M, double *H);
/* with the evaluation speedup: es_mode 0 plain, 1 compute and save into slot es_slot, 2 extrapolate
 * with the weights es_a of K saved fields (per layer on the common grid) */
int orc_ml_eval_es(orc_ml *s, const double *M, double *H, int es_mode, int es_slot, const double *es_a, int K);
/* one layer's mesh transfer alone: Mc = transfer in of M, Hmesh = transfer out of Hc */
int orc_ml_transfer(orc_ml *s, int layer, const double *M, double *Mc, const double *Hc, double *Hmesh);
void orc_ml_destroy(orc_ml *s);

/* ---- supermesh demag (SDemag with the multilayered convolution off) ----
 * meshes: n3, h3, o3 (3 per mesh); h_request: requested supermesh cellsize; pbc: images of the
 * supermesh convolution (NULL: none) */
typedef struct orc_sm orc_sm;
orc_sm *orc_sm_create(int nmesh, const int *n3, const double *h3, const double *o3, const double *h_request,
                      const int *pbc);
int orc_sm_info(orc_sm *s, int *n3, double *h3, double *rect6, long *nonempty);
/* H (meshes concatenated, AoS) from M; returns the supermesh energy density */
double orc_sm_eval(orc_sm *s, const double *M, double *H);
void orc_sm_destroy(orc_sm *s);
/* one supermesh convolution replaces the per-mesh demag of every mesh with ORC_DEMAG */
int orc_solver_set_supermesh(orc_solver *s, const double *o3, const double *h_request, const int *pbc);

/* ---- discrete adjoint of RK4 (FP64) ----
 * One mesh, modules demag / exchange / uniaxial anisotropy (K2 = 0) / Zeeman (piecewise-constant
 * samples, the sample at each step's start time), per-cell Ms and K1 maps; initial state Ms * m0;
 * loss (1/n) sum_i |M_i(T)/Ms_i - target_i|^2 after `steps` steps of dt. Returns the loss and its
 * gradients with respect to the Ms map, the K1 map and the 3 * nHa field samples (gHa may be NULL). */
int orc_adjoint_rk4(const orc_mesh_desc *d, const double *m0, const double *target, int steps, double dt,
                    double *loss, double *gMs, double *gK1, double *gHa);

/* FP64 in-place complex DFT (fftw_shim.c) */
void bm_oracle_fft(int n, double *data, int sign);

#ifdef __cplusplus
}
#endif
#endif
