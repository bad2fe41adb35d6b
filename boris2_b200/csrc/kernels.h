// Internal declarations shared by the kernel translation units and the host runtime.
#pragma once
#include "common.cuh"
#include "fft.cuh"

#define BM_FARQ_PER_COMP 94   // 6 + 15 + 28 + 45 monomials for orders 2, 4, 6, 8

// ---------------------------------------------------------------- tensor / kernels
template <typename T>
int build_kernels_device(T *K, int nx, int ny, int nz, int Nx, int Ny, int Nz, double hx, double hy, double hz,
                         const double *farq_dev, const cpx<double> *twx, const cpx<double> *twy,
                         const cpx<double> *twz, cudaStream_t s, const int *pbc = nullptr);
int tensor_octant_device(double *oct_dev, int nx, int ny, int nz, double hx, double hy, double hz, const double *farq_dev,
                         cudaStream_t s, const int *pbc = nullptr);
template <typename T>
int launch_fft_strided(cpx<T> *data, const FFTPlan &P, const cpx<T> *tw, long long es, long long ls, int ninner,
                       long long os, int nouter, bool inv, cudaStream_t s);
// host: far-field polynomial coefficients (6 * BM_FARQ_PER_COMP doubles) for normalised cellsize
void bm_far_coeffs(double hx, double hy, double hz, double *out);

// ---------------------------------------------------------------- gating of kernels by step state
#define BM_GATE_ALWAYS 0
#define BM_GATE_ACCEPTED 1      // skip when the current attempt was rejected
#define BM_GATE_RESTORE 2       // run only when a restore is pending
#define BM_GATE_ES 3            // evaluation speedup (RKDP54): run unless the evaluation extrapolates
#define BM_GATE_ES_ACC 4        // as BM_GATE_ES, and skip when the current attempt was rejected

// ---------------------------------------------------------------- y / z passes
template <typename T>
struct YZArgs {
    cpx<T> *S1;          // [3][nz][ny][LX]
    cpx<T> *S2;          // [3][nz][Ny][LX] (3D only)
    const T *K;          // 6 planes [(kz*Ky1 + ky)*Kx1 + kx]
    const cpx<T> *twy, *twz;
    FFTPlan py, pz;
    int nx, ny, nz, LX, Ny, Nz;
    int W;               // column tile width
    StepState *st;
    int gate;
    int yv;              // 3D y transform: 0 two-level register kernel, 1 radix-16 Stockham (Ny >= 256),
                         // 2 the two-level kernel fed by bulk tensor copies (persistent, pipelined)
    int pf_ahead;        // set by the launchers: blocks of the grid resident at once (0: no look-ahead prefetch)
    int zv;              // 3D z pass: 0 one thread per pencil line, 1 the parity split (two threads per line)
};

// Blocks of a launch resident on the whole GPU at once (occupancy per SM times the SMs), or 0 when
// the occupancy query fails; the look-ahead distance of the y passes' L2 prefetch. The query depends
// only on the kernel, the block size and the dynamic shared memory, so its result is kept per kernel
// for the last block shape asked.
template <typename K> inline int resident_blocks(K kern, int nt, size_t smem)
{
    static int nsm = 0;
    static thread_local const void *last_k = nullptr;
    static thread_local int last_nt = -1, last_res = 0;
    static thread_local size_t last_smem = 0;
    if (last_k == (const void *)kern && last_nt == nt && last_smem == smem) return last_res;
    if (nsm == 0) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
            nsm = v;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
    }
    last_k = (const void *)kern; last_nt = nt; last_smem = smem; last_res = per_sm * nsm;
    return last_res;
}

template <typename T> size_t ymid2d_smem(int Ny, int W)
{
    return (size_t)3 * Ny * W * sizeof(cpx<T>) + (size_t)4 * (Ny / 2 + 1) * (W + 1) * sizeof(T);
}
template <typename T> size_t zmid_smem(int Nz, int W)
{
    return (size_t)6 * Nz * W * sizeof(cpx<T>) + (size_t)6 * (Nz / 2 + 1) * (W + 1) * sizeof(T);
}
template <typename T> size_t zmid_reg_smem(int Nz, int W)
{
    // spectra [3][2][Nz][W], kernel tile + Nyquist column, column-0 outputs [3][2][Nz]
    size_t kb = (size_t)6 * (Nz / 2 + 1) * (W + 1) * sizeof(T);
    kb = (kb + sizeof(cpx<T>) - 1) / sizeof(cpx<T>) * sizeof(cpx<T>);
    return (size_t)6 * Nz * W * sizeof(cpx<T>) + kb + (size_t)6 * Nz * sizeof(cpx<T>);
}
bool zmid_has_reg(int Nz);
bool zmid_has_par(int Nz, int W);   // lengths and tile widths of the parity-split z pass
bool ypass_has_reg(int Ny);
// block-size ceiling of the two-level register y kernel: FP64 lines of 32 values need the registers
// a 256-thread bound allows
template <typename T> struct yreg_maxt { static constexpr int v = sizeof(T) == 8 ? 256 : bm_lb<T>::v; };
bool ypass_has_st(int Ny);            // lengths with the Stockham y transform (radix 16, or radix 4/2/3 for 3 * 2^k)
int ypass_st_threads(int Ny, int W);
int ymid2d_reg_threads(int Ny, int W);   // block size of the register 2D y pass
int ypass_reg_threads(int Ny, int W);
// pipelined 3D y passes with bulk tensor copies (ytma.cu): whether they apply, and the launches
// (-1 when they do not apply)
template <typename T> bool ypass_tma_fits(const YZArgs<T> &a);
template <typename T, bool INV> int launch_ypass_tma(const YZArgs<T> &a, cudaStream_t s);
// fused y -> z -> y pass of a 3D mesh in one thread-block-cluster kernel (yzy.cu): 0 when it
// applies to the mesh (sizes, shared memory, the device's cluster occupancy)
template <typename T> int yzy_available(const YZArgs<T> &a);
template <typename T> int launch_yzy(const YZArgs<T> &a, cudaStream_t s);
template <typename T> int launch_ymid2d(const YZArgs<T> &a, cudaStream_t s);
template <typename T> int launch_yfwd(const YZArgs<T> &a, cudaStream_t s);
template <typename T> int launch_zmid(const YZArgs<T> &a, cudaStream_t s);
template <typename T> int launch_yinv(const YZArgs<T> &a, cudaStream_t s);

// ---------------------------------------------------------------- fused x / field / LLG stage kernel
#define BM_MODE_STAGE 0     // fields, LLG, stage update, forward x-FFT of the new M
#define BM_MODE_HEFF 1      // fields only, write Heff to Hout
#define BM_MODE_LTE 2       // fields, LLG, RKDP54 4th-order prediction error (FP64 max), FSAL rhs
#define BM_MODE_UPDATE 3    // no fields: M_out = M_base + dT * sum c_i ev_i, forward x-FFT

#define BM_LAST_NONE 0
#define BM_LAST_FINISH 1    // time += dT, accepted++
#define BM_LAST_CONTROL 2   // RKDP54 step control on the reduced lte
#define BM_LAST_RESTORED 3  // clear need_restore

template <typename T>
struct StageArgs {
    int nx, ny, nz, LX, Nx;
    double hx, hy, hz;
    cpx<T> *S1;
    const cpx<T> *twx;   // length LX
    const cpx<T> *twx2;  // length Nx (R2C split twiddles)
    FFTPlan px;
    int rpb;             // rows per block
    T scale;             // 2 / (Nx Ny Nz)
    int modules;
    T Ms, A, D, alpha, grel, K1, K2;
    T ea[3];
    const T *Ms_map, *K1_map;
    const double *Ha;
    int nHa;
    double Ha_tspan;
    StepState *st;
    const T *Min, *Mbase;
    T *Mout, *copy_to, *ev_out, *Hout;
    const T *Hd;         // demag field per cell from a multilayered convolution (added when set)
    T *Hsave, *Ysave;    // adjoint stage cache: the field used by LLG, the update before renormalisation
    int nev;
    const T *ev[6];
    double cev[6];
    double crhs;
    int renorm, mode, do_xfwd, last_kind, gate;
    int diag;            // BM_DIAG_* bits: this launch evaluates mxh / dmdt when requested, and publishes
    int lte_embedded;    // LTE mode: the 5th-order solution recomputed in FP64 from the base and cev5 (nev 5)
    double cev5[6];      // LTE mode with lte_embedded: 5th-order weights of the same stage rhs as cev
    long long n;         // cells
    int staged;          // prefetch the per-cell input rows into shared memory (register kernel)
    int xv;              // register x transform: 0 two-level P x Q, 1 radix-8 Stockham at 64 (FP32) registers
    // derived per-launch constants (products replace per-cell divisions)
    T hh[3], ih[3], ih2[3];   // h, 1 / h, 1 / h^2
    T iMs;                    // 1 / Ms (uniform Ms)
    T rrD;                    // D / (2 A): iDMI boundary condition slope factor (0 when A = 0)
    T exA, exD;               // 2 A / mu0, -2 D / mu0 (times 1 / Ms^2 per cell)
    T two_mu0;                // 2 / mu0
    T llg_pre;                // -gamma grel / (1 + alpha^2)
    int pbc[3];               // per axis: 0 no wrap, +1 / -1 periodic neighbour with that sign (mesh PBC)
    // evaluation speedup formed in the stage kernel: es_fold 0 off, 1 RK4 (extrapolate once es_K are
    // saved, weights from the saved times), 2 RKDP54 (extrapolate when the decision says so, its
    // weights); the S1 row becomes es_cs[c] S1 + sum_k a_k G_k before the inverse x transform
    int es_fold;
    const cpx<T> *esG;        // saved slots [slot][c][row][LX]
    double es_cs[3];
    double es_ceval;          // evaluation time as a fraction of dT
};

// fills the derived constants of a StageArgs from its material and cellsize fields
template <typename T> inline void stage_derive(StageArgs<T> &a)
{
    const double h[3] = {a.hx, a.hy, a.hz};
    for (int i = 0; i < 3; i++) {
        a.hh[i] = (T)h[i];
        a.ih[i] = (T)(1.0 / h[i]);
        a.ih2[i] = (T)(1.0 / (h[i] * h[i]));
    }
    const double Ms = (double)a.Ms, A = (double)a.A, D = (double)a.D, al = (double)a.alpha;
    a.iMs = (T)(Ms != 0.0 ? 1.0 / Ms : 0.0);
    a.rrD = (T)(A != 0.0 ? D / (2.0 * A) : 0.0);
    a.exA = (T)(2.0 * A / BM_MU0);
    a.exD = (T)(-2.0 * D / BM_MU0);
    a.two_mu0 = (T)(2.0 / BM_MU0);
    a.llg_pre = (T)(-BM_GAMMA * (double)a.grel / (1.0 + al * al));
}

// Shared-memory row staging of the register stage kernel: per block row, kr rows of nx values:
// 3*ns rows of M (slot 0 the row itself, 1/2 the y-1/y+1 rows, 3/4 the z-1/z+1 rows, each x,y,z),
// 3 rows of the update base (when it differs from M), 3 per earlier stage evaluation, then the
// Ms map row and the K1 map row when present and used.
struct StageLayout {
    int ns, mb, ms, k1, kr;
};
template <typename T> __host__ __device__ inline StageLayout stage_layout(const StageArgs<T> &a)
{
    StageLayout L;
    const bool fields = a.mode != BM_MODE_UPDATE;
    L.ns = (fields && (a.modules & (BM_MOD_EXCH | BM_MOD_IDMI))) ? 5 : 1;
    L.mb = (a.mode != BM_MODE_HEFF && a.Mbase && a.Mbase != a.Min) ? 1 : 0;
    L.ms = a.Ms_map ? 1 : 0;
    L.k1 = (a.K1_map && fields && (a.modules & BM_MOD_ANIUNI)) ? 1 : 0;
    L.kr = 3 * L.ns + 3 * L.mb + 3 * (a.mode == BM_MODE_HEFF ? 0 : a.nev) + L.ms + L.k1;
    return L;
}

template <typename T> int launch_stage(const StageArgs<T> &a, cudaStream_t s);

// ---------------------------------------------------------------- many meshes per launch
// Work items (mesh, tile index); the argument blocks and the work list live in device memory.
// Tile index: stage = row block; ymid2d = column tile; y passes = column tile + tiles * (z + nz *
// component); z pass = column tile + tiles * ky.
#define BM_BATCH_YMID2D 1
#define BM_BATCH_YFWD 2
#define BM_BATCH_ZMID 3
#define BM_BATCH_YINV 4
// register-kernel buckets: every mesh of the launch has the same transform length (key)
#define BM_BATCH_ZMID_REG 5   // key Nz
#define BM_BATCH_YFWD_REG 6   // key Ny
#define BM_BATCH_YINV_REG 7   // key Ny
#define BM_BATCH_YMID2D_REG 8 // key Ny
#define BM_BATCH_YFWD_ST 9    // key Ny (Stockham y transform)
#define BM_BATCH_YINV_ST 10   // key Ny
template <typename T>
int launch_yz_batch(int kind, int key, const YZArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem,
                    cudaStream_t s);
// key 0: generic-length stage kernel; key LX: the radix-8 register kernel of that length
// the plain stage update of the RK stages (SPEC 1 of the radix-16 and batched register stage kernels):
// stage mode, exchange and demag on, the rhs and new M written, the new M's x transform; no saved
// fields or states, no external field, no copy, no staging, no folded extrapolation
template <typename T> inline bool stage_plain(const StageArgs<T> &a)
{
    return a.mode == BM_MODE_STAGE && !a.staged && !a.es_fold && !a.Hd && !a.Hsave && !a.Ysave && !a.copy_to && a.ev_out &&
           a.Mout && a.do_xfwd && (a.modules & BM_MOD_DEMAG) && (a.modules & (BM_MOD_EXCH | BM_MOD_IDMI));
}
// the plain RKDP54 error estimate (SPEC 2): the rhs written, no new M, no forward transform, fields on
template <typename T> inline bool stage_lte_plain(const StageArgs<T> &a)
{
    return a.mode == BM_MODE_LTE && !a.staged && !a.es_fold && !a.Hd && !a.Hsave && !a.Ysave && !a.copy_to && a.ev_out &&
           !a.Mout && !a.do_xfwd && (a.modules & BM_MOD_DEMAG) && (a.modules & (BM_MOD_EXCH | BM_MOD_IDMI));
}
// the plain advance of the base state (SPEC 3): no fields, the base copied, the new M written and
// transformed, no rhs output, no renormalisation
template <typename T> inline bool stage_adv_plain(const StageArgs<T> &a)
{
    return a.mode == BM_MODE_UPDATE && !a.staged && !a.es_fold && !a.Hd && !a.Hsave && !a.Ysave && a.copy_to && a.Mout &&
           a.do_xfwd && !a.ev_out && !a.renorm;
}
// plain: every argument block of the launch satisfies stage_plain (FP32 takes the SPEC 1 kernels)
template <typename T>
int launch_stage_batch(int key, const StageArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s,
                       int plain = 0);
int stage_reg_q(int LX, int xv = 0);   // threads per x line of the register stage kernel, variant xv (0: generic kernel)
int launch_scalar_reset(StepState *st, cudaStream_t s);

// ---------------------------------------------------------------- discrete adjoint of RK4
// Per-cell material of the adjoint kernels (single mesh): Ms and K1 maps or constants.
template <typename T>
struct AdjArgs {
    int nx, ny, nz;
    long long n;
    T hx, hy, hz;
    const T *Ms_map, *K1_map;
    T Ms, K1, A, alpha, grel;
    T ea[3];
    int modules;
    int pbc[3];   // per axis: 0 no wrap, +1 / -1 periodic neighbour with that sign
};
template <typename T>
int launch_adj_loss(const AdjArgs<T> &a, const T *M, const double *target, T *lam, double *gMs, double *loss, cudaStream_t s);
template <typename T>
int launch_adj_renorm(const AdjArgs<T> &a, T *lam, const T *Y, T *lamY, T *mu, double dt, double *gMs, cudaStream_t s);
template <typename T>
int launch_adj_vjp_a(const AdjArgs<T> &a, const T *X, const T *H, const T *mu, T *gH, T *gXd, T *w, double *gMs, double *gK1,
                     double *gHa3, cudaStream_t s);
template <typename T>
int launch_adj_vjp_c(const AdjArgs<T> &a, const T *gXd, const T *w, const T *gD, const T *lamY, T *lam, T *mu, double cY,
                     double cX, int write_mu, cudaStream_t s);
template <typename T>
int launch_adj_m0(const AdjArgs<T> &a, const T *M0, const T *lam, double *gMs, cudaStream_t s);

// ---------------------------------------------------------------- evaluation speedup (RK4)
// Lagrange weights of the saved fields at this evaluation: RK4 (sel 0) from the saved times at
// time + c_eval dT, RKDP54 (sel 1) as k_es_decide recorded them
template <typename T>
__device__ __forceinline__ void bm_es_weights(const StepState *st, int sel, double c_eval, T a[6])
{
    const int K = st->es_K;
    const double t = st->time + c_eval * st->dT;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double w = 0.0;
        if (sel) w = st->es_a[k];
        else if (k < K) {
            w = 1.0;
            for (int j = 0; j < K; j++)
                if (j != k) w *= (t - st->es_t[j]) / (st->es_t[k] - st->es_t[j]);
        }
        a[k] = (T)w;
    }
}
// the weight of saved field k alone (as bm_es_weights)
__device__ __forceinline__ double bm_es_weight(const StepState *st, int sel, double c_eval, int k)
{
    if (sel) return st->es_a[k];
    const int K = st->es_K;
    const double t = st->time + c_eval * st->dT;
    double w = 1.0;
    for (int j = 0; j < K; j++)
        if (j != k) w *= (t - st->es_t[j]) / (st->es_t[k] - st->es_t[j]);
    return w;
}
// whether the register stage kernels (which can form the extrapolated spectrum themselves) serve
// this x length and variant
bool stage_reg_path(int LX, int xv);
void self_demag_host(double hx, double hy, double hz, double out3[3]);   // -N of one cell (tensor.cu)
// -N of one cell as the reference's evaluation speedup computes it, on the cellsize in metres (tensor.cu)
void self_demag_metres_host(double hx, double hy, double hz, double out3[3]);
// -N of one cell plus the far field of its PBC images (tensor.cu); n = cells, img = images per axis;
// metres: the cell's own term as self_demag_metres_host
void self_demag_pbc_host(double hx, double hy, double hz, const int n[3], const int img[3], double out3[3],
                         int metres = 0);
// Demag extrapolation in the x-spectrum domain S1[c][z][y][kx] (plane = nz ny LX complex values per
// component). G holds es_K slots of 3 planes: the saved field minus its self term. cs[c] is the
// self-demag coefficient (-N_c) times Ny Nz, the factor between the x-spectrum of M the stage kernel
// writes and the x-spectrum of H the y inverse pass leaves.
// sel 0: RK4 (the first evaluation of a step saves, the rest extrapolate once es_K are saved);
// sel 1: RKDP54, each kernel acting on the decision k_es_decide recorded for the evaluation
template <typename T>
int launch_es_pre(const cpx<T> *S1, cpx<T> *G, long long plane, const double *cs, const StepState *st, cudaStream_t s,
                  int sel = 0);
template <typename T>
int launch_es_post(const cpx<T> *S1, cpx<T> *G, long long plane, const StepState *st, cudaStream_t s, int sel = 0);
int launch_es_commit(StepState *st, cudaStream_t s, int sel = 0);
int launch_es_decide(StepState *st, int eval, double c_eval, cudaStream_t s);
// all meshes of a batched context in one launch: a device table of one EsMesh per mesh with demag
struct EsMesh {
    void *S1, *G;
    long long plane;
    double cs[3];
};
template <typename T>
int launch_es_pre_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, cudaStream_t s, int sel = 0);
template <typename T>
int launch_es_post_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, cudaStream_t s, int sel = 0);
template <typename T>
int launch_es_extrap_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, double c_eval,
                           cudaStream_t s, int sel = 0);
template <typename T>
int launch_es_extrap(cpx<T> *S1, const cpx<T> *G, long long plane, const double *cs, const StepState *st, double c_eval,
                     cudaStream_t s, int sel = 0);
