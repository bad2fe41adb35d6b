// Host runtime behind the C ABI (include/boris_b200.h): contexts, meshes, device buffers,
// kernel-spectrum build, step sequencing and CUDA-graph replay.
//
// Step structure (per mesh, per effective-field evaluation):
//   [stage kernel of the previous evaluation wrote S1 = x-FFT(M_stage)]
//   2D: ymid2d            3D: yfwd -> zmid -> yinv
//   stage kernel: inverse x FFT -> Heff -> LLG -> stage update -> x-FFT of the new M
// RK4 (Boris/DiffEqFM_Evals_RK4.cpp): 4 evaluations per step, the last one finishes the step.
// RKDP54 (Boris/DiffEqFM_Evals_RKDP54.cpp, DiffEq_CommonBase_Iterate.cpp:1214): one attempt =
//   [restore if the previous attempt was rejected] -> evaluation 0 (FSAL rhs, FP64 error norm,
//   step controller in the last block) -> advance -> evaluations 1..5 (skipped on reject).
// The step controller runs on the device, so a bm_run of many steps needs no host round trip
// except one read of the accepted-step counter per batch of graph launches.
#include "../../include/boris_b200.h"
#include "kernels.h"
#include "ml.h"
#include "util.h"
#include <vector>
#include <map>
#include <string>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(BM_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CKL(rc, what)                                                                             \
    do {                                                                                          \
        int r_ = (rc);                                                                            \
        if (r_) return fail(BM_ECUDA, std::string(what) + " launch failed (" + std::to_string(r_) + "): " + \
                                          cudaGetErrorString(cudaGetLastError()));                \
    } while (0)

// smallest 2^p or 3*2^p >= n
int nice_size(int n)
{
    int best = 1;
    while (best < n) best *= 2;
    for (int t = 3; t < best; t *= 2)
        if (t >= n) { best = t; break; }
    return best;
}

struct Mesh {
    int nx = 0, ny = 0, nz = 0;
    double h[3] = {0, 0, 0}, o[3] = {0, 0, 0};
    double Ms = 8e5, A = 1.3e-11, D = 0.0, alpha = 0.5, grel = 1.0, K1 = 0.0, K2 = 0.0;
    double ea[3] = {0, 0, 1};
    std::vector<double> Ms_map, K1_map;
    int modules = BM_DEMAG | BM_EXCH | BM_ZEEMAN;
    std::vector<double> Ha{0.0, 0.0, 0.0};
    double Ha_tspan = 0.0;
    std::vector<double> M0;     // host copy of M until the device is ready
    int pbc[3] = {0, 0, 0};     // periodic images per axis (0: none; the sign is the stencil's wrap sign)
    // derived
    long long n = 0;
    int Nx = 1, Ny = 1, Nz = 1, LX = 1;
    FFTPlan px, py, pz;
    int W2 = 1, Wy = 1, Wz = 1, rpb = 1, staged = 0, xv = 0, yv = 0;
    int yzy = 0;                // 3D: the fused y -> z -> y cluster pass instead of three launches
    int zv = 0;                 // 3D z pass: 1 the parity split (two threads per pencil line)
    // device (element type depends on the context precision)
    void *buf[4] = {nullptr, nullptr, nullptr, nullptr};   // A (M), P (sM1), B, C
    void *ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    void *S1 = nullptr, *S2 = nullptr, *K = nullptr;
    void *twx = nullptr, *twx2 = nullptr, *twy = nullptr, *twz = nullptr;
    void *Msd = nullptr, *K1d = nullptr, *Hout = nullptr;
    void *G = nullptr;          // evaluation speedup: es_level saved spectra (3 planes each)
    double es_cs[3] = {0, 0, 0};
    double *Had = nullptr, *stage64 = nullptr;
    int nHa = 1;
    // multilayered convolution: 0 not in one, 1 its grid is the common grid (spectra in S1/S2),
    // 2 mesh transfer to and from the common grid (demag field arrives in Hd)
    int ml_role = 0;
    void *Hd = nullptr;         // demag field of the mesh (role 2)
    void *Hc = nullptr;         // common-grid demag fields of the mesh's layers, [layer][c][cell]
    int *out_ptr = nullptr, *out_idx = nullptr;
    void *out_w = nullptr;
};

// multilayered convolution state of a context
struct MLRun {
    MLGeom g;
    std::vector<int> mesh_of;       // multilayer mesh -> context mesh
    std::vector<Mesh> grids;        // per layer: the common grid of a transfer layer
    std::vector<int> direct;        // per layer: context mesh whose grid is the common grid, or -1
    std::vector<int> block;         // per layer: block of the layer in its mesh's Hc
    std::vector<int *> in_ptr, in_idx;
    std::vector<void *> in_w;
    void *K = nullptr;
    void *twz = nullptr;
    int W = 8;
    long long ncc = 0;
    // supermesh demag (BM_ML_SUPERMESH): one demag grid over the meshes' bounding box
    bool sm = false;
    SMGeom smg;
    Mesh smgrid;
    std::vector<int *> sm_in_ptr, sm_in_idx;   // per mesh of mesh_of
    std::vector<void *> sm_in_w;
};

// Graphs of a context with many meshes per launch are built in two passes: the first collects
// every batched launch's argument blocks and work list (host), they are uploaded in one buffer,
// the second (under stream capture) launches them from the uploaded copies.
struct BatchRec {
    int kind;             // 0 stage, else BM_BATCH_*
    int key;              // register-kernel length of the launch (0: generic-length kernel)
    size_t args_off, work_off;
    int nwork, nt;
    size_t smem;
    int plain = 0;        // stage launch: every argument block is a plain stage update (stage_plain)
};
struct BatchPlan {
    bool collect = false;
    std::vector<unsigned char> hbuf;
    std::vector<BatchRec> recs;
    size_t next = 0;
    void *dbuf = nullptr;
};

// Per-launch timing of an eagerly enqueued step (bm_time_step): an event after every launch, the
// launch's kernel kind and its algorithmic bytes.
#define BM_TK_STAGE 0
#define BM_TK_YFWD 1
#define BM_TK_ZMID 2
#define BM_TK_YINV 3
#define BM_TK_YMID2D 4
#define BM_TK_OTHER 5
#define BM_TK_YZY 6
#define BM_TK_COUNT 8
struct LaunchTimer {
    std::vector<cudaEvent_t> ev;   // ev[0] before the first launch, ev[i + 1] after launch i
    std::vector<int> kind;
    std::vector<double> bytes;
};

}  // namespace

struct bm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int precision = BM_MIXED;
    int eval = BM_RK4;
    double dt = 1e-13;
    double tol = 1e-4, dT_incr = 2.0, dT_min = 1e-15, dT_max = 3e-12;
    std::vector<Mesh> meshes;
    StepState *st = nullptr;
    bool ready = false;
    bool s1_dirty = true;
    bool state_dirty = true;   // host-side step parameters need upload
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_eval = -1;
    bool eval_chosen = false;
    bool autotune = true;
    int kernels_per_step = 0;
    double *farq = nullptr;
    StepState host_st;
    bool batched = false;       // many meshes per launch (work lists) instead of one launch per mesh
    BatchPlan bp;
    int ml_mode = -1;           // -1 off; 0 3D, 1 2D, 2 2D layered, 3 supermesh
    double sm_h[3] = {5e-9, 5e-9, 5e-9};   // requested supermesh cellsize (the reference's default h_fm)
    int sm_pbc[3] = {0, 0, 0};  // PBC images of the supermesh convolution
    bool ml_nc_set = false;
    int ml_nc[3] = {1, 1, 1};
    MLRun *ml = nullptr;
    int es_level = 0;           // evaluation speedup level (0 off, 1..6)
    int es_phase = 0;           // step being captured: 1 while fields are still being saved, 2 extrapolating
    cudaGraphExec_t gexec_es = nullptr;   // evaluation speedup: the extrapolating step (gexec saves)
    cudaGraph_t graph_es = nullptr;
    EsMesh *es_tab = nullptr;   // batched meshes: device table for the one-launch extrapolation kernels
    int es_fold_pending = 0;    // the evaluation being captured extrapolates in its stage kernels (1 RK4, 2 RKDP54)
    int es_self_metres = 0;     // the speedup's self term on the cellsize in metres, as the reference computes it
    double es_fold_ceval = 0.0; // its time as a fraction of dT
    int es_nmesh = 0;
    long long es_max_plane = 0;
    bool es_reset = true;       // clear the saved fields at the next state upload
    LaunchTimer *lt = nullptr;  // set while bm_time_step enqueues its eager steps
    size_t mem_limit = 0;       // bm_set_memory_limit (0: the free device memory is the limit)
};

namespace {

template <typename T> size_t esz() { return sizeof(T); }

void free_mesh(Mesh &m)
{
    for (auto &p : m.buf) { if (p) cudaFree(p); p = nullptr; }
    for (auto &p : m.ev) { if (p) cudaFree(p); p = nullptr; }
    void **ps[] = {&m.S1, &m.S2, &m.K, &m.twx, &m.twx2, &m.twy, &m.twz, &m.Msd, &m.K1d, &m.Hout, &m.G};
    for (auto pp : ps) { if (*pp) cudaFree(*pp); *pp = nullptr; }
    if (m.Had) cudaFree(m.Had);
    m.Had = nullptr;
    if (m.stage64) cudaFree(m.stage64);
    m.stage64 = nullptr;
    void **pm[] = {&m.Hd, &m.Hc, &m.out_w};
    for (auto pp : pm) { if (*pp) cudaFree(*pp); *pp = nullptr; }
    if (m.out_ptr) cudaFree(m.out_ptr);
    if (m.out_idx) cudaFree(m.out_idx);
    m.out_ptr = m.out_idx = nullptr;
    m.ml_role = 0;
}

void free_ml(bm_ctx *c)
{
    if (!c->ml) return;
    MLRun &r = *c->ml;
    for (auto &g : r.grids) free_mesh(g);
    for (auto p : r.in_ptr) if (p) cudaFree(p);
    for (auto p : r.in_idx) if (p) cudaFree(p);
    for (auto p : r.in_w) if (p) cudaFree(p);
    for (auto p : r.sm_in_ptr) if (p) cudaFree(p);
    for (auto p : r.sm_in_idx) if (p) cudaFree(p);
    for (auto p : r.sm_in_w) if (p) cudaFree(p);
    free_mesh(r.smgrid);
    if (r.K) cudaFree(r.K);
    if (r.twz) cudaFree(r.twz);
    delete c->ml;
    c->ml = nullptr;
}

void drop_graph(bm_ctx *c)
{
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->gexec_es) cudaGraphExecDestroy(c->gexec_es);
    if (c->graph_es) cudaGraphDestroy(c->graph_es);
    c->gexec = nullptr;
    c->graph = nullptr;
    c->gexec_es = nullptr;
    c->graph_es = nullptr;
    if (c->es_tab) cudaFree(c->es_tab);
    c->es_tab = nullptr;
    c->es_nmesh = 0;
    c->es_max_plane = 0;
    c->graph_eval = -1;
    if (c->bp.dbuf) cudaFree(c->bp.dbuf);
    c->bp = BatchPlan();
}

void unprepare(bm_ctx *c)
{
    if (!c->ready) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    drop_graph(c);
    // keep the current M on the host
    for (auto &m : c->meshes) {
        if (m.buf[0]) {
            std::vector<double> tmp(3 * (size_t)m.n);
            double *d = nullptr;
            if (cudaMalloc(&d, sizeof(double) * 3 * m.n) == cudaSuccess) {
                if (c->precision == BM_FP64) launch_planes_to_aos<double>(d, (double *)m.buf[0], m.n, c->stream);
                else launch_planes_to_aos<float>(d, (float *)m.buf[0], m.n, c->stream);
                cudaMemcpyAsync(tmp.data(), d, sizeof(double) * 3 * m.n, cudaMemcpyDeviceToHost, c->stream);
                cudaStreamSynchronize(c->stream);
                cudaFree(d);
                m.M0 = tmp;
            }
        }
        free_mesh(m);
    }
    free_ml(c);
    c->ready = false;
    c->s1_dirty = true;
}

template <typename T>
int upload_table(void **dst, int L, bool fp64_only, cudaStream_t s)
{
    std::vector<double> tw(2 * (size_t)L);
    for (int m = 0; m < L; m++) {
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)L;
        tw[2 * m] = (double)cosl(a);
        tw[2 * m + 1] = (double)-sinl(a);
    }
    size_t bytes = (fp64_only ? sizeof(double) : sizeof(T)) * 2 * (size_t)L;
    if (cudaMalloc(dst, bytes) != cudaSuccess) return fail(BM_ENOMEM, "twiddle table allocation failed");
    if (fp64_only || sizeof(T) == sizeof(double)) {
        if (cudaMemcpyAsync(*dst, tw.data(), bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return fail(BM_ECUDA, "twiddle upload");
    } else {
        std::vector<float> f(2 * (size_t)L);
        for (size_t i = 0; i < f.size(); i++) f[i] = (float)tw[i];
        if (cudaMemcpyAsync(*dst, f.data(), bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return fail(BM_ECUDA, "twiddle upload");
        cudaStreamSynchronize(s);
    }
    cudaStreamSynchronize(s);
    return 0;
}

int pow2_floor(int v)
{
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

template <typename T>
void choose_tiles(Mesh &m)
{
    const size_t cs = sizeof(cpx<T>);
    const int lim = bm_lb<T>::v;
    // 2D y pass: 3 components per block, transformed one after another; keep the grid at
    // least one wave of the GPU where the mesh allows it
    {
        int W = 16;
        while (W > 1 && (ymid2d_smem<T>(m.Ny, W) > 110 * 1024 || W * m.py.tpl > lim || (m.LX / W) < 148)) W /= 2;
        if (W > m.LX) W = pow2_floor(m.LX);
        m.W2 = W;
    }
    // 3D y passes: small tiles so several blocks share an SM and overlap load and compute
    {
        int W = 8;
        if (ypass_has_reg(m.Ny))
            while (W > 1 && ((size_t)m.Ny * W * cs > 100 * 1024 || ypass_reg_threads(m.Ny, W) > yreg_maxt<T>::v)) W /= 2;
        else
            while (W > 1 && ((size_t)m.Ny * W * cs > 100 * 1024 || W * m.py.tpl > lim)) W /= 2;
        if (W > m.LX) W = pow2_floor(m.LX);
        m.Wy = W;
    }
    // 3D z pass: register transforms (6 lines per column) or the generic shared-memory path
    {
        int W = 32;
        if (zmid_has_reg(m.Nz))
            while (W > 1 && (zmid_reg_smem<T>(m.Nz, W) > 72 * 1024 || 6 * W > lim)) W /= 2;
        else
            while (W > 1 && (zmid_smem<T>(m.Nz, W) > 72 * 1024 || 2 * W * m.pz.tpl > lim)) W /= 2;
        if (W > m.LX) W = pow2_floor(m.LX);
        m.Wz = W;
    }
    // stage kernel rows per block
    {
        int tpl = stage_reg_q(m.LX, m.xv) ? stage_reg_q(m.LX, m.xv) : m.px.tpl;
        int rpb = lim / (3 * tpl);
        if (rpb < 1) rpb = 1;
        while (rpb > 1 && ((3 * rpb * tpl + 31) & ~31) > lim) rpb--;
        while (rpb > 1 && (size_t)3 * rpb * padded_len(m.LX) * cs > 64 * 1024) rpb--;
        int rows = m.ny * m.nz;
        if (rpb > rows) rpb = rows;
        m.rpb = rpb;
    }
}

template <typename T>
int prepare_mesh(bm_ctx *c, Mesh &m)
{
    cudaStream_t s = c->stream;
    m.n = (long long)m.nx * m.ny * m.nz;
    m.Nx = 2 * nice_size(m.nx);
    m.Ny = 2 * nice_size(m.ny);
    m.Nz = m.nz > 1 ? 2 * nice_size(m.nz) : 1;
    m.LX = m.Nx / 2;
    if (!bm_make_plan(m.LX, m.px) || !bm_make_plan(m.Ny, m.py) || !bm_make_plan(m.Nz, m.pz))
        return fail(BM_EUNSUPPORTED, "unsupported FFT size");
    choose_tiles<T>(m);
    size_t v3 = sizeof(T) * 3 * (size_t)m.n;
    int nbuf = (c->eval == BM_RKDP54) ? 4 : 4;
    int nev = (c->eval == BM_RKDP54) ? 6 : 3;
    for (int i = 0; i < nbuf; i++) {
        if (cudaMalloc(&m.buf[i], v3) != cudaSuccess) return fail(BM_ENOMEM, "M buffers");
        cudaMemsetAsync(m.buf[i], 0, v3, s);
    }
    for (int i = 0; i < nev; i++) {
        if (cudaMalloc(&m.ev[i], v3) != cudaSuccess) return fail(BM_ENOMEM, "stage buffers");
        cudaMemsetAsync(m.ev[i], 0, v3, s);
    }
    if (cudaMalloc(&m.Hout, v3) != cudaSuccess) return fail(BM_ENOMEM, "H buffer");
    if (cudaMalloc(&m.stage64, sizeof(double) * 3 * m.n) != cudaSuccess) return fail(BM_ENOMEM, "staging buffer");
    if (m.ml_role == 2) {
        if (cudaMalloc(&m.Hd, v3) != cudaSuccess) return fail(BM_ENOMEM, "multilayer demag field");
        cudaMemsetAsync(m.Hd, 0, v3, s);
    }
    if ((m.modules & BM_DEMAG) && m.ml_role != 2) {
        size_t s1 = sizeof(cpx<T>) * 3 * (size_t)m.nz * m.ny * m.LX;
        if (cudaMalloc(&m.S1, s1) != cudaSuccess) return fail(BM_ENOMEM, "S1");
        cudaMemsetAsync(m.S1, 0, s1, s);
        if (c->es_level > 0) {
            if (cudaMalloc(&m.G, s1 * c->es_level) != cudaSuccess) return fail(BM_ENOMEM, "evaluation speedup slots");
            cudaMemsetAsync(m.G, 0, s1 * c->es_level, s);
            double S[3];
            const int nc3[3] = {m.nx, m.ny, m.nz};
            self_demag_pbc_host(m.h[0], m.h[1], m.h[2], nc3, m.pbc, S, c->es_self_metres);
            for (int k = 0; k < 3; k++) m.es_cs[k] = S[k] * (double)m.Ny * (double)m.Nz;
        }
        if (m.nz > 1 || m.ml_role == 1) {
            size_t s2 = sizeof(cpx<T>) * 3 * (size_t)m.nz * m.Ny * m.LX;
            if (cudaMalloc(&m.S2, s2) != cudaSuccess) return fail(BM_ENOMEM, "S2");
            cudaMemsetAsync(m.S2, 0, s2, s);
        }
        int rc;
        if ((rc = upload_table<T>(&m.twx, m.LX, false, s))) return rc;
        if ((rc = upload_table<T>(&m.twx2, m.Nx, false, s))) return rc;
        if ((rc = upload_table<T>(&m.twy, m.Ny, false, s))) return rc;
        if ((rc = upload_table<T>(&m.twz, m.Nz, false, s))) return rc;
    }
    if ((m.modules & BM_DEMAG) && m.ml_role == 0) {
        int rc;
        size_t nk = (size_t)(m.Nx / 2 + 1) * (m.Ny / 2 + 1) * (m.Nz / 2 + 1);
        if (cudaMalloc(&m.K, sizeof(T) * 6 * nk) != cudaSuccess) return fail(BM_ENOMEM, "kernel spectra");
        void *tx = nullptr, *ty = nullptr, *tz = nullptr;
        if ((rc = upload_table<double>(&tx, m.Nx, true, s))) return rc;
        if ((rc = upload_table<double>(&ty, m.Ny, true, s))) return rc;
        if ((rc = upload_table<double>(&tz, m.Nz, true, s))) return rc;
        double hm = std::fmax(m.h[0], std::fmax(m.h[1], m.h[2]));
        std::vector<double> fq(6 * BM_FARQ_PER_COMP);
        bm_far_coeffs(m.h[0] / hm, m.h[1] / hm, m.h[2] / hm, fq.data());
        CK(cudaMemcpyAsync(c->farq, fq.data(), sizeof(double) * fq.size(), cudaMemcpyHostToDevice, s));
        rc = build_kernels_device<T>((T *)m.K, m.nx, m.ny, m.nz, m.Nx, m.Ny, m.Nz, m.h[0], m.h[1], m.h[2], c->farq,
                                     (const cpx<double> *)tx, (const cpx<double> *)ty, (const cpx<double> *)tz, s, m.pbc);
        cudaFree(tx); cudaFree(ty); cudaFree(tz);
        if (rc) return fail(BM_ECUDA, "kernel build failed (" + std::to_string(rc) + ")");
    }
    // material maps
    if (!m.Ms_map.empty()) {
        if (cudaMalloc(&m.Msd, sizeof(T) * m.n) != cudaSuccess) return fail(BM_ENOMEM, "Ms map");
        CK(cudaMemcpyAsync(m.stage64, m.Ms_map.data(), sizeof(double) * m.n, cudaMemcpyHostToDevice, s));
        CKL(launch_convert<T>((T *)m.Msd, m.stage64, m.n, s), "convert");
    }
    if (!m.K1_map.empty()) {
        if (cudaMalloc(&m.K1d, sizeof(T) * m.n) != cudaSuccess) return fail(BM_ENOMEM, "K1 map");
        CK(cudaStreamSynchronize(s));
        CK(cudaMemcpyAsync(m.stage64, m.K1_map.data(), sizeof(double) * m.n, cudaMemcpyHostToDevice, s));
        CKL(launch_convert<T>((T *)m.K1d, m.stage64, m.n, s), "convert");
    }
    m.nHa = (int)(m.Ha.size() / 3);
    if (cudaMalloc(&m.Had, sizeof(double) * m.Ha.size()) != cudaSuccess) return fail(BM_ENOMEM, "Ha");
    CK(cudaMemcpyAsync(m.Had, m.Ha.data(), sizeof(double) * m.Ha.size(), cudaMemcpyHostToDevice, s));
    // initial M
    CK(cudaStreamSynchronize(s));
    if (m.M0.size() == 3 * (size_t)m.n) {
        CK(cudaMemcpyAsync(m.stage64, m.M0.data(), sizeof(double) * 3 * m.n, cudaMemcpyHostToDevice, s));
        CKL(launch_aos_to_planes<T>((T *)m.buf[0], m.stage64, m.n, s), "aos_to_planes");
    }
    CK(cudaStreamSynchronize(s));
    return 0;
}

int upload_state(bm_ctx *c)
{
    StepState &h = c->host_st;
    h.dT = c->dt;
    h.tol = c->tol;
    h.dT_incr = c->dT_incr;
    h.dT_min = c->dT_min;
    h.dT_max = c->dT_max;
    h.eval_order = (c->eval == BM_RKDP54) ? 5 : 4;
    h.es_K = c->es_level;
    if (c->es_reset) {
        h.es_saved = 0;
        for (int k = 0; k < 6; k++) h.es_t[k] = 0.0;
        h.es_available = 1;
        h.es_mode = 0;
        c->es_reset = false;
    }
    h.reject_flag = 0;
    h.need_restore = 0;
    h.lte_bits = 0;
    h.blocks_done = 0;
    h.mxh_acc = 0;
    h.dmdt_acc = 0;
    CK(cudaMemcpyAsync(c->st, &h, sizeof(StepState), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->state_dirty = false;
    return 0;
}

int read_state(bm_ctx *c)
{
    CK(cudaMemcpyAsync(&c->host_st, c->st, sizeof(StepState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

// ------------------------------------------------------------------ autotuner
// Times candidate tile shapes of each pass on the mesh's own buffers (CUDA events, a few
// launches each) and keeps the fastest. Runs once per geometry at setup; the spectrum
// buffers it scribbles on are re-primed before the first step.
template <typename T> YZArgs<T> yz_args(bm_ctx *c, Mesh &m, int gate);
template <typename T> StageArgs<T> stage_args(bm_ctx *c, Mesh &m);

template <typename F>
float time_launches(cudaStream_t s, F launch, int reps)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (launch()) { cudaEventDestroy(e0); cudaEventDestroy(e1); cudaGetLastError(); return 1e30f; }
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; r++) launch();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess) return 1e30f;
    return ms / reps;
}

// 3D y passes of one grid: transform variant (two-level register / radix-16 Stockham) x column
// tile width, timed as a forward + inverse pair on the grid's own spectra
template <typename T>
void tune_ypass(bm_ctx *c, Mesh &m)
{
    cudaStream_t s = c->stream;
    const int lim = bm_lb<T>::v;
    const size_t cs = sizeof(cpx<T>);
    YZArgs<T> a = yz_args<T>(c, m, BM_GATE_ALWAYS);
    float best = 1e30f; int bw = m.Wy, byv = m.yv;
    const char *tma = getenv("BM_Y_TMA");   // "0": leave the pipelined bulk-copy y passes out of the tuning
    for (int yv = 0; yv <= 2; yv++)
        for (int W = 1; W <= 32 && W <= m.LX; W *= 2) {
            if ((size_t)m.Ny * W * cs > 200 * 1024) continue;
            a.W = W;
            if (yv == 2) {
                if ((tma && tma[0] == '0') || !ypass_tma_fits<T>(a)) continue;
            } else if (yv == 1) {
                if (!ypass_has_st(m.Ny)) continue;
                const int nt = ypass_st_threads(m.Ny, W);
                if (nt > lim || nt % 32) continue;
            } else if (ypass_has_reg(m.Ny) ? ypass_reg_threads(m.Ny, W) > yreg_maxt<T>::v : W * m.py.tpl > lim) {
                continue;
            }
            a.W = W;
            a.yv = yv;
            // the better of two timings of 5 launches each (single short timings mis-ranked the
            // Stockham and generic kernels of large multilayer grids)
            float t = 1e30f;
            for (int trial = 0; trial < 2; trial++)
                t = std::min(t, time_launches(s, [&]() { return launch_yfwd<T>(a, s); }, 5) +
                                    time_launches(s, [&]() { return launch_yinv<T>(a, s); }, 5));
            if (t < best) { best = t; bw = W; byv = yv; }
        }
    m.Wy = bw;
    m.yv = byv;
}

template <typename T> T *B(Mesh &m, int i);

// x transforms of a multilayer common grid (x forward after the transfer in, x inverse before the
// transfer out): register variant x rows per block, timed on the grid's own buffers
template <typename T>
int tune_grid_x(bm_ctx *c, Mesh &G)
{
    cudaStream_t s = c->stream;
    const int lim = bm_lb<T>::v;
    const size_t cs = sizeof(cpx<T>);
    if (!stage_reg_q(G.LX, 1)) return 0;
    T *tmp = nullptr;
    if (cudaMalloc(&tmp, sizeof(T) * 3 * G.n) != cudaSuccess) return 0;   // keep the heuristic choice
    StageArgs<T> f = stage_args<T>(c, G);
    f.st = nullptr;
    f.mode = BM_MODE_UPDATE;
    f.Min = B<T>(G, 0); f.Mbase = B<T>(G, 0);
    f.nev = 0;
    StageArgs<T> h = stage_args<T>(c, G);
    h.st = nullptr;
    h.mode = BM_MODE_HEFF;
    h.modules = BM_DEMAG;
    h.do_xfwd = 0;
    h.Min = B<T>(G, 0);
    h.Hout = tmp;
    float best = 1e30f; int br = G.rpb, bx = G.xv;
    const int rows = G.ny * G.nz;
    for (int xv = 0; xv <= (stage_reg_q(G.LX, 2) ? (sizeof(T) == 4 ? 3 : 2) : 1); xv++)
        for (int rpb = 1; rpb <= 16 && rpb <= rows; rpb++) {
            const int tpl = stage_reg_q(G.LX, xv) ? stage_reg_q(G.LX, xv) : G.px.tpl;
            if (((3 * rpb * tpl + 31) & ~31) > lim) break;
            if ((size_t)3 * rpb * padded_len(G.LX) * cs > 200 * 1024) break;
            f.rpb = h.rpb = rpb;
            f.xv = h.xv = xv;
            f.staged = h.staged = 0;
            float t = time_launches(s, [&]() { return launch_stage<T>(f, s); }, 3) +
                      time_launches(s, [&]() { return launch_stage<T>(h, s); }, 3);
            if (t < best) { best = t; br = rpb; bx = xv; }
        }
    G.rpb = br;
    G.xv = bx;
    G.staged = 0;
    cudaStreamSynchronize(s);
    cudaFree(tmp);
    cudaGetLastError();
    return 0;
}

template <typename T>
void tune_grid_yz(bm_ctx *c, Mesh &m)
{
    cudaStream_t s = c->stream;
    const int lim = bm_lb<T>::v;
    const int reps = 3;
    {
        YZArgs<T> a = yz_args<T>(c, m, BM_GATE_ALWAYS);
        if (m.nz == 1) {
            float best = 1e30f; int bw = m.W2;
            for (int W = 1; W <= 16 && W <= m.LX; W *= 2) {
                if (ymid2d_smem<T>(m.Ny, W) > 200 * 1024 || W * m.py.tpl > lim) continue;
                a.W = W;
                float t = time_launches(s, [&]() { return launch_ymid2d<T>(a, s); }, reps);
                if (t < best) { best = t; bw = W; }
            }
            m.W2 = bw;
        } else {
            tune_ypass<T>(c, m);
            a.yv = m.yv;
            float best = 1e30f; int bw = m.Wz, bzv = 0;
            for (int W = 4; W <= 128 && W <= m.LX; W *= 2) {
                if (zmid_has_reg(m.Nz) ? (zmid_reg_smem<T>(m.Nz, W) > 200 * 1024 || 6 * W > lim)
                                       : (zmid_smem<T>(m.Nz, W) > 200 * 1024 || 2 * W * m.pz.tpl > lim)) continue;
                a.W = W;
                // one thread per pencil line, and the parity split where it applies
                for (int zv = 0; zv <= (zmid_has_par(m.Nz, W) ? 1 : 0); zv++) {
                    a.zv = zv;
                    float t = time_launches(s, [&]() { return launch_zmid<T>(a, s); }, reps);
                    if (t < best) { best = t; bw = W; bzv = zv; }
                }
            }
            a.zv = 0;
            m.Wz = bw;
            m.zv = bzv;
            // the fused cluster pass, where it applies, against the three tuned launches
            // (BM_YZY=0 keeps the three launches)
            const char *sz = getenv("BM_YZY");
            m.yzy = 0;
            YZArgs<T> f = yz_args<T>(c, m, BM_GATE_ALWAYS);
            if (!(sz && sz[0] == '0') && yzy_available<T>(f) == 0) {
                YZArgs<T> y = f, z = f;
                y.W = m.Wy; z.W = m.Wz;
                const float t3 = time_launches(s, [&]() { return launch_yfwd<T>(y, s); }, reps) +
                                 time_launches(s, [&]() { return launch_zmid<T>(z, s); }, reps) +
                                 time_launches(s, [&]() { return launch_yinv<T>(y, s); }, reps);
                const float tf = time_launches(s, [&]() { return launch_yzy<T>(f, s); }, reps);
                if (tf < t3) m.yzy = 1;
            }
        }
    }
}

template <typename T>
int autotune_mesh(bm_ctx *c, Mesh &m)
{
    cudaStream_t s = c->stream;
    const int lim = bm_lb<T>::v;
    const size_t cs = sizeof(cpx<T>);
    const int reps = 3;
    if ((m.modules & BM_DEMAG) && m.ml_role == 1) tune_ypass<T>(c, m);   // its y passes feed the multilayer z pass
    if ((m.modules & BM_DEMAG) && m.ml_role == 0) tune_grid_yz<T>(c, m);
    // stage kernel: rows per block
    T *tmp = nullptr;
    if (cudaMalloc(&tmp, sizeof(T) * 6 * m.n) != cudaSuccess) return 0;   // keep heuristic choice
    {
        StageArgs<T> a = stage_args<T>(c, m);
        a.st = nullptr;   // no step-state side effects while tuning
        a.mode = BM_MODE_STAGE;
        a.Min = (const T *)m.buf[0];
        a.Mbase = (const T *)m.buf[0];
        a.nev = 2;
        a.ev[0] = (const T *)m.buf[0]; a.ev[1] = (const T *)m.buf[0];
        a.ev_out = tmp;
        a.Mout = tmp + 3 * m.n;
        float best = 1e30f; int br = m.rpb, bs = 0, bx = 0;
        int rows = m.ny * m.nz;
        const bool reg = stage_reg_q(m.LX, 1) != 0;
        // x-transform variant x rows per block x (per-cell rows prefetched to shared memory or
        // read from global); variants and staging apply to the register kernels only
        for (int xv = 0; xv <= (stage_reg_q(m.LX, 2) ? (sizeof(T) == 4 ? 3 : 2) : reg ? 1 : 0); xv++)
            for (int stg = 0; stg <= (reg ? 1 : 0); stg++)
                for (int rpb = 1; rpb <= 16 && rpb <= rows; rpb++) {
                    const int tpl = stage_reg_q(m.LX, xv) ? stage_reg_q(m.LX, xv) : m.px.tpl;
                    if (((3 * rpb * tpl + 31) & ~31) > lim) break;
                    if ((size_t)3 * rpb * padded_len(m.LX) * cs > 200 * 1024) break;
                    a.rpb = rpb;
                    a.staged = stg;
                    a.xv = xv;
                    float t = time_launches(s, [&]() { return launch_stage<T>(a, s); }, reps);
                    if (t < best) { best = t; br = rpb; bs = stg; bx = xv; }
                }
        m.rpb = br;
        m.staged = bs;
        m.xv = bx;
    }
    cudaStreamSynchronize(s);
    cudaFree(tmp);
    cudaGetLastError();
    return 0;
}

// The periodic tensor build evaluates (octant points) x (image terms) tensor values; bound it so a
// set-up cannot hold the device for minutes.
int pbc_work_check(const int nc[3], const int pbc[3])
{
    double work = 1.0;
    for (int a = 0; a < 3; a++) {
        const int X = std::abs(pbc[a]);
        work *= X ? (double)(nc[a] / 2 + 1) * (2.0 * X + 2.0) : (double)nc[a];
    }
    if (work > 1e10)
        return fail(BM_EUNSUPPORTED, "periodic tensor build of " + std::to_string(work) +
                                         " tensor evaluations is above the limit of 1e10 (fewer images or cells)");
    return 0;
}

// ------------------------------------------------------------------ multilayered convolution setup
// Geometry and roles (host only, before the meshes allocate): every mesh with the demag module
// takes part; a layer whose grid is its mesh's grid keeps its spectra in the mesh's S1/S2,
// every other layer gets a common-grid buffer set and the weighted transfers.
int ml_plan(bm_ctx *c)
{
    if (c->ml_mode < 0) return 0;
    std::vector<MLMeshIn> in;
    std::vector<int> of;
    for (int i = 0; i < (int)c->meshes.size(); i++) {
        Mesh &m = c->meshes[i];
        if (!(m.modules & BM_DEMAG)) continue;
        MLMeshIn x;
        x.n[0] = m.nx; x.n[1] = m.ny; x.n[2] = m.nz;
        for (int a = 0; a < 3; a++) { x.h[a] = m.h[a]; x.o[a] = m.o[a]; }
        in.push_back(x);
        of.push_back(i);
    }
    if (in.empty()) return 0;
    MLRun *r = new MLRun();
    c->ml = r;
    r->mesh_of = of;
    std::string err;
    if (c->ml_mode == BM_ML_SUPERMESH) {
        r->sm = true;
        if (sm_build_geometry(in, c->sm_h, r->smg, err)) return fail(BM_EINVAL, err);
        const int *n = r->smg.n;
        if (nice_size(n[0]) > 4096 || nice_size(n[1]) > 4096 || nice_size(n[2]) > 2048)
            return fail(BM_EUNSUPPORTED, "supermesh: cell counts above the supported FFT size");
        for (int k : of) c->meshes[k].ml_role = 2;
        return pbc_work_check(n, c->sm_pbc);
    }
    if (ml_build_geometry(in, c->ml_mode, c->ml_nc_set ? c->ml_nc : nullptr, r->g, err)) return fail(BM_EINVAL, err);
    if (!zmid_ml_supported(r->g.N[2])) return fail(BM_EUNSUPPORTED, "multilayer: common n.z above 32 is not supported");
    for (int l = 0; l < r->g.L; l++) c->meshes[of[r->g.layers[l].mesh]].ml_role = r->g.layers[l].transfer ? 2 : 1;
    return 0;
}

template <typename T>
int prepare_grid(bm_ctx *c, Mesh &g)
{
    cudaStream_t s = c->stream;
    g.n = (long long)g.nx * g.ny * g.nz;
    g.Nx = 2 * nice_size(g.nx);
    g.Ny = 2 * nice_size(g.ny);
    g.Nz = g.nz > 1 ? 2 * nice_size(g.nz) : 1;
    g.LX = g.Nx / 2;
    if (!bm_make_plan(g.LX, g.px) || !bm_make_plan(g.Ny, g.py) || !bm_make_plan(g.Nz, g.pz))
        return fail(BM_EUNSUPPORTED, "unsupported FFT size");
    choose_tiles<T>(g);
    size_t v3 = sizeof(T) * 3 * (size_t)g.n;
    if (cudaMalloc(&g.buf[0], v3) != cudaSuccess) return fail(BM_ENOMEM, "multilayer grid M");
    cudaMemsetAsync(g.buf[0], 0, v3, s);
    size_t s1 = sizeof(cpx<T>) * 3 * (size_t)g.nz * g.ny * g.LX, s2 = sizeof(cpx<T>) * 3 * (size_t)g.nz * g.Ny * g.LX;
    if (cudaMalloc(&g.S1, s1) != cudaSuccess) return fail(BM_ENOMEM, "multilayer S1");
    if (cudaMalloc(&g.S2, s2) != cudaSuccess) return fail(BM_ENOMEM, "multilayer S2");
    cudaMemsetAsync(g.S1, 0, s1, s);
    cudaMemsetAsync(g.S2, 0, s2, s);
    int rc;
    if ((rc = upload_table<T>(&g.twx, g.LX, false, s))) return rc;
    if ((rc = upload_table<T>(&g.twx2, g.Nx, false, s))) return rc;
    if ((rc = upload_table<T>(&g.twy, g.Ny, false, s))) return rc;
    if ((rc = upload_table<T>(&g.twz, g.Nz, false, s))) return rc;
    return 0;
}

template <typename T>
int upload_vec(void **dst, const std::vector<T> &v, cudaStream_t s)
{
    size_t bytes = sizeof(T) * (v.empty() ? 1 : v.size());
    if (cudaMalloc(dst, bytes) != cudaSuccess) return fail(BM_ENOMEM, "multilayer transfer lists");
    if (!v.empty()) CK(cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return 0;
}

template <typename T>
std::vector<T> as_type(const std::vector<double> &v)
{
    std::vector<T> o(v.size());
    for (size_t i = 0; i < v.size(); i++) o[i] = (T)v[i];
    return o;
}

template <typename T> MLZArgs<T> ml_zargs(bm_ctx *c, int W, int gate);

template <typename T>
int prepare_sm(bm_ctx *c)
{
    MLRun &r = *c->ml;
    const SMGeom &g = r.smg;
    cudaStream_t s = c->stream;
    Mesh &G = r.smgrid;
    G.nx = g.n[0]; G.ny = g.n[1]; G.nz = g.n[2];
    for (int a = 0; a < 3; a++) { G.h[a] = g.h[a]; G.o[a] = g.rs[a]; G.pbc[a] = c->sm_pbc[a]; }
    G.modules = BM_DEMAG;
    int rc;
    if ((rc = prepare_grid<T>(c, G))) return rc;
    size_t v3 = sizeof(T) * 3 * (size_t)G.n;
    if (cudaMalloc(&G.Hout, v3) != cudaSuccess) return fail(BM_ENOMEM, "supermesh field");
    cudaMemsetAsync(G.Hout, 0, v3, s);
    // kernel spectra of the supermesh grid (with its PBC images)
    size_t nk = (size_t)(G.Nx / 2 + 1) * (G.Ny / 2 + 1) * (G.Nz / 2 + 1);
    if (cudaMalloc(&G.K, sizeof(T) * 6 * nk) != cudaSuccess) return fail(BM_ENOMEM, "supermesh kernel spectra");
    void *tx = nullptr, *ty = nullptr, *tz = nullptr;
    if ((rc = upload_table<double>(&tx, G.Nx, true, s)) || (rc = upload_table<double>(&ty, G.Ny, true, s)) ||
        (rc = upload_table<double>(&tz, G.Nz, true, s))) return rc;
    double hm = std::fmax(G.h[0], std::fmax(G.h[1], G.h[2]));
    std::vector<double> fq(6 * BM_FARQ_PER_COMP);
    bm_far_coeffs(G.h[0] / hm, G.h[1] / hm, G.h[2] / hm, fq.data());
    CK(cudaMemcpyAsync(c->farq, fq.data(), sizeof(double) * fq.size(), cudaMemcpyHostToDevice, s));
    rc = build_kernels_device<T>((T *)G.K, G.nx, G.ny, G.nz, G.Nx, G.Ny, G.Nz, G.h[0], G.h[1], G.h[2], c->farq,
                                 (const cpx<double> *)tx, (const cpx<double> *)ty, (const cpx<double> *)tz, s, G.pbc);
    cudaFree(tx); cudaFree(ty); cudaFree(tz);
    if (rc) return fail(BM_ECUDA, "supermesh kernel build failed (" + std::to_string(rc) + ")");
    // transfer lists: in per mesh (into the supermesh cells), out per mesh (into the mesh's Hd)
    const size_t nm = r.mesh_of.size();
    r.sm_in_ptr.assign(nm, nullptr);
    r.sm_in_idx.assign(nm, nullptr);
    r.sm_in_w.assign(nm, nullptr);
    for (size_t k = 0; k < nm; k++) {
        const SMMeshXfer &x = g.mesh[k];
        Mesh &m = c->meshes[r.mesh_of[k]];
        if ((rc = upload_vec<int>((void **)&r.sm_in_ptr[k], x.in_ptr, s))) return rc;
        if ((rc = upload_vec<int>((void **)&r.sm_in_idx[k], x.in_idx, s))) return rc;
        if ((rc = upload_vec<T>(&r.sm_in_w[k], as_type<T>(x.in_w), s))) return rc;
        if ((rc = upload_vec<int>((void **)&m.out_ptr, x.out_ptr, s))) return rc;
        if ((rc = upload_vec<int>((void **)&m.out_idx, x.out_idx, s))) return rc;
        if ((rc = upload_vec<T>(&m.out_w, as_type<T>(x.out_w), s))) return rc;
    }
    CK(cudaStreamSynchronize(s));
    if (c->autotune) {
        tune_grid_yz<T>(c, G);
        if ((rc = tune_grid_x<T>(c, G))) return rc;
    }
    cudaGetLastError();
    CK(cudaStreamSynchronize(s));
    return 0;
}

template <typename T>
int prepare_ml(bm_ctx *c)
{
    if (!c->ml) return 0;
    if (c->ml->sm) return prepare_sm<T>(c);
    MLRun &r = *c->ml;
    MLGeom &g = r.g;
    cudaStream_t s = c->stream;
    const int L = g.L;
    r.ncc = (long long)g.nc[0] * g.nc[1] * g.nc[2];
    r.grids.assign(L, Mesh());
    r.direct.assign(L, -1);
    r.block.assign(L, -1);
    r.in_ptr.assign(L, nullptr);
    r.in_idx.assign(L, nullptr);
    r.in_w.assign(L, nullptr);
    int rc;
    for (int l = 0; l < L; l++) {
        const MLLayerGeom &y = g.layers[l];
        if (!y.transfer) { r.direct[l] = r.mesh_of[y.mesh]; continue; }
        Mesh &G = r.grids[l];
        G.nx = g.nc[0]; G.ny = g.nc[1]; G.nz = g.nc[2];
        for (int a = 0; a < 3; a++) { G.h[a] = y.hc[a]; G.o[a] = y.rs[a]; }
        G.modules = BM_DEMAG;
        if ((rc = prepare_grid<T>(c, G))) return rc;
        if (c->es_level > 0) {
            // evaluation speedup: the layer's saved fields, and its self term SelfDemag_PBC(h_common,
            // n_common) (Boris/SDemag_Demag.cpp:328) scaled as the unnormalised transforms carry it
            size_t s1 = sizeof(cpx<T>) * 3 * (size_t)G.nz * G.ny * G.LX;
            if (cudaMalloc(&G.G, s1 * c->es_level) != cudaSuccess) return fail(BM_ENOMEM, "evaluation speedup slots");
            cudaMemsetAsync(G.G, 0, s1 * c->es_level, s);
            double S[3];
            if (c->es_self_metres) self_demag_metres_host(G.h[0], G.h[1], G.h[2], S);
            else self_demag_host(G.h[0], G.h[1], G.h[2], S);
            for (int k = 0; k < 3; k++) G.es_cs[k] = S[k] * (double)G.Ny * (double)G.Nz;
        }
        if ((rc = upload_vec<int>((void **)&r.in_ptr[l], y.in_ptr, s))) return rc;
        if ((rc = upload_vec<int>((void **)&r.in_idx[l], y.in_idx, s))) return rc;
        if ((rc = upload_vec<T>(&r.in_w[l], as_type<T>(y.in_w), s))) return rc;
    }
    for (size_t k = 0; k < g.out.size(); k++) {
        const MLMeshOut &o = g.out[k];
        if (o.layers.empty()) continue;
        Mesh &m = c->meshes[r.mesh_of[k]];
        if ((rc = upload_vec<int>((void **)&m.out_ptr, o.ptr, s))) return rc;
        if ((rc = upload_vec<int>((void **)&m.out_idx, o.idx, s))) return rc;
        if ((rc = upload_vec<T>(&m.out_w, as_type<T>(o.w), s))) return rc;
        size_t hb = sizeof(T) * 3 * (size_t)r.ncc * o.layers.size();
        if (cudaMalloc(&m.Hc, hb) != cudaSuccess) return fail(BM_ENOMEM, "multilayer common-grid fields");
        cudaMemsetAsync(m.Hc, 0, hb, s);
        for (size_t b = 0; b < o.layers.size(); b++) r.block[o.layers[b]] = (int)b;
    }
    // kernel collection
    size_t total = 0;
    for (auto &K : g.kernels) total = std::max(total, K.off + ((K.count + 31) & ~(size_t)31));
    if (cudaMalloc(&r.K, sizeof(T) * total) != cudaSuccess) return fail(BM_ENOMEM, "multilayer kernels");
    void *tx = nullptr, *ty = nullptr, *tz = nullptr;
    if ((rc = upload_table<double>(&tx, g.N[0], true, s)) || (rc = upload_table<double>(&ty, g.N[1], true, s)) ||
        (rc = upload_table<double>(&tz, g.N[2], true, s))) return rc;
    for (auto &K : g.kernels) {
        double hq[3];
        if (K.kind == BM_MLK_SELF) {
            double hm = std::fmax(K.hd[0], std::fmax(K.hd[1], K.hd[2]));
            for (int a = 0; a < 3; a++) hq[a] = K.hd[a] / hm;
        } else {
            for (int a = 0; a < 3; a++) hq[a] = K.irregular ? K.hd[a] : K.hs[a];
        }
        std::vector<double> fq(6 * BM_FARQ_PER_COMP);
        bm_far_coeffs(hq[0], hq[1], hq[2], fq.data());
        CK(cudaMemcpyAsync(c->farq, fq.data(), sizeof(double) * fq.size(), cudaMemcpyHostToDevice, s));
        rc = build_ml_kernel_device<T>((T *)r.K + K.off, K, g.nc, g.N, c->farq, (const cpx<double> *)tx,
                                       (const cpx<double> *)ty, (const cpx<double> *)tz, s);
        if (rc) break;
    }
    cudaFree(tx); cudaFree(ty); cudaFree(tz);
    if (rc) return fail(BM_ECUDA, "multilayer kernel build failed (" + std::to_string(rc) + ")");
    if ((rc = upload_table<T>(&r.twz, g.N[2], false, s))) return rc;
    CK(cudaStreamSynchronize(s));
    // common grids: y-pass variant and width, x-transform variant and rows per block
    if (c->autotune)
        for (int l = 0; l < L; l++) {
            if (r.direct[l] >= 0) continue;
            tune_ypass<T>(c, r.grids[l]);
            if ((rc = tune_grid_x<T>(c, r.grids[l]))) return rc;
        }
    // z pass tile: columns per block, the fastest of the widths that fit (timed on the layer
    // spectra, which the first evaluation rewrites)
    const int lim = bm_lb<T>::v, LX = g.N[0] / 2;
    r.W = 0;
    float best = 1e30f;
    const char *fw = getenv("BM_ML_W");   // fixed width (profiling runs)
    if (fw && atoi(fw) >= 1 && (atoi(fw) & (atoi(fw) - 1)) == 0) {
        r.W = atoi(fw);
        return 0;
    }
    for (int W = 1; W <= 32 && W <= LX; W *= 2) {
        MLZArgs<T> z = ml_zargs<T>(c, W, BM_GATE_ALWAYS);
        z.st = nullptr;
        if (((6 * L * W + 31) & ~31) > lim || zmid_ml_smem<T>(L, g.N[2], W, z.ksm) > 200 * 1024) continue;
        if (!r.W) r.W = W;
        if (!c->autotune) continue;
        float t = time_launches(s, [&]() { return launch_zmid_ml<T>(z, s); }, 3);
        if (t < best) { best = t; r.W = W; }
    }
    if (!r.W) return fail(BM_EUNSUPPORTED, "multilayer: no z-pass tile fits");
    cudaGetLastError();
    CK(cudaStreamSynchronize(s));
    return 0;
}

template <typename T>
int prepare_T(bm_ctx *c)
{
    if (int rc = ml_plan(c)) { free_ml(c); for (auto &mm : c->meshes) mm.ml_role = 0; return rc; }
    for (auto &m : c->meshes) {
        int rc = prepare_mesh<T>(c, m);
        if (rc) { for (auto &mm : c->meshes) free_mesh(mm); free_ml(c); return rc; }
        // BM_TILES="w2,wy,wz,rows" fixes the tile shapes (profiling runs); otherwise autotune
        const char *ev = getenv("BM_TILES");
        int t4[4];
        if (ev && sscanf(ev, "%d,%d,%d,%d", &t4[0], &t4[1], &t4[2], &t4[3]) == 4) {
            m.W2 = t4[0]; m.Wy = t4[1]; m.Wz = t4[2]; m.rpb = t4[3];
            const char *sr = getenv("BM_STAGE_ROWS");
            m.staged = (sr && sr[0] == '1') ? 1 : 0;
            const char *sx = getenv("BM_STAGE_XV");
            m.xv = (sx && sx[0] == '1' && stage_reg_q(m.LX, 1)) ? 1 : (sx && sx[0] == '2' && stage_reg_q(m.LX, 2)) ? 2
                 : (sx && sx[0] == '3' && stage_reg_q(m.LX, 2)) ? 3 : 0;
            const char *sy = getenv("BM_Y_XV");
            m.yv = (sy && sy[0] == '1' && ypass_has_st(m.Ny) && m.nz > 1 && ypass_st_threads(m.Ny, m.Wy) % 32 == 0) ? 1 : 0;
            if (sy && sy[0] == '2' && m.nz > 1) {
                YZArgs<T> ya = yz_args<T>(c, m, BM_GATE_ALWAYS);
                ya.W = m.Wy;
                if (ypass_tma_fits<T>(ya)) m.yv = 2;
            }
            const char *szv = getenv("BM_Z_XV");
            m.zv = (szv && szv[0] == '1' && m.nz > 1 && zmid_has_par(m.Nz, m.Wz)) ? 1 : 0;
            const char *sz = getenv("BM_YZY");
            m.yzy = 0;
            if (sz && sz[0] == '1' && m.nz > 1 && m.ml_role == 0 && (m.modules & BM_DEMAG) && !c->batched)
                m.yzy = yzy_available<T>(yz_args<T>(c, m, BM_GATE_ALWAYS)) == 0 ? 1 : 0;
        } else if (c->autotune && !c->batched) autotune_mesh<T>(c, m);
    }
    if (int rc = prepare_ml<T>(c)) { for (auto &mm : c->meshes) free_mesh(mm); free_ml(c); return rc; }
    return 0;
}

// Device bytes a context's meshes need (their own buffers; a multilayered convolution's common
// grids and kernels come on top), and the largest transient scratch of a kernel-spectrum build.
void plan_bytes(const bm_ctx *c, size_t elem, double *persistent, double *transient)
{
    double per = 0.0, tr = 0.0;
    for (const Mesh &m : c->meshes) {
        const double n = (double)m.nx * m.ny * m.nz;
        const double Nx = 2.0 * nice_size(m.nx), Ny = 2.0 * nice_size(m.ny), Nz = m.nz > 1 ? 2.0 * nice_size(m.nz) : 1.0;
        const double LX = Nx / 2, v3 = 3.0 * elem * n;
        per += (4 + (c->eval == BM_RKDP54 ? 6 : 3) + 1) * v3 + 24.0 * n;
        if (!m.Ms_map.empty()) per += elem * n;
        if (!m.K1_map.empty()) per += elem * n;
        if (m.modules & BM_DEMAG) {
            const double s1 = 6.0 * elem * m.nz * m.ny * LX;
            per += s1 * (1 + c->es_level);
            if (m.nz > 1) per += 6.0 * elem * m.nz * Ny * LX;
            per += 6.0 * elem * (LX + 1) * (Ny / 2 + 1) * (Nz / 2 + 1);
            tr = std::max(tr, 48.0 * n + 16.0 * Nx * Ny * Nz);   // tensor octant + one FP64 transform grid
        }
    }
    *persistent = per;
    *transient = tr;
}

int prepare(bm_ctx *c)
{
    if (c->ready) return 0;
    if (c->meshes.empty()) return fail(BM_ESTATE, "no mesh");
    if (c->batched && c->ml_mode >= 0) return fail(BM_EUNSUPPORTED, "batched meshes with a multilayered convolution");
    // the reference has no evaluation speedup for the supermesh convolution (Boris/SDemag.cpp:742)
    if (c->es_level > 0 && c->ml_mode == BM_ML_SUPERMESH)
        return fail(BM_EUNSUPPORTED, "evaluation speedup with the supermesh demag");
    for (auto &m : c->meshes) {
        if (!(m.modules & BM_DEMAG) || !(m.pbc[0] || m.pbc[1] || m.pbc[2]) || c->ml_mode == BM_ML_SUPERMESH) continue;
        if (c->ml_mode >= 0) return fail(BM_EUNSUPPORTED, "periodic boundary conditions with a multilayered convolution");
        const int nc[3] = {m.nx, m.ny, m.nz};
        if (int rc = pbc_work_check(nc, m.pbc)) return rc;
    }
    CK(cudaSetDevice(c->device));
    // refuse up front, before any allocation, when the meshes cannot fit: the free device memory,
    // or the context's own limit (bm_set_memory_limit) when it is lower
    {
        double per = 0.0, tr = 0.0;
        plan_bytes(c, c->precision == BM_FP64 ? sizeof(double) : sizeof(float), &per, &tr);
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        double avail = (double)fr;
        const char *what = "free device memory";
        if (c->mem_limit > 0 && (double)c->mem_limit < avail) { avail = (double)c->mem_limit; what = "the context's memory limit"; }
        if (per + tr > avail) {
            char msg[256];
            snprintf(msg, sizeof(msg), "the meshes need %.1f MB of device memory (%.1f MB more while the kernels are built); "
                     "%s is %.1f MB", per / 1e6, tr / 1e6, what, avail / 1e6);
            return fail(BM_ENOMEM, msg);
        }
    }
    int rc = (c->precision == BM_FP64) ? prepare_T<double>(c) : prepare_T<float>(c);
    if (rc) return rc;
    c->ready = true;
    c->s1_dirty = true;
    c->es_reset = true;
    return upload_state(c);
}

// ------------------------------------------------------------------ per-launch timing records
// Records an event after a launch (when bm_time_step is collecting) with its kind and bytes.
void lt_mark(bm_ctx *c, int kind, double bytes)
{
    if (!c->lt) return;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, c->stream);
    c->lt->ev.push_back(e);
    c->lt->kind.push_back(kind);
    c->lt->bytes.push_back(bytes);
}

// Algorithmic bytes of one stage-kernel launch: every array it must read once and write once
// (the exchange stencil's neighbour reads are re-reads of M), from its arguments.
template <typename T>
double stage_alg_bytes(const StageArgs<T> &a)
{
    const double p = sizeof(T), v = 3.0 * p * (double)a.n;
    const double s1 = 3.0 * a.nz * a.ny * (double)a.LX * sizeof(cpx<T>);
    const bool fields = a.mode != BM_MODE_UPDATE;
    double b = v;                                                   // Min
    if (a.mode != BM_MODE_HEFF) {
        if (a.Mbase && a.Mbase != a.Min) b += v;
        b += a.nev * v;
    }
    if (a.Ms_map) b += p * (double)a.n;
    if (fields && a.K1_map && (a.modules & BM_MOD_ANIUNI)) b += p * (double)a.n;
    if (fields && (a.modules & BM_MOD_DEMAG) && a.S1) b += s1;      // demag spectrum rows, inverse x
    if (fields && a.Hd) b += v;
    if (a.mode == BM_MODE_HEFF) return b + v;                       // Hout
    if (a.Hsave) b += v;
    if (a.ev_out) b += v;
    if (a.mode == BM_MODE_LTE) return b;
    if (a.Ysave) b += v;
    if (a.copy_to) b += v;
    if (a.Mout) b += v;
    if (a.do_xfwd && a.S1) b += s1;                                 // forward x of the new M
    return b;
}

// Algorithmic bytes of the y / z passes of one mesh: spectra read once and written once, the
// kernel spectra read once.
double yz_alg_bytes(const Mesh &m, int kind, size_t p)
{
    const double cs = 2.0 * p;
    const double s1 = 3.0 * m.nz * m.ny * (double)m.LX * cs, s2 = 3.0 * m.nz * m.Ny * (double)m.LX * cs;
    const double kb = 6.0 * (m.LX + 1) * (m.Ny / 2 + 1) * (double)(m.Nz / 2 + 1) * p;
    switch (kind) {
    case BM_TK_YFWD: case BM_TK_YINV: return s1 + s2;
    case BM_TK_ZMID: return 2.0 * s2 + kb;
    case BM_TK_YMID2D: return 2.0 * s1 + 4.0 / 6.0 * kb;
    case BM_TK_YZY: return 2.0 * s1 + kb;
    default: return 0.0;
    }
}

// ------------------------------------------------------------------ kernel argument builders
template <typename T>
YZArgs<T> yz_args(bm_ctx *c, Mesh &m, int gate)
{
    YZArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.S1 = (cpx<T> *)m.S1; a.S2 = (cpx<T> *)m.S2; a.K = (const T *)m.K;
    a.twy = (const cpx<T> *)m.twy; a.twz = (const cpx<T> *)m.twz;
    a.py = m.py; a.pz = m.pz;
    a.nx = m.nx; a.ny = m.ny; a.nz = m.nz; a.LX = m.LX; a.Ny = m.Ny; a.Nz = m.Nz;
    a.W = m.nz > 1 ? m.Wy : m.W2;
    a.st = c->st; a.gate = gate;
    a.yv = m.yv;
    a.zv = m.zv;
    return a;
}

template <typename T>
int enqueue_yz(bm_ctx *c, Mesh &m, int gate, int *count)
{
    if (!(m.modules & BM_DEMAG)) return 0;
    YZArgs<T> a = yz_args<T>(c, m, gate);
    if (m.nz == 1) {
        CKL(launch_ymid2d<T>(a, c->stream), "ymid2d");
        lt_mark(c, BM_TK_YMID2D, yz_alg_bytes(m, BM_TK_YMID2D, sizeof(T)));
        (*count)++;
    } else if (m.yzy) {
        CKL(launch_yzy<T>(a, c->stream), "yzy");
        lt_mark(c, BM_TK_YZY, yz_alg_bytes(m, BM_TK_YZY, sizeof(T)));
        (*count)++;
    } else {
        CKL(launch_yfwd<T>(a, c->stream), "yfwd");
        lt_mark(c, BM_TK_YFWD, yz_alg_bytes(m, BM_TK_YFWD, sizeof(T)));
        a.W = m.Wz;
        CKL(launch_zmid<T>(a, c->stream), "zmid");
        lt_mark(c, BM_TK_ZMID, yz_alg_bytes(m, BM_TK_ZMID, sizeof(T)));
        a.W = m.Wy;
        CKL(launch_yinv<T>(a, c->stream), "yinv");
        lt_mark(c, BM_TK_YINV, yz_alg_bytes(m, BM_TK_YINV, sizeof(T)));
        (*count) += 3;
    }
    return 0;
}

template <typename T>
StageArgs<T> stage_args(bm_ctx *c, Mesh &m)
{
    StageArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.nx = m.nx; a.ny = m.ny; a.nz = m.nz; a.LX = m.LX; a.Nx = m.Nx;
    a.hx = m.h[0]; a.hy = m.h[1]; a.hz = m.h[2];
    a.S1 = (cpx<T> *)m.S1;
    a.twx = (const cpx<T> *)m.twx; a.twx2 = (const cpx<T> *)m.twx2;
    a.px = m.px;
    a.rpb = m.rpb;
    a.scale = (T)(2.0 / ((double)m.Nx * m.Ny * m.Nz));
    a.modules = m.modules;
    a.Ms = (T)m.Ms; a.A = (T)m.A; a.D = (T)m.D; a.alpha = (T)m.alpha; a.grel = (T)m.grel;
    a.K1 = (T)m.K1; a.K2 = (T)m.K2;
    double en = std::sqrt(m.ea[0] * m.ea[0] + m.ea[1] * m.ea[1] + m.ea[2] * m.ea[2]);
    for (int i = 0; i < 3; i++) a.ea[i] = (T)(en > 0 ? m.ea[i] / en : 0.0);
    a.Ms_map = (const T *)m.Msd; a.K1_map = (const T *)m.K1d;
    a.Ha = m.Had; a.nHa = m.nHa; a.Ha_tspan = m.Ha_tspan;
    a.st = c->st;
    a.n = m.n;
    a.do_xfwd = (m.modules & BM_DEMAG) ? 1 : 0;
    a.staged = m.staged;
    a.xv = m.xv;
    for (int i = 0; i < 3; i++) a.pbc[i] = (m.pbc[i] > 0) - (m.pbc[i] < 0);
    stage_derive(a);
    if (m.ml_role == 2) {
        // multilayer with mesh transfer: the demag field arrives in Hd, no x transforms here
        a.modules &= ~BM_DEMAG;
        a.do_xfwd = 0;
        a.S1 = nullptr;
        a.Hd = (const T *)m.Hd;
    }
    return a;
}

template <typename T> T *B(Mesh &m, int i) { return (T *)m.buf[i]; }
template <typename T> T *E(Mesh &m, int i) { return (T *)m.ev[i]; }

// ------------------------------------------------------------------ many meshes per launch
size_t bp_append(BatchPlan &bp, const void *p, size_t bytes)
{
    size_t off = (bp.hbuf.size() + 255) & ~(size_t)255;
    bp.hbuf.resize(off + bytes);
    memcpy(bp.hbuf.data() + off, p, bytes);
    return off;
}

// stage kernels of several meshes: per-mesh launches, or one launch over (mesh, row block) items
// with the generic-length kernel (rows per block chosen so every mesh fills ~256 threads)
// stage kernels of every mesh: one launch per x length with a radix-8 register kernel, one for
// the remaining lengths (generic kernel). Only the last launch finishes the step (error-norm
// controller, time advance); the earlier ones only add to the error-norm maximum.
template <typename T>
int stage_batch_one(bm_ctx *c, int key, std::vector<StageArgs<T>> &v, int *count)
{
    BatchPlan &bp = c->bp;
    if (bp.collect) {
        std::vector<int2> work;
        int nt = 32;
        size_t smem = 0;
        for (size_t i = 0; i < v.size(); i++) {
            StageArgs<T> &a = v[i];
            a.staged = 0;
            const int rows = a.ny * a.nz;
            // register groups: the radix-16 variant where it exists (x 256 .. 1024), else radix 8 / 4-3
            const int xvb = stage_reg_q(a.LX, 2) ? 2 : 1;
            const int tpl = key ? stage_reg_q(a.LX, xvb) : a.px.tpl;
            int rpb = 256 / (3 * tpl);
            rpb = std::max(1, std::min(rpb, rows));
            a.rpb = rpb;
            a.xv = key ? xvb : 0;
            for (int b = 0; b < (rows + rpb - 1) / rpb; b++) work.push_back(make_int2((int)i, b));
            nt = std::max(nt, (3 * rpb * tpl + 31) & ~31);
            const size_t lsp = key ? (size_t)(a.LX + a.LX / 16 + 1) : (size_t)padded_len(a.LX);
            smem = std::max(smem, (size_t)3 * rpb * lsp * sizeof(cpx<T>));
        }
        BatchRec r;
        r.kind = 0;
        r.key = key;
        r.args_off = bp_append(bp, v.data(), sizeof(StageArgs<T>) * v.size());
        r.work_off = bp_append(bp, work.data(), sizeof(int2) * work.size());
        r.nwork = (int)work.size();
        r.nt = nt;
        r.smem = smem;
        r.plain = key ? 1 : 0;
        for (auto &a : v) if (!stage_plain(a)) r.plain = 0;
        bp.recs.push_back(r);
        return 0;
    }
    if (bp.next >= bp.recs.size()) return fail(BM_ESTATE, "batched launch plan out of step");
    const BatchRec &r = bp.recs[bp.next++];
    const char *base = (const char *)bp.dbuf;
    CKL(launch_stage_batch<T>(r.key, (const StageArgs<T> *)(base + r.args_off), (const int2 *)(base + r.work_off), r.nwork,
                              r.nt, r.smem, c->stream, r.plain), "stage batch");
    (*count)++;
    return 0;
}

template <typename T>
int stage_multi(bm_ctx *c, std::vector<StageArgs<T>> &v, int *count)
{
    if (v.empty()) return 0;
    if (!c->batched || v.size() == 1) {
        for (auto &a : v) {
            CKL(launch_stage<T>(a, c->stream), "stage");
            // a restore launch only works after a rejection: timed under "other", no bytes credited
            if (a.gate == BM_GATE_RESTORE) lt_mark(c, BM_TK_OTHER, 0.0);
            else lt_mark(c, BM_TK_STAGE, stage_alg_bytes(a));
            (*count)++;
        }
        return 0;
    }
    int lk = BM_LAST_NONE, pub = 0;
    for (auto &a : v) if (a.last_kind != BM_LAST_NONE) lk = a.last_kind;
    for (auto &a : v) if (a.diag & BM_DIAG_PUBLISH) pub = BM_DIAG_PUBLISH;
    std::map<int, std::vector<StageArgs<T>>> groups;   // x length with a register kernel, or 0
    for (auto &a : v) groups[stage_reg_q(a.LX, 1) ? a.LX : 0].push_back(a);
    size_t gi = 0;
    for (auto &kv : groups) {
        const bool last = (++gi == groups.size());
        for (auto &a : kv.second) {
            a.last_kind = last ? lk : BM_LAST_NONE;
            a.diag = (a.diag & ~BM_DIAG_PUBLISH) | (last ? pub : 0);   // every block of the last launch counts
        }
        if (int rc = stage_batch_one<T>(c, kv.first, kv.second, count)) return rc;
    }
    return 0;
}

template <typename T>
void batch_tiles(const Mesh &m, int &Wy, int &Wz)
{
    const int lim = 256;
    Wy = 16;
    while (Wy > 1 && (Wy * m.py.tpl > lim || (size_t)m.Ny * Wy * sizeof(cpx<T>) > 64 * 1024)) Wy /= 2;
    Wz = 16;
    while (Wz > 1 && (2 * Wz * m.pz.tpl > lim || zmid_smem<T>(m.Nz, Wz) > 64 * 1024)) Wz /= 2;
    while (Wy > 1 && Wy > m.LX) Wy /= 2;
    while (Wz > 1 && Wz > m.LX) Wz /= 2;
}

template <typename T>
int yz_batch_one(bm_ctx *c, int kind, int key, std::vector<YZArgs<T>> &v, int *count)
{
    if (v.empty()) return 0;
    BatchPlan &bp = c->bp;
    if (bp.collect) {
        std::vector<int2> work;
        int nt = 32;
        size_t smem = 0;
        for (size_t i = 0; i < v.size(); i++) {
            const YZArgs<T> &a = v[i];
            const int nbx = (a.LX + a.W - 1) / a.W;
            int items = nbx;
            if (kind == BM_BATCH_YFWD_ST || kind == BM_BATCH_YINV_ST) {
                items = nbx * a.nz * 3;
                nt = std::max(nt, (ypass_st_threads(a.Ny, a.W) + 31) & ~31);
                smem = std::max(smem, ((size_t)a.Ny * a.W + (size_t)(a.Ny / 16) * 8) * sizeof(cpx<T>));
            } else if (kind == BM_BATCH_YFWD_REG || kind == BM_BATCH_YINV_REG) {
                items = nbx * a.nz * 3;
                nt = std::max(nt, (ypass_reg_threads(a.Ny, a.W) + 31) & ~31);
                smem = std::max(smem, (size_t)a.Ny * a.W * sizeof(cpx<T>));
            } else if (kind == BM_BATCH_YMID2D_REG) {
                nt = std::max(nt, (ymid2d_reg_threads(a.Ny, a.W) + 31) & ~31);
                smem = std::max(smem, ymid2d_smem<T>(a.Ny, a.W));
            } else if (kind == BM_BATCH_ZMID_REG) {
                items = nbx * (a.Ny / 2 + 1);
                nt = std::max(nt, (6 * a.W + 31) & ~31);
                smem = std::max(smem, zmid_reg_smem<T>(a.Nz, a.W));
            } else if (kind == BM_BATCH_YFWD || kind == BM_BATCH_YINV) {
                items = nbx * a.nz * 3;
                nt = std::max(nt, (a.W * a.py.tpl + 31) & ~31);
                smem = std::max(smem, (size_t)a.Ny * a.W * sizeof(cpx<T>));
            } else if (kind == BM_BATCH_ZMID) {
                items = nbx * (a.Ny / 2 + 1);
                nt = std::max(nt, (2 * a.W * a.pz.tpl + 31) & ~31);
                smem = std::max(smem, zmid_smem<T>(a.Nz, a.W));
            } else {
                nt = std::max(nt, (a.W * a.py.tpl + 31) & ~31);
                smem = std::max(smem, ymid2d_smem<T>(a.Ny, a.W));
            }
            for (int b = 0; b < items; b++) work.push_back(make_int2((int)i, b));
        }
        BatchRec r;
        r.kind = kind;
        r.key = key;
        r.args_off = bp_append(bp, v.data(), sizeof(YZArgs<T>) * v.size());
        r.work_off = bp_append(bp, work.data(), sizeof(int2) * work.size());
        r.nwork = (int)work.size();
        r.nt = nt;
        r.smem = smem;
        bp.recs.push_back(r);
        return 0;
    }
    if (bp.next >= bp.recs.size()) return fail(BM_ESTATE, "batched launch plan out of step");
    const BatchRec &r = bp.recs[bp.next++];
    const char *base = (const char *)bp.dbuf;
    CKL(launch_yz_batch<T>(r.kind, r.key, (const YZArgs<T> *)(base + r.args_off), (const int2 *)(base + r.work_off), r.nwork,
                           r.nt, r.smem, c->stream), "y/z batch");
    (*count)++;
    return 0;
}

// y/z passes of every mesh with demag: the 2D y pass in one launch; the 3D y forward, z pass and
// y inverse each in one launch per transform length with a register kernel plus one launch for the
// remaining lengths (generic kernels)
template <typename T>
int yz_multi(bm_ctx *c, int gate, int *count)
{
    const int lim = 256;
    std::map<int, std::vector<YZArgs<T>>> g2, gy, gz;   // key Ny / Nz with a register kernel, or 0
    for (auto &m : c->meshes) {
        if (!(m.modules & BM_DEMAG)) continue;
        YZArgs<T> a = yz_args<T>(c, m, gate);
        if (m.nz == 1) {
            // batched launches take their parallelism from the many meshes: wide column tiles
            int W = 16;
            if (ypass_has_reg(m.Ny)) {
                while (W > 1 && (ymid2d_reg_threads(m.Ny, W) > 384 || ymid2d_smem<T>(m.Ny, W) > 100 * 1024 || W > m.LX)) W /= 2;
                a.W = W;
                g2[m.Ny].push_back(a);
            } else {
                while (W > 1 && (W * m.py.tpl > lim || ymid2d_smem<T>(m.Ny, W) > 100 * 1024 || W > m.LX)) W /= 2;
                a.W = W;
                g2[0].push_back(a);
            }
            continue;
        }
        int Wy, Wz;
        batch_tiles<T>(m, Wy, Wz);
        if (ypass_has_reg(m.Ny)) {
            int W = 16;
            while (W > 1 && (ypass_reg_threads(m.Ny, W) > std::min(lim, yreg_maxt<T>::v) || (size_t)m.Ny * W * sizeof(cpx<T>) > 64 * 1024 ||
                             W > m.LX)) W /= 2;
            a.W = W;
            gy[m.Ny].push_back(a);
        } else if (ypass_has_st(m.Ny)) {
            // Stockham (3 * 2^k lengths), keyed negative to keep it apart from the register groups
            int W = 16;
            while (W > 2 && (ypass_st_threads(m.Ny, W) > lim || (size_t)m.Ny * W * sizeof(cpx<T>) > 64 * 1024 || W > m.LX)) W /= 2;
            a.W = W;
            gy[-m.Ny].push_back(a);
        } else {
            a.W = Wy;
            gy[0].push_back(a);
        }
        if (zmid_has_reg(m.Nz)) {
            int W = 16;
            while (W > 1 && (6 * W > lim || zmid_reg_smem<T>(m.Nz, W) > 64 * 1024 || W > m.LX)) W /= 2;
            a.W = W;
            gz[m.Nz].push_back(a);
        } else {
            a.W = Wz;
            gz[0].push_back(a);
        }
    }
    int rc;
    for (auto &kv : g2)
        if ((rc = yz_batch_one<T>(c, kv.first ? BM_BATCH_YMID2D_REG : BM_BATCH_YMID2D, kv.first, kv.second, count))) return rc;
    auto ykind = [](int key, bool inv) {
        return key > 0 ? (inv ? BM_BATCH_YINV_REG : BM_BATCH_YFWD_REG) : key < 0 ? (inv ? BM_BATCH_YINV_ST : BM_BATCH_YFWD_ST)
                                                                            : (inv ? BM_BATCH_YINV : BM_BATCH_YFWD);
    };
    for (auto &kv : gy)
        if ((rc = yz_batch_one<T>(c, ykind(kv.first, false), kv.first < 0 ? -kv.first : kv.first, kv.second, count))) return rc;
    for (auto &kv : gz)
        if ((rc = yz_batch_one<T>(c, kv.first ? BM_BATCH_ZMID_REG : BM_BATCH_ZMID, kv.first, kv.second, count))) return rc;
    for (auto &kv : gy)
        if ((rc = yz_batch_one<T>(c, ykind(kv.first, true), kv.first < 0 ? -kv.first : kv.first, kv.second, count))) return rc;
    return 0;
}

Mesh &ml_grid(bm_ctx *c, int l)
{
    return c->ml->direct[l] >= 0 ? c->meshes[c->ml->direct[l]] : c->ml->grids[l];
}

// Demag spectra -> fields for one effective-field evaluation whose stage kernels read
// M from buffer bi of every mesh. Without a multilayered convolution: each mesh's own y/z
// passes. With one: transfer in and x FFT of the transfer layers, y passes of every layer, the
// fused z pass with the L x L products, inverse y, then inverse x and transfer out into Hd.
// arguments of the fused multilayer z pass for tile width W: layer spectra, the unique kernels
// with their shared-memory tile offsets, and the (dest, src) -> kernel map
template <typename T>
MLZArgs<T> ml_zargs(bm_ctx *c, int W, int gate)
{
    MLRun &r = *c->ml;
    const MLGeom &g = r.g;
    const int L = g.L;
    MLZArgs<T> z;
    memset(&z, 0, sizeof(z));
    for (int l = 0; l < L; l++) z.S2[l] = (cpx<T> *)ml_grid(c, l).S2;
    z.K = (const T *)r.K;
    int sm = 0;
    z.nu = (int)g.kernels.size();
    for (int u = 0; u < z.nu; u++) {
        z.u[u].kind = g.kernels[u].kind;
        z.u[u].off = (long long)g.kernels[u].off;
        z.u[u].sm = sm;
        sm += zmid_ml_tile_bytes<T>(g.kernels[u].kind, g.N[2], W);
    }
    z.ksm = sm;
    for (int i = 0; i < L * L; i++) {
        z.pu[i] = (unsigned char)g.pair_kernel[i];
        z.pinv[i] = (unsigned char)g.pair_inv[i];
    }
    z.twz = (const cpx<T> *)r.twz;
    z.L = L; z.nz = g.nc[2]; z.Ny = g.N[1]; z.Nz = g.N[2]; z.LX = g.N[0] / 2; z.W = W;
    z.st = c->st; z.gate = gate;
    return z;
}

// multilayer parts: 0 transfer in + x forward, 1 y forward, 2 z pass + products, 3 y inverse,
// 4 x inverse + transfer out
template <typename T>
int ml_enqueue_part(bm_ctx *c, int part, int gate, int bi, int *count)
{
    MLRun &r = *c->ml;
    const MLGeom &g = r.g;
    const int L = g.L;
    cudaStream_t s = c->stream;
    if (part == 0) for (int l = 0; l < L; l++) {
        if (r.direct[l] >= 0) continue;
        Mesh &G = r.grids[l];
        Mesh &M = c->meshes[r.mesh_of[g.layers[l].mesh]];
        CKL(launch_ml_gather<T>(B<T>(G, 0), r.ncc, r.ncc, B<T>(M, bi), M.n, r.in_ptr[l], r.in_idx[l], (const T *)r.in_w[l],
                                c->st, gate, s), "multilayer transfer in");
        StageArgs<T> a = stage_args<T>(c, G);
        a.mode = BM_MODE_UPDATE;
        a.gate = gate;
        a.Min = B<T>(G, 0); a.Mbase = B<T>(G, 0);
        a.nev = 0;
        CKL(launch_stage<T>(a, s), "multilayer x forward");
        (*count) += 2;
    }
    if (part == 1) for (int l = 0; l < L; l++) {
        Mesh &G = ml_grid(c, l);
        YZArgs<T> a = yz_args<T>(c, G, gate);
        a.W = G.Wy;
        CKL(launch_yfwd<T>(a, s), "multilayer y forward");
        (*count)++;
    }
    if (part == 2) {
        MLZArgs<T> z = ml_zargs<T>(c, r.W, gate);
        CKL(launch_zmid_ml<T>(z, s), "multilayer z pass");
        (*count)++;
    }
    if (part == 3) for (int l = 0; l < L; l++) {
        Mesh &G = ml_grid(c, l);
        YZArgs<T> a = yz_args<T>(c, G, gate);
        a.W = G.Wy;
        CKL(launch_yinv<T>(a, s), "multilayer y inverse");
        (*count)++;
    }
    if (part == 4) for (int l = 0; l < L; l++) {
        if (r.direct[l] >= 0) continue;
        Mesh &G = r.grids[l];
        Mesh &M = c->meshes[r.mesh_of[g.layers[l].mesh]];
        StageArgs<T> a = stage_args<T>(c, G);
        a.mode = BM_MODE_HEFF;
        a.modules = BM_DEMAG;
        a.do_xfwd = 0;
        a.gate = gate;
        a.Min = B<T>(G, 0);
        a.Hout = (T *)M.Hc + (size_t)r.block[l] * 3 * r.ncc;
        CKL(launch_stage<T>(a, s), "multilayer x inverse");
        (*count)++;
    }
    if (part == 4) for (size_t k = 0; k < g.out.size(); k++) {
        if (g.out[k].layers.empty()) continue;
        Mesh &M = c->meshes[r.mesh_of[k]];
        CKL(launch_ml_gather<T>((T *)M.Hd, M.n, M.n, (const T *)M.Hc, r.ncc, M.out_ptr, M.out_idx, (const T *)M.out_w, c->st,
                                gate, s), "multilayer transfer out");
        (*count)++;
    }
    return 0;
}

// Supermesh demag: every mesh's M gathered onto the supermesh grid (one accumulating gather per mesh),
// its x forward transform, the y / z passes with the supermesh kernel, the inverse x transform into
// the grid's field, and one gather per mesh into its Hd (SDemag::UpdateField, Boris/SDemag.cpp:737-760:
// transfer_in, Convolute, transfer_out).
template <typename T>
int sm_enqueue(bm_ctx *c, int gate, int bi, int *count)
{
    MLRun &r = *c->ml;
    Mesh &G = r.smgrid;
    cudaStream_t s = c->stream;
    for (size_t k = 0; k < r.mesh_of.size(); k++) {
        Mesh &M = c->meshes[r.mesh_of[k]];
        CKL(launch_ml_gather<T>(B<T>(G, 0), G.n, G.n, B<T>(M, bi), M.n, r.sm_in_ptr[k], r.sm_in_idx[k],
                                (const T *)r.sm_in_w[k], c->st, gate, s, k > 0), "supermesh transfer in");
        (*count)++;
    }
    StageArgs<T> a = stage_args<T>(c, G);
    a.mode = BM_MODE_UPDATE;
    a.gate = gate;
    a.Min = B<T>(G, 0); a.Mbase = B<T>(G, 0);
    a.nev = 0;
    CKL(launch_stage<T>(a, s), "supermesh x forward");
    (*count)++;
    if (int rc = enqueue_yz<T>(c, G, gate, count)) return rc;
    StageArgs<T> h = stage_args<T>(c, G);
    h.mode = BM_MODE_HEFF;
    h.modules = BM_DEMAG;
    h.do_xfwd = 0;
    h.gate = gate;
    h.Min = B<T>(G, 0);
    h.Hout = (T *)G.Hout;
    CKL(launch_stage<T>(h, s), "supermesh x inverse");
    (*count)++;
    for (size_t k = 0; k < r.mesh_of.size(); k++) {
        Mesh &M = c->meshes[r.mesh_of[k]];
        CKL(launch_ml_gather<T>((T *)M.Hd, M.n, M.n, (const T *)G.Hout, G.n, M.out_ptr, M.out_idx, (const T *)M.out_w,
                                c->st, gate, s), "supermesh transfer out");
        (*count)++;
    }
    return 0;
}

template <typename T>
int enqueue_fields(bm_ctx *c, int gate, int bi, int *count)
{
    if (c->ml && c->ml->sm) return sm_enqueue<T>(c, gate, bi, count);
    if (!c->ml) {
        if (c->batched && c->meshes.size() > 1) return yz_multi<T>(c, gate, count);
        for (auto &m : c->meshes) {
            int rc = enqueue_yz<T>(c, m, gate, count);
            if (rc) return rc;
        }
        return 0;
    }
    for (int part = 0; part < 5; part++) {
        int rc = ml_enqueue_part<T>(c, part, gate, bi, count);
        if (rc) return rc;
    }
    return 0;
}

// S1 = x-FFT(M) for every mesh (after set_m, compute_* or a fresh start)
template <typename T>
int enqueue_prime(bm_ctx *c, int *count)
{
    for (auto &m : c->meshes) {
        if (!(m.modules & BM_DEMAG) || m.ml_role == 2) continue;
        StageArgs<T> a = stage_args<T>(c, m);
        a.mode = BM_MODE_UPDATE;
        a.Min = B<T>(m, 0); a.Mbase = B<T>(m, 0);
        a.nev = 0;
        CKL(launch_stage<T>(a, c->stream), "prime");
        (*count)++;
    }
    return 0;
}

long long es_plane(const Mesh &m) { return (long long)m.nz * m.ny * m.LX; }

// Whether a mesh's extrapolated spectrum is formed by its own stage kernel (the register stage kernels,
// one launch per mesh, no multilayered convolution) in place of a k_es_extrap pass. Opt-in (BM_ES_FOLD=1):
// on the headline film the separate pass is faster (RK4 quadratic 2779 against 2351 Mcell-steps/s,
// RKDP54 1599 against 1358): the stage kernel's slot loads come after its spectrum row has landed and
// stall it, where the separate pass streams the slots at 75 % of the copy bandwidth.
bool es_fold_ok(const bm_ctx *c, const Mesh &m)
{
    const char *env = getenv("BM_ES_FOLD");
    if (!(env && env[0] == '1')) return false;
    return !c->ml && !c->batched && (m.modules & BM_DEMAG) && m.G && stage_reg_path(m.LX, m.xv);
}

template <typename T>
void es_fold_args(const bm_ctx *c, const Mesh &m, StageArgs<T> &a)
{
    if (!c->es_fold_pending || !es_fold_ok(c, m)) return;
    a.es_fold = c->es_fold_pending;
    a.esG = (const cpx<T> *)m.G;
    for (int k = 0; k < 3; k++) a.es_cs[k] = m.es_cs[k];
    a.es_ceval = c->es_fold_ceval;
}

// The spectra the evaluation speedup saves and extrapolates: every mesh with demag, or with the
// multilayered convolution every layer's (its common grid, or its mesh when the mesh's grid is the
// common grid), as SDemagCUDA::UpdateField does per layer (Boris/SDemagCUDA.cpp:587-930).
std::vector<Mesh *> es_targets(bm_ctx *c)
{
    std::vector<Mesh *> v;
    if (c->ml) {
        for (int l = 0; l < c->ml->g.L; l++) v.push_back(&ml_grid(c, l));
    } else {
        for (auto &m : c->meshes)
            if (m.modules & BM_DEMAG) v.push_back(&m);
    }
    return v;
}

// Multilayered convolution with the speedup, one evaluation: the layers' x forward transforms (part 0)
// give the x spectra of their inputs; a saving evaluation then runs es_pre, the y / z passes and the
// L x L product (parts 1-3, gated on the decision), es_post and es_commit; an extrapolating one runs
// es_extrap on the same spectra; the x inverse and the transfers out (part 4) finish both.
// mode: 1 save (RK4), 2 extrapolate (RK4), 3 decided on the device (RKDP54, sel 1).
template <typename T>
int enqueue_ml_es(bm_ctx *c, int mode, int gate_xt, int gate_yz, double c_eval, int bi, int *count)
{
    const int sel = (mode == 3) ? 1 : 0;
    if (int rc = ml_enqueue_part<T>(c, 0, gate_xt, bi, count)) return rc;
    const std::vector<Mesh *> tg = es_targets(c);
    if (mode != 2) {
        for (Mesh *m : tg) {
            CKL(launch_es_pre<T>((const cpx<T> *)m->S1, (cpx<T> *)m->G, es_plane(*m), m->es_cs, c->st, c->stream, sel),
                "es_pre");
            (*count)++;
        }
        for (int part = 1; part <= 3; part++)
            if (int rc = ml_enqueue_part<T>(c, part, gate_yz, bi, count)) return rc;
        for (Mesh *m : tg) {
            CKL(launch_es_post<T>((const cpx<T> *)m->S1, (cpx<T> *)m->G, es_plane(*m), c->st, c->stream, sel), "es_post");
            (*count)++;
        }
        CKL(launch_es_commit(c->st, c->stream, sel), "es_commit");
        (*count)++;
    }
    if (mode != 1) {
        for (Mesh *m : tg) {
            CKL(launch_es_extrap<T>((cpx<T> *)m->S1, (const cpx<T> *)m->G, es_plane(*m), m->es_cs, c->st, c_eval,
                                    c->stream, sel), "es_extrap");
            (*count)++;
        }
    }
    return ml_enqueue_part<T>(c, 4, gate_xt, bi, count);
}

template <typename T>
int enqueue_rk4_step(bm_ctx *c, int *count, void *const *cacheX = nullptr, void *const *cacheH = nullptr, void *cacheY = nullptr)
{
    // buffers: 0 = M (step start, sM1), 2 = B, 3 = C ; evals 0..2
    // cacheX/cacheH/cacheY (adjoint recompute, one mesh): each stage's input M, its field, and the
    // update before renormalisation are also written there
    const int nm = (int)c->meshes.size();
    static const int min_buf[4] = {0, 2, 3, 2};
    static const double c_eval[4] = {0.0, 0.5, 0.5, 1.0};   // RK4 evaluation times (Get_EvalStep_Time)
    for (int s = 0; s < 4; s++) {
        // the evaluation-speedup kernels are not batched: nothing to record in the batched plan's
        // collect pass (which must launch nothing)
        const bool es_launch = !c->bp.collect;
        const bool es_tab = c->es_tab != nullptr;
        if (c->es_level > 0 && s == 0 && c->ml) {
            if (int rc = enqueue_ml_es<T>(c, 1, BM_GATE_ALWAYS, BM_GATE_ALWAYS, 0.0, min_buf[s], count)) return rc;
        } else if (c->es_level > 0 && s == 0) {
            // evaluation speedup: compute and save the field at the first evaluation of the step
            if (es_tab && es_launch) {
                CKL(launch_es_pre_batch<T>(c->es_tab, c->es_nmesh, c->es_max_plane, c->st, c->stream), "es_pre_batch");
                (*count)++;
            }
            for (auto &m : c->meshes) {
                if (!(m.modules & BM_DEMAG) || !es_launch || es_tab) continue;
                CKL(launch_es_pre<T>((const cpx<T> *)m.S1, (cpx<T> *)m.G, es_plane(m), m.es_cs, c->st, c->stream), "es_pre");
                (*count)++;
            }
            if (int rc = enqueue_fields<T>(c, BM_GATE_ALWAYS, min_buf[s], count)) return rc;
            if (es_tab && es_launch) {
                CKL(launch_es_post_batch<T>(c->es_tab, c->es_nmesh, c->es_max_plane, c->st, c->stream), "es_post_batch");
                (*count)++;
            }
            for (auto &m : c->meshes) {
                if (!(m.modules & BM_DEMAG) || !es_launch || es_tab) continue;
                CKL(launch_es_post<T>((const cpx<T> *)m.S1, (cpx<T> *)m.G, es_plane(m), c->st, c->stream), "es_post");
                (*count)++;
            }
            if (es_launch) {
                CKL(launch_es_commit(c->st, c->stream), "es_commit");
                (*count)++;
            }
        } else if (c->es_level > 0 && c->es_phase != 2) {
            // too few fields saved yet: the full field
            if (int rc = enqueue_fields<T>(c, BM_GATE_ALWAYS, min_buf[s], count)) return rc;
        } else if (c->es_level > 0 && c->ml) {
            if (int rc = enqueue_ml_es<T>(c, 2, BM_GATE_ALWAYS, BM_GATE_ALWAYS, c_eval[s], min_buf[s], count)) return rc;
        } else if (c->es_level > 0) {
            // the extrapolation in place of the y/z passes
            if (es_tab && es_launch) {
                CKL(launch_es_extrap_batch<T>(c->es_tab, c->es_nmesh, c->es_max_plane, c->st, c_eval[s], c->stream),
                    "es_extrap_batch");
                (*count)++;
            }
            for (auto &m : c->meshes) {
                if (!(m.modules & BM_DEMAG) || !es_launch || es_tab || es_fold_ok(c, m)) continue;
                CKL(launch_es_extrap<T>((cpx<T> *)m.S1, (const cpx<T> *)m.G, es_plane(m), m.es_cs, c->st, c_eval[s],
                                        c->stream), "es_extrap");
                (*count)++;
            }
            if (!es_tab) { c->es_fold_pending = 1; c->es_fold_ceval = c_eval[s]; }
        } else {
            int rc = enqueue_fields<T>(c, BM_GATE_ALWAYS, min_buf[s], count);
            if (rc) return rc;
        }
        std::vector<StageArgs<T>> v;
        for (int i = 0; i < nm; i++) {
            Mesh &m = c->meshes[i];
            StageArgs<T> a = stage_args<T>(c, m);
            a.mode = BM_MODE_STAGE;
            a.Mbase = B<T>(m, 0);
            if (s == 0) {
                a.Min = B<T>(m, 0); a.ev_out = E<T>(m, 0); a.crhs = 0.5; a.Mout = B<T>(m, 2);
                a.diag = BM_DIAG_MXH | (i == nm - 1 ? BM_DIAG_PUBLISH : 0);   // the step's first evaluation
            }
            else if (s == 1) { a.Min = B<T>(m, 2); a.ev_out = E<T>(m, 1); a.crhs = 0.5; a.Mout = B<T>(m, 3); }
            else if (s == 2) { a.Min = B<T>(m, 3); a.ev_out = E<T>(m, 2); a.crhs = 1.0; a.Mout = B<T>(m, 2); }
            else {
                a.Min = B<T>(m, 2);
                a.nev = 3;
                a.ev[0] = E<T>(m, 0); a.ev[1] = E<T>(m, 1); a.ev[2] = E<T>(m, 2);
                a.cev[0] = 1.0 / 6; a.cev[1] = 2.0 / 6; a.cev[2] = 2.0 / 6;
                a.crhs = 1.0 / 6;
                a.Mout = B<T>(m, 0);
                a.renorm = 1;
                a.diag = BM_DIAG_DMDT | (i == nm - 1 ? BM_DIAG_PUBLISH : 0);   // the step's last stage
                if (i == nm - 1) a.last_kind = BM_LAST_FINISH;
            }
            if (cacheX) {
                a.copy_to = (T *)cacheX[s];
                a.Hsave = (T *)cacheH[s];
                if (s == 3) a.Ysave = (T *)cacheY;
            }
            es_fold_args<T>(c, m, a);
            v.push_back(a);
        }
        c->es_fold_pending = 0;
        if (int rc = stage_multi<T>(c, v, count)) return rc;
    }
    return 0;
}

// One RKDP54 field evaluation with the evaluation speedup: the device decides (k_es_decide) whether
// it computes and saves the field or extrapolates; the save kernels, the y / z passes and the
// extrapolation are all captured and each runs or skips on that decision.
template <typename T>
int enqueue_es_fields_dp(bm_ctx *c, int eval, double c_eval, int bi, int *count)
{
    const bool launch = !c->bp.collect;   // the speedup kernels are not part of a batched plan
    const bool tab = c->es_tab != nullptr;
    if (c->ml) {
        CKL(launch_es_decide(c->st, eval, c_eval, c->stream), "es_decide");
        (*count)++;
        return enqueue_ml_es<T>(c, 3, eval ? BM_GATE_ACCEPTED : BM_GATE_ALWAYS, eval ? BM_GATE_ES_ACC : BM_GATE_ES, c_eval,
                                bi, count);
    }
    if (launch) {
        CKL(launch_es_decide(c->st, eval, c_eval, c->stream), "es_decide");
        (*count)++;
        if (tab) {
            CKL(launch_es_pre_batch<T>(c->es_tab, c->es_nmesh, c->es_max_plane, c->st, c->stream, 1), "es_pre_batch");
            (*count)++;
        } else {
            for (auto &m : c->meshes) {
                if (!(m.modules & BM_DEMAG)) continue;
                CKL(launch_es_pre<T>((const cpx<T> *)m.S1, (cpx<T> *)m.G, es_plane(m), m.es_cs, c->st, c->stream, 1), "es_pre");
                (*count)++;
            }
        }
    }
    if (int rc = enqueue_fields<T>(c, eval ? BM_GATE_ES_ACC : BM_GATE_ES, bi, count)) return rc;
    if (!launch) return 0;
    if (tab) {
        CKL(launch_es_post_batch<T>(c->es_tab, c->es_nmesh, c->es_max_plane, c->st, c->stream, 1), "es_post_batch");
        (*count)++;
    } else {
        for (auto &m : c->meshes) {
            if (!(m.modules & BM_DEMAG)) continue;
            CKL(launch_es_post<T>((const cpx<T> *)m.S1, (cpx<T> *)m.G, es_plane(m), c->st, c->stream, 1), "es_post");
            (*count)++;
        }
    }
    CKL(launch_es_commit(c->st, c->stream, 1), "es_commit");
    (*count)++;
    if (tab) {
        CKL(launch_es_extrap_batch<T>(c->es_tab, c->es_nmesh, c->es_max_plane, c->st, c_eval, c->stream, 1), "es_extrap_batch");
        (*count)++;
    } else {
        for (auto &m : c->meshes) {
            if (!(m.modules & BM_DEMAG) || es_fold_ok(c, m)) continue;
            CKL(launch_es_extrap<T>((cpx<T> *)m.S1, (const cpx<T> *)m.G, es_plane(m), m.es_cs, c->st, c_eval, c->stream, 1),
                "es_extrap");
            (*count)++;
        }
        c->es_fold_pending = 2;
        c->es_fold_ceval = c_eval;
    }
    return 0;
}

template <typename T>
int enqueue_rkdp_attempt(bm_ctx *c, int *count)
{
    // evaluation times of the Dormand-Prince stages (Get_EvalStep_Time, Boris/DiffEq_CommonBase_Iterate.cpp:1562)
    static const double c_dp[6] = {0.0, 0.2, 0.3, 0.8, 8.0 / 9, 1.0};
    const bool es = c->es_level > 0;
    // buffers: 0 = M, 1 = P (sM1), 2 = B, 3 = C ; evals 0..5
    const int nm = (int)c->meshes.size();
    // restore after a rejection: M = sM1 and its x transform
    {
        std::vector<StageArgs<T>> v;
        for (int i = 0; i < nm; i++) {
            Mesh &m = c->meshes[i];
            StageArgs<T> a = stage_args<T>(c, m);
            a.mode = BM_MODE_UPDATE;
            a.gate = BM_GATE_RESTORE;
            a.Min = B<T>(m, 1); a.Mbase = B<T>(m, 1); a.Mout = B<T>(m, 0);
            if (i == nm - 1) a.last_kind = BM_LAST_RESTORED;
            v.push_back(a);
        }
        if (int rc = stage_multi<T>(c, v, count)) return rc;
    }
    // evaluation 0: FSAL rhs + error of the previous step + controller
    {
        int rc = es ? enqueue_es_fields_dp<T>(c, 0, c_dp[0], 0, count) : enqueue_fields<T>(c, BM_GATE_ALWAYS, 0, count);
        if (rc) return rc;
    }
    static const double bs[5] = {5179.0 / 57600, 7571.0 / 16695, 393.0 / 640, -92097.0 / 339200, 187.0 / 2100};
    // 5th-order weights of k0, k2, k3, k4, k5 (k1 has none)
    static const double as5[5] = {35.0 / 384, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84};
    {
        std::vector<StageArgs<T>> v;
        for (int i = 0; i < nm; i++) {
            Mesh &m = c->meshes[i];
            StageArgs<T> a = stage_args<T>(c, m);
            a.mode = BM_MODE_LTE;
            a.do_xfwd = 0;
            a.Min = B<T>(m, 0); a.Mbase = B<T>(m, 1);
            a.nev = 5;
            a.ev[0] = E<T>(m, 0); a.ev[1] = E<T>(m, 2); a.ev[2] = E<T>(m, 3); a.ev[3] = E<T>(m, 4); a.ev[4] = E<T>(m, 5);
            for (int k = 0; k < 5; k++) a.cev[k] = bs[k];
            a.crhs = 1.0 / 40;
            if (sizeof(T) == 4) {
                // mixed precision: the reference's |M - prediction| (Boris/DiffEqFM_Evals_RKDP54.cpp:72-76)
                // with M, the renormalised 5th-order solution, recomputed in FP64 from sM1 and the stage
                // rhs; the FP32-stored M would add its rounding (~1e-7 relative), a floor under the error
                // estimate that holds small steps back
                for (int k = 0; k < 5; k++) a.cev5[k] = as5[k];
                a.lte_embedded = 1;
            }
            a.ev_out = E<T>(m, 0);
            a.diag = BM_DIAG_MXH | (i == nm - 1 ? BM_DIAG_PUBLISH : 0);   // evaluation 0 at the step's M
            if (i == nm - 1) a.last_kind = BM_LAST_CONTROL;
            es_fold_args<T>(c, m, a);
            v.push_back(a);
        }
        c->es_fold_pending = 0;
        if (int rc = stage_multi<T>(c, v, count)) return rc;
    }
    // advance: sM1 = M, M1 = M + dT/5 k0
    {
        std::vector<StageArgs<T>> v;
        for (int i = 0; i < nm; i++) {
            Mesh &m = c->meshes[i];
            StageArgs<T> a = stage_args<T>(c, m);
            a.mode = BM_MODE_UPDATE;
            a.gate = BM_GATE_ACCEPTED;
            a.Min = B<T>(m, 0); a.Mbase = B<T>(m, 0); a.copy_to = B<T>(m, 1);
            a.nev = 1; a.ev[0] = E<T>(m, 0); a.cev[0] = 0.2;
            a.Mout = B<T>(m, 2);
            v.push_back(a);
        }
        if (int rc = stage_multi<T>(c, v, count)) return rc;
    }
    static const double av[6][6] = {
        {0},
        {3.0 / 40, 9.0 / 40},
        {44.0 / 45, -56.0 / 15, 32.0 / 9},
        {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729},
        {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656},
        {35.0 / 384, 0.0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
    for (int s = 1; s <= 5; s++) {
        {
            const int bi = (s % 2 == 1) ? 2 : 3;
            int rc = es ? enqueue_es_fields_dp<T>(c, s, c_dp[s], bi, count) : enqueue_fields<T>(c, BM_GATE_ACCEPTED, bi, count);
            if (rc) return rc;
        }
        std::vector<StageArgs<T>> v;
        for (int i = 0; i < nm; i++) {
            Mesh &m = c->meshes[i];
            StageArgs<T> a = stage_args<T>(c, m);
            a.mode = BM_MODE_STAGE;
            a.gate = BM_GATE_ACCEPTED;
            a.Min = (s % 2 == 1) ? B<T>(m, 2) : B<T>(m, 3);
            a.Mbase = B<T>(m, 1);
            a.ev_out = E<T>(m, s);
            a.nev = 0;
            for (int e = 0; e < s; e++) {
                if (av[s][e] == 0.0) continue;
                a.ev[a.nev] = E<T>(m, e);
                a.cev[a.nev] = av[s][e];
                a.nev++;
            }
            a.crhs = av[s][s];
            if (s < 5) a.Mout = (s % 2 == 1) ? B<T>(m, 3) : B<T>(m, 2);
            else {
                a.Mout = B<T>(m, 0);
                a.renorm = 1;
                a.diag = BM_DIAG_DMDT | (i == nm - 1 ? BM_DIAG_PUBLISH : 0);   // the 5th-order state
                if (i == nm - 1) a.last_kind = BM_LAST_FINISH;
            }
            es_fold_args<T>(c, m, a);
            v.push_back(a);
        }
        c->es_fold_pending = 0;
        if (int rc = stage_multi<T>(c, v, count)) return rc;
    }
    return 0;
}

template <typename T>
int build_graph(bm_ctx *c)
{
    drop_graph(c);
    int count = 0;
    // evaluation speedup: under RK4 one graph for the steps that still save fields, one for the
    // extrapolating steps; under RKDP54 one graph whose evaluations decide on the device
    const bool es = c->es_level > 0 && c->eval == BM_RK4;
    if (c->es_level > 0 && c->batched && c->meshes.size() > 1) {
        std::vector<EsMesh> tab;
        for (auto &m : c->meshes) {
            if (!(m.modules & BM_DEMAG)) continue;
            EsMesh e;
            e.S1 = m.S1; e.G = m.G; e.plane = es_plane(m);
            for (int k = 0; k < 3; k++) e.cs[k] = m.es_cs[k];
            tab.push_back(e);
            if (e.plane > c->es_max_plane) c->es_max_plane = e.plane;
        }
        if (!tab.empty()) {
            if (cudaMalloc(&c->es_tab, sizeof(EsMesh) * tab.size()) != cudaSuccess) return fail(BM_ENOMEM, "evaluation speedup table");
            CK(cudaMemcpy(c->es_tab, tab.data(), sizeof(EsMesh) * tab.size(), cudaMemcpyHostToDevice));
            c->es_nmesh = (int)tab.size();
        }
    }
    if (c->batched && c->meshes.size() > 1) {
        // pass 1: collect the batched launches' argument blocks and work lists (of both steps, in
        // capture order, with evaluation speedup), upload them
        c->bp = BatchPlan();
        c->bp.collect = true;
        int rc = 0;
        for (int phase = 1; phase <= (es ? 2 : 1) && !rc; phase++) {
            c->es_phase = es ? phase : 0;
            rc = (c->eval == BM_RKDP54) ? enqueue_rkdp_attempt<T>(c, &count) : enqueue_rk4_step<T>(c, &count);
        }
        c->es_phase = 0;
        c->bp.collect = false;
        if (rc) return rc;
        if (!c->bp.hbuf.empty()) {
            if (cudaMalloc(&c->bp.dbuf, c->bp.hbuf.size()) != cudaSuccess) return fail(BM_ENOMEM, "batched launch plan");
            CK(cudaMemcpy(c->bp.dbuf, c->bp.hbuf.data(), c->bp.hbuf.size(), cudaMemcpyHostToDevice));
        }
        c->bp.next = 0;
        count = 0;
    }
    for (int phase = 1; phase <= (es ? 2 : 1); phase++) {
        c->es_phase = es ? phase : 0;
        count = 0;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = (c->eval == BM_RKDP54) ? enqueue_rkdp_attempt<T>(c, &count) : enqueue_rk4_step<T>(c, &count);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        c->es_phase = 0;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return fail(BM_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        if (phase == 1) {
            c->graph = g;
            CK(cudaGraphInstantiate(&c->gexec, g, 0));
        } else {
            c->graph_es = g;
            CK(cudaGraphInstantiate(&c->gexec_es, g, 0));
        }
    }
    c->graph_eval = c->eval;
    c->kernels_per_step = count;
    return 0;
}

template <typename T>
int run_T(bm_ctx *c, int steps)
{
    if (c->s1_dirty) {
        int cnt = 0;
        int rc = enqueue_prime<T>(c, &cnt);
        if (rc) return rc;
        c->s1_dirty = false;
    }
    if (!c->gexec || c->graph_eval != c->eval) {
        int rc = build_graph<T>(c);
        if (rc) return rc;
    }
    int rc = read_state(c);
    if (rc) return rc;
    if (c->host_st.error & BM_ERR_NONFINITE)
        return fail(BM_ENONFINITE, "the state is not finite (NaN or infinity): set a new M before running");
    long long target = c->host_st.accepted + steps;
    long long guard = 0;
    while (c->host_st.accepted < target) {
        long long k = target - c->host_st.accepted;
        // evaluation speedup: every step saves one more field (up to es_K) at its first evaluation;
        // a step whose save brings the count to es_K already extrapolates its other evaluations, so
        // gexec (full evaluations) runs while fewer than es_K - 1 are saved at the step start
        long long warm = k;
        if (c->gexec_es) {
            long long need = (long long)c->host_st.es_K - 1 - c->host_st.es_saved;
            warm = need > 0 ? (need < k ? need : k) : 0;
        }
        for (long long i = 0; i < warm; i++) CK(cudaGraphLaunch(c->gexec, c->stream));
        for (long long i = warm; i < k; i++) CK(cudaGraphLaunch(c->gexec_es, c->stream));
        guard += k;
        if ((rc = read_state(c))) return rc;
        if (c->host_st.error & BM_ERR_WAIT)
            return fail(BM_ECUDA, "a kernel's bounded wait for its bulk tensor copies gave up");
        if (c->host_st.error & BM_ERR_NONFINITE)
            return fail(BM_ENONFINITE, c->eval == BM_RK4
                                           ? "a step produced a non-finite M (NaN or infinity); its steps are counted"
                                           : "a step produced a non-finite M (NaN or infinity); it was not accepted");
        if (c->eval == BM_RK4) break;
        if (guard > 100LL * steps + 1000) return fail(BM_ESTATE, "step control did not converge");
    }
    return 0;
}

template <typename T>
int compute_field_T(bm_ctx *c, Mesh &m, int modules_mask, double *H)
{
    int cnt = 0;
    if ((m.modules & BM_DEMAG) && m.ml_role) {
        // x transforms of the layers that live on their mesh's grid, then the whole convolution
        for (auto &mm : c->meshes) {
            if (mm.ml_role != 1) continue;
            StageArgs<T> a = stage_args<T>(c, mm);
            a.mode = BM_MODE_UPDATE;
            a.Min = B<T>(mm, 0); a.Mbase = B<T>(mm, 0);
            CKL(launch_stage<T>(a, c->stream), "xfwd");
        }
        int rc = enqueue_fields<T>(c, BM_GATE_ALWAYS, 0, &cnt);
        if (rc) return rc;
    } else if (m.modules & BM_DEMAG) {
        StageArgs<T> a = stage_args<T>(c, m);
        a.mode = BM_MODE_UPDATE;
        a.Min = B<T>(m, 0); a.Mbase = B<T>(m, 0);
        CKL(launch_stage<T>(a, c->stream), "xfwd");
        int rc = enqueue_yz<T>(c, m, BM_GATE_ALWAYS, &cnt);
        if (rc) return rc;
    }
    StageArgs<T> a = stage_args<T>(c, m);
    a.mode = BM_MODE_HEFF;
    a.modules = m.modules & modules_mask;
    a.do_xfwd = 0;
    if (m.ml_role == 2) {
        a.modules &= ~BM_DEMAG;
        a.Hd = (modules_mask & BM_DEMAG) ? (const T *)m.Hd : nullptr;
    }
    a.Min = B<T>(m, 0);
    a.Hout = (T *)m.Hout;
    CKL(launch_stage<T>(a, c->stream), "heff");
    CKL(launch_planes_to_aos<T>(m.stage64, (const T *)m.Hout, m.n, c->stream), "planes_to_aos");
    CK(cudaMemcpyAsync(H, m.stage64, sizeof(double) * 3 * m.n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->s1_dirty = true;
    return 0;
}

// ------------------------------------------------------------------ discrete adjoint of RK4
// Forward: the step graph with a checkpoint of M and the time every k steps. Backward, per segment
// from the last: restore the checkpoint, replay a captured graph that recomputes the segment's k
// steps with the fused stage kernels also writing each stage's input, field and pre-normalisation
// update into a k-slot cache, then replay a captured graph that walks the k steps in reverse
// (renormalisation VJP, then per stage the LLG / local-field VJP, the demag of gH through the
// convolution pipeline, and the Laplacian / accumulation kernel). Gradients accumulate in FP64;
// the Zeeman gradient of each step is summed per step and mapped to its sample on the host with
// the step start time the device used.
struct AdjBufs {
    std::vector<void *> all;
    void *get(size_t bytes, bool zero, cudaStream_t s)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        if (zero) cudaMemsetAsync(p, 0, bytes, s);
        all.push_back(p);
        return p;
    }
    ~AdjBufs() { for (auto p : all) cudaFree(p); }
};

template <typename T>
int adjoint_T(bm_ctx *c, int steps, int k, const double *target, int m0_scales, double *loss, double *gMs_h, double *gK1_h,
              double *gHa_h, double *times2)
{
    Mesh &m = c->meshes[0];
    cudaStream_t s = c->stream;
    const long long n = m.n;
    const size_t v3 = sizeof(T) * 3 * (size_t)n;
    const int S = steps / k;
    AdjBufs ab;
    auto need = [&](void *p) { return p != nullptr; };
    // forward with checkpoints
    if (c->s1_dirty) {
        int cnt = 0;
        if (int rc = enqueue_prime<T>(c, &cnt)) return rc;
        c->s1_dirty = false;
    }
    if (!c->gexec || c->graph_eval != c->eval) {
        if (int rc = build_graph<T>(c)) return rc;
    }
    if (int rc = read_state(c)) return rc;
    const StepState st0 = c->host_st;
    void *ckM = ab.get(v3 * S, false, s), *ckT = ab.get(sizeof(double) * S, false, s);
    if (!need(ckM) || !need(ckT)) return fail(BM_ENOMEM, "adjoint checkpoints");
    cudaEvent_t e0, e1, e2, e3;
    CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1)); CK(cudaEventCreate(&e2)); CK(cudaEventCreate(&e3));
    CK(cudaEventRecord(e0, s));
    for (int g = 0; g < S; g++) {
        CK(cudaMemcpyAsync((char *)ckM + v3 * g, m.buf[0], v3, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync((double *)ckT + g, &c->st->time, sizeof(double), cudaMemcpyDeviceToDevice, s));
        for (int q = 0; q < k; q++) CK(cudaGraphLaunch(c->gexec, s));
    }
    CK(cudaEventRecord(e1, s));
    if (int rc = read_state(c)) return rc;
    const StepState st_end = c->host_st;
    std::vector<double> tck(S);
    CK(cudaMemcpy(tck.data(), ckT, sizeof(double) * S, cudaMemcpyDeviceToHost));
    // adjoint buffers
    void *Mfin = ab.get(v3, false, s), *tgt = ab.get(sizeof(double) * 3 * n, false, s);
    void *lam = ab.get(v3, true, s), *lamY = ab.get(v3, true, s), *mu = ab.get(v3, true, s), *gH = ab.get(v3, true, s);
    void *gXd = ab.get(v3, true, s), *w = ab.get(v3, true, s), *gD = ab.get(v3, true, s);
    void *gMs = ab.get(sizeof(double) * n, true, s), *gK1 = ab.get(sizeof(double) * n, true, s);
    void *gHs = ab.get(sizeof(double) * 3 * k, true, s), *gHall = ab.get(sizeof(double) * 3 * (size_t)steps, true, s);
    void *lossd = ab.get(sizeof(double), true, s);
    void *cache = ab.get(v3 * 9 * (size_t)k, false, s);
    for (void *p : {Mfin, tgt, lam, lamY, mu, gH, gXd, w, gD, gMs, gK1, gHs, gHall, lossd, cache})
        if (!need(p)) return fail(BM_ENOMEM, "adjoint buffers");
    auto slot = [&](int j, int q) -> void * { return (char *)cache + v3 * (9 * (size_t)j + q); };   // 0..3 X, 4..7 H, 8 Y
    CK(cudaMemcpyAsync(Mfin, m.buf[0], v3, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(tgt, target, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    AdjArgs<T> aa;
    memset(&aa, 0, sizeof(aa));
    aa.nx = m.nx; aa.ny = m.ny; aa.nz = m.nz; aa.n = n;
    aa.hx = (T)m.h[0]; aa.hy = (T)m.h[1]; aa.hz = (T)m.h[2];
    aa.Ms_map = (const T *)m.Msd; aa.K1_map = (const T *)m.K1d;
    aa.Ms = (T)m.Ms; aa.K1 = (T)m.K1; aa.A = (T)m.A; aa.alpha = (T)m.alpha; aa.grel = (T)m.grel;
    double en = std::sqrt(m.ea[0] * m.ea[0] + m.ea[1] * m.ea[1] + m.ea[2] * m.ea[2]);
    for (int q = 0; q < 3; q++) aa.ea[q] = (T)(en > 0 ? m.ea[q] / en : 0.0);
    aa.modules = m.modules;
    for (int q = 0; q < 3; q++) aa.pbc[q] = (m.pbc[q] > 0) - (m.pbc[q] < 0);
    const double dt = c->dt;
    // the two segment graphs
    cudaGraph_t gr = nullptr, gb = nullptr;
    cudaGraphExec_t xr = nullptr, xb = nullptr;
    int cnt = 0, rc = 0;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_prime<T>(c, &cnt);
    for (int j = 0; j < k && !rc; j++) {
        void *cx[4] = {slot(j, 0), slot(j, 1), slot(j, 2), slot(j, 3)}, *ch[4] = {slot(j, 4), slot(j, 5), slot(j, 6), slot(j, 7)};
        rc = enqueue_rk4_step<T>(c, &cnt, cx, ch, slot(j, 8));
    }
    cudaError_t ce = cudaStreamEndCapture(s, &gr);
    if (rc || ce != cudaSuccess) { if (gr) cudaGraphDestroy(gr); return rc ? rc : fail(BM_ECUDA, "adjoint recompute capture"); }
    CK(cudaGraphInstantiate(&xr, gr, 0));
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    static const double cYs[4] = {0.0, 1.0 / 6, 1.0 / 3, 1.0 / 3}, cXs[4] = {0.0, 0.5, 0.5, 1.0};
    for (int j = k - 1; j >= 0 && !rc; j--) {
        rc = launch_adj_renorm<T>(aa, (T *)lam, (const T *)slot(j, 8), (T *)lamY, (T *)mu, dt, (double *)gMs, s);
        for (int q = 3; q >= 0 && !rc; q--) {
            rc = launch_adj_vjp_a<T>(aa, (const T *)slot(j, q), (const T *)slot(j, 4 + q), (const T *)mu, (T *)gH, (T *)gXd,
                                     (T *)w, (double *)gMs, (double *)gK1, (double *)gHs + 3 * j, s);
            if (!rc && (m.modules & BM_DEMAG)) {
                // gD = D gH through the convolution pipeline
                StageArgs<T> a = stage_args<T>(c, m);
                a.mode = BM_MODE_UPDATE;
                a.Min = (const T *)gH; a.Mbase = (const T *)gH;
                a.st = nullptr;
                rc = launch_stage<T>(a, s);
                if (!rc) rc = enqueue_yz<T>(c, m, BM_GATE_ALWAYS, &cnt);
                if (!rc) {
                    StageArgs<T> b = stage_args<T>(c, m);
                    b.mode = BM_MODE_HEFF;
                    b.modules = BM_DEMAG;
                    b.do_xfwd = 0;
                    b.st = nullptr;
                    b.Min = (const T *)gH;
                    b.Hout = (T *)gD;
                    rc = launch_stage<T>(b, s);
                }
            }
            if (!rc)
                rc = launch_adj_vjp_c<T>(aa, (const T *)gXd, (const T *)w, (m.modules & BM_DEMAG) ? (const T *)gD : nullptr,
                                         (const T *)lamY, (T *)lam, (T *)mu, cYs[q] * dt, cXs[q] * dt, q > 0 ? 1 : 0, s);
        }
    }
    ce = cudaStreamEndCapture(s, &gb);
    if (rc || ce != cudaSuccess) {
        if (gb) cudaGraphDestroy(gb);
        cudaGraphExecDestroy(xr); cudaGraphDestroy(gr);
        return rc ? fail(BM_ECUDA, "adjoint backward launch failed (" + std::to_string(rc) + ")") : fail(BM_ECUDA, "adjoint capture");
    }
    cudaError_t ie = cudaGraphInstantiate(&xb, gb, 0);
    if (ie != cudaSuccess) { cudaGraphDestroy(gb); cudaGraphExecDestroy(xr); cudaGraphDestroy(gr); return fail(BM_ECUDA, "adjoint instantiate"); }
    // backward sweep
    CK(cudaEventRecord(e2, s));
    rc = launch_adj_loss<T>(aa, (const T *)Mfin, (const double *)tgt, (T *)lam, (double *)gMs, (double *)lossd, s);
    for (int g = S - 1; g >= 0 && !rc; g--) {
        CK(cudaMemcpyAsync(m.buf[0], (char *)ckM + v3 * g, v3, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(&c->st->time, (double *)ckT + g, sizeof(double), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(&c->st->stagetime, (double *)ckT + g, sizeof(double), cudaMemcpyDeviceToDevice, s));
        CK(cudaGraphLaunch(xr, s));
        CK(cudaGraphLaunch(xb, s));
        CK(cudaMemcpyAsync((double *)gHall + 3 * (size_t)k * g, gHs, sizeof(double) * 3 * k, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemsetAsync(gHs, 0, sizeof(double) * 3 * k, s));
    }
    if (!rc && m0_scales) rc = launch_adj_m0<T>(aa, (const T *)ckM, (const T *)lam, (double *)gMs, s);
    CK(cudaEventRecord(e3, s));
    CK(cudaStreamSynchronize(s));
    cudaGraphExecDestroy(xb); cudaGraphDestroy(gb);
    cudaGraphExecDestroy(xr); cudaGraphDestroy(gr);
    if (rc) return fail(BM_ECUDA, "adjoint launch failed (" + std::to_string(rc) + ")");
    float f_ms = 0.f, b_ms = 0.f;
    cudaEventElapsedTime(&f_ms, e0, e1);
    cudaEventElapsedTime(&b_ms, e2, e3);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
    if (times2) { times2[0] = f_ms; times2[1] = b_ms; }
    // results
    CK(cudaMemcpy(loss, lossd, sizeof(double), cudaMemcpyDeviceToHost));
    if (gMs_h) CK(cudaMemcpy(gMs_h, gMs, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (gK1_h) CK(cudaMemcpy(gK1_h, gK1, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (gHa_h) {
        const int nHa = m.nHa;
        for (int q = 0; q < 3 * nHa; q++) gHa_h[q] = 0.0;
        if ((m.modules & BM_ZEEMAN) && nHa > 0) {
            std::vector<double> gall(3 * (size_t)steps);
            CK(cudaMemcpy(gall.data(), gHall, sizeof(double) * 3 * steps, cudaMemcpyDeviceToHost));
            for (int g = 0; g < S; g++) {
                double t = tck[g];
                for (int j = 0; j < k; j++) {
                    int hi = 0;
                    if (nHa > 1 && m.Ha_tspan > 0.0) {
                        hi = (int)std::floor(t / m.Ha_tspan * nHa);
                        hi = hi < 0 ? 0 : (hi >= nHa ? nHa - 1 : hi);
                    }
                    for (int q = 0; q < 3; q++) gHa_h[3 * hi + q] += gall[3 * ((size_t)g * k + j) + q];
                    t = t + dt;
                }
            }
        }
    }
    // leave the context at the end of the forward run
    CK(cudaMemcpy(m.buf[0], Mfin, v3, cudaMemcpyDeviceToDevice));
    c->host_st = st_end;
    CK(cudaMemcpy(c->st, &c->host_st, sizeof(StepState), cudaMemcpyHostToDevice));
    c->s1_dirty = true;
    (void)st0;
    return 0;
}

int check_ctx(bm_ctx *c) { return c ? 0 : fail(BM_EINVAL, "null context"); }
int check_mesh(bm_ctx *c, int mesh)
{
    if (!c) return fail(BM_EINVAL, "null context");
    if (mesh < 0 || mesh >= (int)c->meshes.size()) return fail(BM_EINVAL, "bad mesh index");
    return 0;
}

}  // namespace

// error text for entry points defined in other translation units
int bm_set_error(int code, const std::string &msg) { return fail(code, msg); }

// =============================================================================== C ABI
extern "C" {

const char *bm_last_error(void) { return g_err.c_str(); }
int bm_version(void) { return 1; }

int bm_create(int device, bm_ctx **out)
{
    if (!out) return fail(BM_EINVAL, "null out");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return fail(BM_ECUDA, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(BM_EINVAL, "bad device index");
    bm_ctx *c = new bm_ctx();
    c->device = device;
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return fail(BM_ECUDA, "stream"); }
    if (cudaMalloc(&c->st, sizeof(StepState)) != cudaSuccess) { delete c; return fail(BM_ENOMEM, "state"); }
    if (cudaMalloc(&c->farq, sizeof(double) * 6 * BM_FARQ_PER_COMP) != cudaSuccess) { delete c; return fail(BM_ENOMEM, "farq"); }
    memset(&c->host_st, 0, sizeof(StepState));
    *out = c;
    return 0;
}

int bm_destroy(bm_ctx *c)
{
    if (!c) return 0;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    for (auto &m : c->meshes) free_mesh(m);
    if (c->st) cudaFree(c->st);
    if (c->farq) cudaFree(c->farq);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return 0;
}

int bm_add_mesh(bm_ctx *c, int nx, int ny, int nz, double hx, double hy, double hz, double ox, double oy, double oz, int *mesh_id)
{
    if (int rc = check_ctx(c)) return rc;
    if (nx < 1 || ny < 1 || nz < 1) return fail(BM_EINVAL, "mesh dimensions must be >= 1");
    if (!(hx > 0 && hy > 0 && hz > 0)) return fail(BM_EINVAL, "cellsize must be > 0");
    if ((long long)nx * ny * nz > (1LL << 31)) return fail(BM_EINVAL, "mesh too large");
    if (nice_size(nx) > 4096 || nice_size(ny) > 4096 || nice_size(nz) > 2048) return fail(BM_EUNSUPPORTED, "mesh dimension above the supported FFT size");
    unprepare(c);
    Mesh m;
    m.nx = nx; m.ny = ny; m.nz = nz;
    m.h[0] = hx; m.h[1] = hy; m.h[2] = hz;
    m.o[0] = ox; m.o[1] = oy; m.o[2] = oz;
    m.n = (long long)nx * ny * nz;
    m.M0.assign(3 * (size_t)m.n, 0.0);
    for (long long i = 0; i < m.n; i++) m.M0[3 * i] = m.Ms;
    c->meshes.push_back(m);
    if (mesh_id) *mesh_id = (int)c->meshes.size() - 1;
    return 0;
}

int bm_set_material(bm_ctx *c, int mesh, double Ms, double A, double alpha, double grel, double K1, double K2, const double *ea3, double D)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!(Ms > 0)) return fail(BM_EINVAL, "Ms must be > 0");
    unprepare(c);
    Mesh &m = c->meshes[mesh];
    m.Ms = Ms; m.A = A; m.alpha = alpha; m.grel = grel; m.K1 = K1; m.K2 = K2; m.D = D;
    if (ea3) { m.ea[0] = ea3[0]; m.ea[1] = ea3[1]; m.ea[2] = ea3[2]; }
    return 0;
}

int bm_set_material_maps(bm_ctx *c, int mesh, const double *Ms_map, const double *K1_map)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    unprepare(c);
    Mesh &m = c->meshes[mesh];
    if (Ms_map) {
        for (long long i = 0; i < m.n; i++) if (!(Ms_map[i] > 0)) return fail(BM_EINVAL, "Ms map values must be > 0");
        m.Ms_map.assign(Ms_map, Ms_map + m.n);
    } else m.Ms_map.clear();
    if (K1_map) m.K1_map.assign(K1_map, K1_map + m.n);
    else m.K1_map.clear();
    return 0;
}

int bm_set_pbc(bm_ctx *c, int mesh, int x_images, int y_images, int z_images)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    const int img[3] = {x_images, y_images, z_images};
    for (int a = 0; a < 3; a++)
        if (img[a] > BM_PBC_MAX_IMAGES || img[a] < -BM_PBC_MAX_IMAGES)
            return fail(BM_EINVAL, "PBC images must be within +-" + std::to_string(BM_PBC_MAX_IMAGES));
    unprepare(c);
    Mesh &m = c->meshes[mesh];
    for (int a = 0; a < 3; a++) m.pbc[a] = img[a];
    return 0;
}

int bm_get_pbc(bm_ctx *c, int mesh, int *images3)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!images3) return fail(BM_EINVAL, "null out");
    for (int a = 0; a < 3; a++) images3[a] = c->meshes[mesh].pbc[a];
    return 0;
}

int bm_set_modules(bm_ctx *c, int mesh, int modules)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (modules & ~(BM_DEMAG | BM_EXCH | BM_IDMI | BM_ANIUNI | BM_ZEEMAN)) return fail(BM_EINVAL, "unknown module bit");
    if ((modules & BM_EXCH) && (modules & BM_IDMI)) return fail(BM_EINVAL, "BM_EXCH and BM_IDMI are exclusive");
    unprepare(c);
    c->meshes[mesh].modules = modules;
    return 0;
}

int bm_set_field(bm_ctx *c, int mesh, const double *Ha, int nsamples, double t_span)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!Ha || nsamples < 1) return fail(BM_EINVAL, "field samples");
    Mesh &m = c->meshes[mesh];
    m.Ha.assign(Ha, Ha + 3 * (size_t)nsamples);
    m.Ha_tspan = t_span;
    m.nHa = nsamples;
    if (c->ready) {
        cudaSetDevice(c->device);
        CK(cudaStreamSynchronize(c->stream));
        if (m.Had) cudaFree(m.Had);
        m.Had = nullptr;
        CK(cudaMalloc(&m.Had, sizeof(double) * m.Ha.size()));
        CK(cudaMemcpy(m.Had, m.Ha.data(), sizeof(double) * m.Ha.size(), cudaMemcpyHostToDevice));
        drop_graph(c);
    }
    return 0;
}

int bm_set_ode(bm_ctx *c, int eval, double dt)
{
    if (int rc = check_ctx(c)) return rc;
    if (eval != BM_RK4 && eval != BM_RKDP54) return fail(BM_EUNSUPPORTED, "evaluation method");
    if (!(dt > 0)) return fail(BM_EINVAL, "dt must be > 0");
    bool changed = (eval != c->eval) || !c->eval_chosen;
    if (eval != c->eval) unprepare(c);
    c->eval = eval;
    c->eval_chosen = true;
    c->dt = dt;
    if (eval == BM_RKDP54 && changed) {
        // Boris/DiffEq_Defs.h:58-63 defaults, Boris/DiffEq_CommonBase_Control.cpp:111
        c->tol = 1e-4; c->dT_incr = 2.0; c->dT_min = 1e-15; c->dT_max = 3e-12;
    }
    if (c->ready) {
        if (int rc = read_state(c)) return rc;
        c->host_st.primed = 0;
        return upload_state(c);
    }
    return 0;
}

int bm_set_evalspeedup(bm_ctx *c, int level)
{
    if (int rc = check_ctx(c)) return rc;
    if (level < 0 || level > 6) return fail(BM_EINVAL, "evaluation speedup level must be 0..6");
    if (level == c->es_level) return 0;
    unprepare(c);
    c->es_level = level;
    c->es_reset = true;
    return 0;
}

int bm_set_evalspeedup_self(bm_ctx *c, int metres)
{
    if (int rc = check_ctx(c)) return rc;
    if (metres != 0 && metres != 1) return fail(BM_EINVAL, "evaluation speedup self term: 0 normalised, 1 metres");
    if (metres == c->es_self_metres) return 0;
    unprepare(c);
    c->es_self_metres = metres;
    c->es_reset = true;
    return 0;
}

int bm_set_astepctrl(bm_ctx *c, double err_fail, double dT_incr, double dT_min, double dT_max)
{
    if (int rc = check_ctx(c)) return rc;
    if (!(err_fail > 0) || !(dT_incr >= 1) || !(dT_min > 0) || !(dT_max >= dT_min)) return fail(BM_EINVAL, "astepctrl values");
    c->tol = err_fail; c->dT_incr = dT_incr; c->dT_min = dT_min; c->dT_max = dT_max;
    if (c->ready) {
        if (int rc = read_state(c)) return rc;
        c->host_st.tol = err_fail; c->host_st.dT_incr = dT_incr; c->host_st.dT_min = dT_min; c->host_st.dT_max = dT_max;
        c->dt = c->host_st.dT;
        return upload_state(c);
    }
    return 0;
}

int bm_set_memory_limit(bm_ctx *c, long long bytes)
{
    if (int rc = check_ctx(c)) return rc;
    if (bytes < 0) return fail(BM_EINVAL, "memory limit < 0");
    c->mem_limit = (size_t)bytes;
    return 0;
}

int bm_set_batched(bm_ctx *c, int on)
{
    if (int rc = check_ctx(c)) return rc;
    unprepare(c);
    c->batched = on != 0;
    return 0;
}

int bm_set_precision(bm_ctx *c, int precision)
{
    if (int rc = check_ctx(c)) return rc;
    if (precision != BM_FP64 && precision != BM_MIXED) return fail(BM_EINVAL, "precision");
    if (precision != c->precision) unprepare(c);
    c->precision = precision;
    return 0;
}

int bm_set_multiconvolution(bm_ctx *c, int mode, const int *n_common)
{
    if (int rc = check_ctx(c)) return rc;
    if (mode < BM_ML_OFF || mode > BM_ML_SUPERMESH) return fail(BM_EINVAL, "multiconvolution mode");
    if (n_common && (n_common[0] < 1 || n_common[1] < 1 || n_common[2] < 1)) return fail(BM_EINVAL, "n_common must be >= 1");
    if (n_common && (nice_size(n_common[0]) > 4096 || nice_size(n_common[1]) > 4096 || n_common[2] > 32))
        return fail(BM_EUNSUPPORTED, "n_common above the supported FFT size");
    unprepare(c);
    c->ml_mode = mode;
    c->ml_nc_set = n_common != nullptr;
    if (n_common) for (int a = 0; a < 3; a++) c->ml_nc[a] = n_common[a];
    return 0;
}

int bm_set_supermesh_cellsize(bm_ctx *c, double hx, double hy, double hz)
{
    if (int rc = check_ctx(c)) return rc;
    if (!(hx > 0) || !(hy > 0) || !(hz > 0)) return fail(BM_EINVAL, "supermesh cellsize must be > 0");
    unprepare(c);
    c->sm_h[0] = hx; c->sm_h[1] = hy; c->sm_h[2] = hz;
    return 0;
}

int bm_set_supermesh_pbc(bm_ctx *c, int x_images, int y_images, int z_images)
{
    if (int rc = check_ctx(c)) return rc;
    const int img[3] = {x_images, y_images, z_images};
    for (int a = 0; a < 3; a++)
        if (img[a] > BM_PBC_MAX_IMAGES || img[a] < -BM_PBC_MAX_IMAGES)
            return fail(BM_EINVAL, "PBC images must be within +-" + std::to_string(BM_PBC_MAX_IMAGES));
    unprepare(c);
    // SDemag::Set_PBC: the supermesh convolution and every mesh's stencils (Set_Magnetic_PBC)
    for (int a = 0; a < 3; a++) c->sm_pbc[a] = img[a];
    for (auto &m : c->meshes)
        for (int a = 0; a < 3; a++) m.pbc[a] = img[a];
    return 0;
}

int bm_supermesh_info(bm_ctx *c, int *n3, double *h3, double *rect6, long long *nonempty)
{
    if (int rc = check_ctx(c)) return rc;
    if (c->ml_mode != BM_ML_SUPERMESH) return fail(BM_ESTATE, "supermesh demag is off");
    if (int rc = prepare(c)) return rc;
    if (!c->ml || !c->ml->sm) return fail(BM_ESTATE, "no mesh with demag on the supermesh");
    const SMGeom &g = c->ml->smg;
    for (int a = 0; a < 3; a++) {
        if (n3) n3[a] = g.n[a];
        if (h3) h3[a] = g.h[a];
        if (rect6) { rect6[a] = g.rs[a]; rect6[3 + a] = g.re[a]; }
    }
    if (nonempty) *nonempty = g.nonempty;
    return 0;
}

int bm_ml_info(bm_ctx *c, int *L, int *nc3, int *layer_mesh, int *transfer, double *rects6, int *kinds)
{
    if (int rc = check_ctx(c)) return rc;
    if (c->ml_mode < 0) return fail(BM_ESTATE, "multilayered convolution is off");
    if (c->ml_mode == BM_ML_SUPERMESH) return fail(BM_ESTATE, "supermesh demag: see bm_supermesh_info");
    if (int rc = prepare(c)) return rc;
    if (!c->ml) return fail(BM_ESTATE, "no mesh with demag in the multilayered convolution");
    const MLRun &r = *c->ml;
    const MLGeom &g = r.g;
    if (L) *L = g.L;
    if (nc3) for (int a = 0; a < 3; a++) nc3[a] = g.nc[a];
    for (int l = 0; l < g.L; l++) {
        if (layer_mesh) layer_mesh[l] = r.mesh_of[g.layers[l].mesh];
        if (transfer) transfer[l] = g.layers[l].transfer;
        if (rects6)
            for (int a = 0; a < 3; a++) { rects6[6 * l + a] = g.layers[l].rs[a]; rects6[6 * l + 3 + a] = g.layers[l].re[a]; }
        if (kinds) for (int q = 0; q < g.L; q++) kinds[l * g.L + q] = g.pair_kind[l * g.L + q];
    }
    return 0;
}

int bm_ml_tile(bm_ctx *c, int *W)
{
    if (int rc = check_ctx(c)) return rc;
    if (int rc = prepare(c)) return rc;
    if (!c->ml || c->ml->sm) return fail(BM_ESTATE, "multilayered convolution is off");
    if (W) *W = c->ml->W;
    return 0;
}

int bm_adjoint_rk4(bm_ctx *c, int steps, int ckpt_every, const double *target, int m0_scales_with_Ms, double *loss,
                   double *dMs, double *dK1, double *dHa, double *times_ms)
{
    if (int rc = check_ctx(c)) return rc;
    if (!target || !loss) return fail(BM_EINVAL, "null target or loss");
    if (c->meshes.size() != 1) return fail(BM_EUNSUPPORTED, "adjoint: one mesh");
    if (c->eval != BM_RK4) return fail(BM_EUNSUPPORTED, "adjoint: RK4 only");
    if (c->ml_mode >= 0 || c->batched) return fail(BM_EUNSUPPORTED, "adjoint: no multilayer or batching");
    if (c->es_level > 0) return fail(BM_EUNSUPPORTED, "adjoint: no evaluation speedup");
    if (ckpt_every < 1 || steps < 1 || steps % ckpt_every) return fail(BM_EINVAL, "adjoint: steps must be a positive multiple of ckpt_every");
    const Mesh &m0 = c->meshes[0];
    if (m0.modules & ~(BM_DEMAG | BM_EXCH | BM_ANIUNI | BM_ZEEMAN)) return fail(BM_EUNSUPPORTED, "adjoint: demag, exchange, anisotropy, Zeeman only");
    if (m0.K2 != 0.0) return fail(BM_EUNSUPPORTED, "adjoint: K2 must be 0");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    return (c->precision == BM_FP64)
               ? adjoint_T<double>(c, steps, ckpt_every, target, m0_scales_with_Ms, loss, dMs, dK1, dHa, times_ms)
               : adjoint_T<float>(c, steps, ckpt_every, target, m0_scales_with_Ms, loss, dMs, dK1, dHa, times_ms);
}

int bm_prepare(bm_ctx *c)
{
    if (int rc = check_ctx(c)) return rc;
    return prepare(c);
}

int bm_set_m(bm_ctx *c, int mesh, const double *M)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!M) return fail(BM_EINVAL, "null M");
    Mesh &m = c->meshes[mesh];
    if (!c->ready) {
        m.M0.assign(M, M + 3 * (size_t)m.n);
        return 0;
    }
    cudaSetDevice(c->device);
    CK(cudaMemcpyAsync(m.stage64, M, sizeof(double) * 3 * m.n, cudaMemcpyHostToDevice, c->stream));
    if (c->precision == BM_FP64) CKL(launch_aos_to_planes<double>((double *)m.buf[0], m.stage64, m.n, c->stream), "aos_to_planes");
    else CKL(launch_aos_to_planes<float>((float *)m.buf[0], m.stage64, m.n, c->stream), "aos_to_planes");
    c->s1_dirty = true;
    // a new M un-primes the RKDP54 error estimate, as a restart of the reference solver does, and
    // drops the fields saved for the evaluation speedup
    if (int rc = read_state(c)) return rc;
    c->host_st.primed = 0;
    c->host_st.error = 0;   // a new M clears a non-finite state
    c->es_reset = true;
    c->dt = c->host_st.dT;
    return upload_state(c);
}

int bm_get_m(bm_ctx *c, int mesh, double *M)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!M) return fail(BM_EINVAL, "null M");
    Mesh &m = c->meshes[mesh];
    if (!c->ready) {
        memcpy(M, m.M0.data(), sizeof(double) * 3 * m.n);
        return 0;
    }
    cudaSetDevice(c->device);
    if (c->precision == BM_FP64) CKL(launch_planes_to_aos<double>(m.stage64, (const double *)m.buf[0], m.n, c->stream), "planes_to_aos");
    else CKL(launch_planes_to_aos<float>(m.stage64, (const float *)m.buf[0], m.n, c->stream), "planes_to_aos");
    CK(cudaMemcpyAsync(M, m.stage64, sizeof(double) * 3 * m.n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int bm_load_ovf2_mag(bm_ctx *c, int mesh, const char *path, double renormalize)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    int n3[3];
    if (int rc = bm_ovf2_read(path, n3, nullptr, nullptr, nullptr, 0)) return rc;
    std::vector<double> src(3 * (size_t)n3[0] * n3[1] * n3[2]);
    if (int rc = bm_ovf2_read(path, nullptr, nullptr, nullptr, src.data(), (long long)src.size())) return rc;
    if (std::fabs(renormalize) > 1e-12) bm_renormalize(src.data(), (long long)(src.size() / 3), renormalize);
    Mesh &m = c->meshes[mesh];
    int dn[3] = {m.nx, m.ny, m.nz};
    std::vector<double> dst(3 * (size_t)m.n);
    if (int rc = bm_map_cells(src.data(), n3, dst.data(), dn)) return rc;
    // the reference marks zero-length cells empty (VEC_VC::copy_values); this path has no empty cells
    for (long long i = 0; i < m.n; i++) {
        const double *v = dst.data() + 3 * i;
        if (!(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] > 0.0))
            return fail(BM_EUNSUPPORTED, "bm_load_ovf2_mag: cell " + std::to_string(i) +
                                             " has a zero-length value (empty cells are not supported)");
    }
    return bm_set_m(c, mesh, dst.data());
}

int bm_save_ovf2_mag(bm_ctx *c, int mesh, const char *path, const char *data_type, int normalize)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    Mesh &m = c->meshes[mesh];
    std::vector<double> M(3 * (size_t)m.n);
    if (int rc = bm_get_m(c, mesh, M.data())) return rc;
    int n3[3] = {m.nx, m.ny, m.nz};
    return bm_ovf2_write(path, n3, m.h, m.o, M.data(), data_type, normalize ? m.Ms : 1.0);
}

int bm_compute_hdemag(bm_ctx *c, int mesh, double *H, double *energy)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!H) return fail(BM_EINVAL, "null H");
    if (!(c->meshes[mesh].modules & BM_DEMAG)) return fail(BM_ESTATE, "mesh has no demag module");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    Mesh &m = c->meshes[mesh];
    int rc = (c->precision == BM_FP64) ? compute_field_T<double>(c, m, BM_DEMAG, H) : compute_field_T<float>(c, m, BM_DEMAG, H);
    if (rc) return rc;
    if (energy) {
        std::vector<double> Mh(3 * (size_t)m.n);
        if ((rc = bm_get_m(c, mesh, Mh.data()))) return rc;
        double dot = 0.0;
        for (size_t i = 0; i < Mh.size(); i++) dot += Mh[i] * H[i];
        *energy = -BM_MU0 * dot / (2.0 * (double)m.n);
    }
    return 0;
}

}  // extern "C"

namespace {
// Device-resident demag field for a caller that keeps M and Heff on the GPU as AoS vectors (the
// reference's cuVEC<cuReal3> data): M into the context's state planes, x transform, y / z passes,
// inverse x with the demag term alone, then H set or added into the caller's AoS array.
template <typename T, typename S>
int demag_device_T(bm_ctx *c, Mesh &m, const S *M, S *H, int add, double *energy)
{
    cudaStream_t s = c->stream;
    CKL((launch_daos_to_planes<S, T>(B<T>(m, 0), M, m.n, s)), "M in");
    StageArgs<T> a = stage_args<T>(c, m);
    a.mode = BM_MODE_UPDATE;
    a.Min = B<T>(m, 0); a.Mbase = B<T>(m, 0);
    CKL(launch_stage<T>(a, s), "xfwd");
    int cnt = 0;
    if (int rc = enqueue_yz<T>(c, m, BM_GATE_ALWAYS, &cnt)) return rc;
    StageArgs<T> h = stage_args<T>(c, m);
    h.mode = BM_MODE_HEFF;
    h.modules = BM_DEMAG;
    h.do_xfwd = 0;
    h.Min = B<T>(m, 0);
    h.Hout = (T *)m.Hout;
    CKL(launch_stage<T>(h, s), "inverse x");
    double *dot = energy ? m.stage64 : nullptr;
    if (dot) CK(cudaMemsetAsync(dot, 0, sizeof(double), s));
    CKL((launch_planes_to_daos<S, T>(H, (const T *)m.Hout, m.n, add, M, dot, s)), "H out");
    if (dot) {
        double d = 0.0;
        CK(cudaMemcpyAsync(&d, dot, sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        *energy = -BM_MU0 * d / (2.0 * (double)m.n);
    }
    CK(cudaStreamSynchronize(s));
    c->s1_dirty = true;
    return 0;
}

template <typename T>
int set_m_device_T(bm_ctx *c, Mesh &m, const void *M, int eb)
{
    if (eb == 4) CKL((launch_daos_to_planes<float, T>(B<T>(m, 0), (const float *)M, m.n, c->stream)), "M in");
    else CKL((launch_daos_to_planes<double, T>(B<T>(m, 0), (const double *)M, m.n, c->stream)), "M in");
    return 0;
}

template <typename T>
int get_m_device_T(bm_ctx *c, Mesh &m, void *M, int eb)
{
    if (eb == 4) CKL((launch_planes_to_daos<float, T>((float *)M, B<T>(m, 0), m.n, 0, nullptr, nullptr, c->stream)), "M out");
    else CKL((launch_planes_to_daos<double, T>((double *)M, B<T>(m, 0), m.n, 0, nullptr, nullptr, c->stream)), "M out");
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int device_entry_checks(bm_ctx *c, int mesh, const void *p, int eb, void *stream)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!p) return fail(BM_EINVAL, "null device array");
    if (eb != 4 && eb != 8) return fail(BM_EINVAL, "element size must be 4 (float) or 8 (double)");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    // the caller's writes to its arrays on its stream come first
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    return 0;
}
}  // namespace

extern "C" {

int bm_demag_field_device(bm_ctx *c, int mesh, const void *M, void *H, int elem_bytes, int add, double *energy,
                          void *stream)
{
    if (int rc = device_entry_checks(c, mesh, M, elem_bytes, stream)) return rc;
    if (!H) return fail(BM_EINVAL, "null device array");
    Mesh &m = c->meshes[mesh];
    if (!(m.modules & BM_DEMAG) || m.ml_role) return fail(BM_ESTATE, "mesh has no demag convolution of its own");
    if (c->precision == BM_FP64)
        return elem_bytes == 4 ? demag_device_T<double, float>(c, m, (const float *)M, (float *)H, add, energy)
                               : demag_device_T<double, double>(c, m, (const double *)M, (double *)H, add, energy);
    return elem_bytes == 4 ? demag_device_T<float, float>(c, m, (const float *)M, (float *)H, add, energy)
                           : demag_device_T<float, double>(c, m, (const double *)M, (double *)H, add, energy);
}

int bm_set_m_device(bm_ctx *c, int mesh, const void *M, int elem_bytes, void *stream)
{
    if (int rc = device_entry_checks(c, mesh, M, elem_bytes, stream)) return rc;
    Mesh &m = c->meshes[mesh];
    int rc = c->precision == BM_FP64 ? set_m_device_T<double>(c, m, M, elem_bytes) : set_m_device_T<float>(c, m, M, elem_bytes);
    if (rc) return rc;
    c->s1_dirty = true;
    if ((rc = read_state(c))) return rc;
    c->host_st.primed = 0;
    c->host_st.error = 0;
    c->es_reset = true;
    c->dt = c->host_st.dT;
    return upload_state(c);
}

int bm_get_m_device(bm_ctx *c, int mesh, void *M, int elem_bytes, void *stream)
{
    if (int rc = device_entry_checks(c, mesh, M, elem_bytes, stream)) return rc;
    Mesh &m = c->meshes[mesh];
    return c->precision == BM_FP64 ? get_m_device_T<double>(c, m, M, elem_bytes) : get_m_device_T<float>(c, m, M, elem_bytes);
}

int bm_compute_heff(bm_ctx *c, int mesh, double *H)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!H) return fail(BM_EINVAL, "null H");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    Mesh &m = c->meshes[mesh];
    return (c->precision == BM_FP64) ? compute_field_T<double>(c, m, ~0, H) : compute_field_T<float>(c, m, ~0, H);
}

int bm_run(bm_ctx *c, int steps, bm_stats *out)
{
    if (int rc = check_ctx(c)) return rc;
    if (steps < 0) return fail(BM_EINVAL, "steps < 0");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    if (steps > 0) {
        int rc = (c->precision == BM_FP64) ? run_T<double>(c, steps) : run_T<float>(c, steps);
        if (rc) return rc;
    }
    return bm_get_stats(c, out);
}

int bm_get_stats(bm_ctx *c, bm_stats *out)
{
    if (int rc = check_ctx(c)) return rc;
    if (c->ready)
        if (int rc = read_state(c)) return rc;
    if (out) {
        out->accepted = c->host_st.accepted;
        out->rejected = c->host_st.rejected;
        out->attempts = c->host_st.attempts;
        out->time = c->host_st.time;
        out->dT = c->ready ? c->host_st.dT : c->dt;
        out->last_lte = c->host_st.last_lte;
    }
    return 0;
}

// ODECommon_Base::Get_mxh / Get_dmdt (Boris/DiffEq_CommonBase_Get.cpp:7,19): the value of the last
// step that computed it (0 before any), and a request that the next step computes it; only the
// device's request flag is written, so the rest of the step state stays the device's
static int get_diag(bm_ctx *c, int which, double *v)
{
    if (int rc = check_ctx(c)) return rc;
    if (!v) return fail(BM_EINVAL, "null output");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    double val = 0.0;
    static const int one = 1;
    const double *src = which ? &c->st->dmdt : &c->st->mxh;
    int *flag = which ? &c->st->calc_dmdt : &c->st->calc_mxh;
    CK(cudaMemcpyAsync(&val, src, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(flag, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *v = val;
    return 0;
}

int bm_get_mxh(bm_ctx *c, double *mxh) { return get_diag(c, 0, mxh); }
int bm_get_dmdt(bm_ctx *c, double *dmdt) { return get_diag(c, 1, dmdt); }

int bm_mesh_info(bm_ctx *c, int mesh, int *n3, int *N3)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    Mesh &m = c->meshes[mesh];
    if (n3) { n3[0] = m.nx; n3[1] = m.ny; n3[2] = m.nz; }
    if (N3) {
        N3[0] = 2 * nice_size(m.nx);
        N3[1] = 2 * nice_size(m.ny);
        N3[2] = m.nz > 1 ? 2 * nice_size(m.nz) : 1;
    }
    return 0;
}

int bm_device_m(bm_ctx *c, int mesh, void **dptr, int *elem_bytes)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (int rc = prepare(c)) return rc;
    if (dptr) *dptr = c->meshes[mesh].buf[0];
    if (elem_bytes) *elem_bytes = (c->precision == BM_FP64) ? 8 : 4;
    return 0;
}

int bm_sync(bm_ctx *c)
{
    if (int rc = check_ctx(c)) return rc;
    cudaSetDevice(c->device);
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int bm_kernels_per_step(bm_ctx *c, int *count)
{
    if (int rc = check_ctx(c)) return rc;
    if (count) *count = c->kernels_per_step;
    return 0;
}

int bm_run_timed(bm_ctx *c, int steps, bm_stats *out, double *device_ms)
{
    if (int rc = check_ctx(c)) return rc;
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    if (c->s1_dirty) {
        int cnt = 0;
        int rc = (c->precision == BM_FP64) ? enqueue_prime<double>(c, &cnt) : enqueue_prime<float>(c, &cnt);
        if (rc) return rc;
        c->s1_dirty = false;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c->stream));
    int rc = bm_run(c, steps, out);
    if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (device_ms) *device_ms = ms;
    return 0;
}

}  // extern "C"

namespace {
// Eager steps with an event after every launch: the launches, buffers and arguments of the
// captured step graph, timed one by one on the context's stream.
template <typename T>
int time_step_T(bm_ctx *c, int steps, double *ms6, double *bytes6, int *launches6)
{
    for (int k = 0; k < BM_TK_COUNT; k++) { ms6[k] = 0.0; bytes6[k] = 0.0; launches6[k] = 0; }
    if (c->batched && c->meshes.size() > 1) return fail(BM_EUNSUPPORTED, "bm_time_step: batched meshes are timed per step only");
    if (c->ml) return fail(BM_EUNSUPPORTED, "bm_time_step: the multilayered convolution has bm_ml_time_kernels");
    if (c->es_level > 0) return fail(BM_EUNSUPPORTED, "bm_time_step: evaluation speedup steps are timed per step only");
    if (c->s1_dirty) {
        int cnt = 0;
        if (int rc = enqueue_prime<T>(c, &cnt)) return rc;
        c->s1_dirty = false;
    }
    LaunchTimer lt;
    cudaEvent_t e0 = nullptr;
    CK(cudaEventCreate(&e0));
    lt.ev.push_back(e0);
    CK(cudaEventRecord(e0, c->stream));
    c->lt = &lt;
    int count = 0, rc = 0;
    for (int i = 0; i < steps && !rc; i++)
        rc = (c->eval == BM_RKDP54) ? enqueue_rkdp_attempt<T>(c, &count) : enqueue_rk4_step<T>(c, &count);
    c->lt = nullptr;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (!rc && e == cudaSuccess) {
        for (size_t i = 0; i < lt.kind.size(); i++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, lt.ev[i], lt.ev[i + 1]);
            ms6[lt.kind[i]] += t;
            bytes6[lt.kind[i]] += lt.bytes[i];
            launches6[lt.kind[i]]++;
        }
    }
    for (auto ev : lt.ev) cudaEventDestroy(ev);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(BM_ECUDA, std::string("bm_time_step: ") + cudaGetErrorString(e));
    return read_state(c);
}

template <typename T>
int time_kernels_T(bm_ctx *c, Mesh &m, int reps, double *ms4, double *bytes4)
{
    for (int i = 0; i < 4; i++) { ms4[i] = 0.0; bytes4[i] = 0.0; }
    if (m.ml_role) return fail(BM_EUNSUPPORTED, "per-mesh kernel timing of a multilayer mesh");
    cudaStream_t s = c->stream;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const double cs = sizeof(cpx<T>), rs = sizeof(T);
    const double s1 = 3.0 * m.nz * m.ny * m.LX * cs, s2 = 3.0 * m.nz * m.Ny * m.LX * cs;
    const double kb = 6.0 * (m.LX + 1) * (m.Ny / 2 + 1) * (m.Nz / 2 + 1) * rs;
    auto timeit = [&](auto launch, int slot, double bytes) -> int {
        for (int w = 0; w < 2; w++) { int rc = launch(); if (rc) return rc; }
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps; r++) { int rc = launch(); if (rc) return rc; }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms4[slot] = ms / reps;
        bytes4[slot] = bytes;
        return 0;
    };
    int rc = 0;
    if ((m.modules & BM_DEMAG) && m.ml_role == 0) {
        YZArgs<T> a = yz_args<T>(c, m, BM_GATE_ALWAYS);
        if (m.nz == 1) {
            rc = timeit([&]() { return launch_ymid2d<T>(a, s); }, 0, 2.0 * s1 + 4.0 / 6.0 * kb);
        } else if (m.yzy) {
            rc = timeit([&]() { return launch_yzy<T>(a, s); }, 0, 2.0 * s1 + kb);
        } else {
            a.W = m.Wy;
            rc = timeit([&]() { return launch_yfwd<T>(a, s); }, 0, s1 + s2);
            YZArgs<T> b = a;
            b.W = m.Wz;
            if (!rc) rc = timeit([&]() { return launch_zmid<T>(b, s); }, 1, 2.0 * s2 + kb);
            if (!rc) rc = timeit([&]() { return launch_yinv<T>(a, s); }, 2, s1 + s2);
        }
    }
    // the stage kernel as RKDP54 stage 3 uses it: stage input, step base and 3 earlier evaluations
    // in five distinct arrays (copies of M), writes rhs and next M into two more
    T *tmp = nullptr;
    if (!rc && cudaMalloc(&tmp, sizeof(T) * 3 * 7 * m.n) != cudaSuccess) rc = BM_ENOMEM;
    for (int k = 0; k < 5 && !rc; k++)
        if (cudaMemcpyAsync(tmp + 3 * k * m.n, m.buf[0], sizeof(T) * 3 * m.n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            rc = BM_ECUDA;
    if (!rc) {
        StageArgs<T> a = stage_args<T>(c, m);
        a.mode = BM_MODE_STAGE;
        a.Min = tmp;
        a.Mbase = tmp + 3 * m.n;
        a.nev = 3;
        a.ev[0] = tmp + 6 * m.n; a.ev[1] = tmp + 9 * m.n; a.ev[2] = tmp + 12 * m.n;
        a.cev[0] = a.cev[1] = a.cev[2] = 0.0;
        a.crhs = 0.0;
        a.ev_out = tmp + 15 * m.n;
        a.Mout = tmp + 18 * m.n;
        double bytes = 3.0 * m.n * rs * (1 + 1 + 3 + 1 + 1);
        if (m.modules & BM_DEMAG) bytes += 2.0 * s1;
        if (a.Ms_map) bytes += m.n * rs;
        if (a.K1_map) bytes += m.n * rs;
        rc = timeit([&]() { return launch_stage<T>(a, s); }, 3, bytes);
    }
    cudaStreamSynchronize(s);
    if (tmp) cudaFree(tmp);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->s1_dirty = true;
    return rc ? fail(BM_ECUDA, "kernel timing launch failed (" + std::to_string(rc) + ")") : 0;
}
}  // namespace

namespace {
// Times the parts of one multilayer demag evaluation (CUDA events, reps launches each after two
// warm-ups) and returns their algorithmic bytes: slots 0..4 as ml_enqueue_part, slot 5 the
// whole evaluation. Algorithmic bytes per evaluation: every layer's native M read and field
// write (2 R n_mesh), its spectra through the y passes and the z pass (4 C S1 + 4 C S2, C the
// complex3 size, S1 = LX ny nz, S2 = LX Ny nz on the common grid) and every unique kernel once.
template <typename T>
int ml_time_T(bm_ctx *c, int reps, double *ms6, double *bytes6)
{
    MLRun &r = *c->ml;
    const MLGeom &g = r.g;
    cudaStream_t s = c->stream;
    const double R3 = 3.0 * sizeof(T), C3 = 6.0 * sizeof(T);
    const double LX = g.N[0] / 2, S1 = LX * g.nc[1] * g.nc[2], S2 = LX * g.N[1] * g.nc[2];
    double kbytes = 0.0;
    for (auto &K : g.kernels) kbytes += (double)K.count * sizeof(T);
    double bin = 0.0, bout = 0.0;
    for (int l = 0; l < g.L; l++) {
        const Mesh &M = c->meshes[r.mesh_of[g.layers[l].mesh]];
        double nm = (double)M.n;
        if (g.force2d == 2) nm /= M.nz;   // a z layer of the mesh
        bin += R3 * nm + C3 * S1;
        bout += R3 * nm + C3 * S1;
    }
    bytes6[0] = bin;
    bytes6[1] = g.L * C3 * (S1 + S2);
    bytes6[2] = g.L * 2.0 * C3 * S2 + kbytes;
    bytes6[3] = g.L * C3 * (S1 + S2);
    bytes6[4] = bout;
    bytes6[5] = bytes6[0] + bytes6[1] + bytes6[2] + bytes6[3] + bytes6[4];
    // the x forward of direct layers happens in their stage kernels; prime it once
    int cnt = 0;
    for (auto &mm : c->meshes) {
        if (mm.ml_role != 1) continue;
        StageArgs<T> a = stage_args<T>(c, mm);
        a.mode = BM_MODE_UPDATE;
        a.Min = B<T>(mm, 0); a.Mbase = B<T>(mm, 0);
        CKL(launch_stage<T>(a, s), "xfwd");
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int part = 0; part <= 5; part++) {
        auto go = [&]() -> int {
            if (part < 5) return ml_enqueue_part<T>(c, part, BM_GATE_ALWAYS, 0, &cnt);
            return enqueue_fields<T>(c, BM_GATE_ALWAYS, 0, &cnt);
        };
        for (int w = 0; w < 2; w++) if (int rc = go()) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
        cudaEventRecord(e0, s);
        for (int q = 0; q < reps; q++) if (int rc = go()) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms6[part] = ms / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->s1_dirty = true;
    return 0;
}
}  // namespace

extern "C" {

int bm_ml_time_kernels(bm_ctx *c, int reps, double *ms6, double *bytes6)
{
    if (int rc = check_ctx(c)) return rc;
    if (!ms6 || !bytes6 || reps < 1) return fail(BM_EINVAL, "args");
    if (int rc = prepare(c)) return rc;
    if (!c->ml || c->ml->sm) return fail(BM_ESTATE, "multilayered convolution is off");
    cudaSetDevice(c->device);
    return (c->precision == BM_FP64) ? ml_time_T<double>(c, reps, ms6, bytes6) : ml_time_T<float>(c, reps, ms6, bytes6);
}

int bm_time_demag(bm_ctx *c, int mesh, int reps, double *ms)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (reps < 1 || !ms) return fail(BM_EINVAL, "bm_time_demag: bad arguments");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    Mesh &m = c->meshes[mesh];
    if (!(m.modules & BM_DEMAG) || m.ml_role) return fail(BM_EUNSUPPORTED, "bm_time_demag: a mesh with its own demag convolution");
    auto one = [&](auto tag) -> int {
        using T = decltype(tag);
        StageArgs<T> a = stage_args<T>(c, m);
        a.mode = BM_MODE_UPDATE;
        a.Min = B<T>(m, 0); a.Mbase = B<T>(m, 0);
        if (int rc = launch_stage<T>(a, c->stream)) return rc;
        int cnt = 0;
        if (int rc = enqueue_yz<T>(c, m, BM_GATE_ALWAYS, &cnt)) return rc;
        StageArgs<T> h = stage_args<T>(c, m);
        h.mode = BM_MODE_HEFF;
        h.modules = BM_DEMAG;
        h.do_xfwd = 0;
        h.Min = B<T>(m, 0);
        h.Hout = (T *)m.Hout;
        return launch_stage<T>(h, c->stream);
    };
    auto run = [&]() -> int { return c->precision == BM_FP64 ? one(0.0) : one(0.0f); };
    if (int rc = run()) return fail(BM_ECUDA, "bm_time_demag: launch failed (" + std::to_string(rc) + ")");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c->stream));
    int rc = 0;
    for (int i = 0; i < reps && !rc; i++) rc = run();
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->s1_dirty = true;
    if (rc) return fail(BM_ECUDA, "bm_time_demag: launch failed (" + std::to_string(rc) + ")");
    *ms = (double)t / reps;
    return 0;
}

int bm_time_step(bm_ctx *c, int steps, double *ms6, double *bytes6, int *launches6)
{
    if (int rc = check_ctx(c)) return rc;
    if (!ms6 || !bytes6 || !launches6 || steps < 1) return fail(BM_EINVAL, "bm_time_step: bad arguments");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    return c->precision == BM_FP64 ? time_step_T<double>(c, steps, ms6, bytes6, launches6)
                                   : time_step_T<float>(c, steps, ms6, bytes6, launches6);
}

int bm_time_kernels(bm_ctx *c, int mesh, int reps, double *ms4, double *bytes4)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!ms4 || !bytes4 || reps < 1) return fail(BM_EINVAL, "args");
    if (int rc = prepare(c)) return rc;
    cudaSetDevice(c->device);
    Mesh &m = c->meshes[mesh];
    return (c->precision == BM_FP64) ? time_kernels_T<double>(c, m, reps, ms4, bytes4)
                                     : time_kernels_T<float>(c, m, reps, ms4, bytes4);
}

int bm_tiles(bm_ctx *c, int mesh, int *tiles4)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    if (!tiles4) return fail(BM_EINVAL, "null out");
    Mesh &m = c->meshes[mesh];
    tiles4[0] = m.W2; tiles4[1] = m.Wy + 100 * m.yv; tiles4[2] = m.Wz + 1000 * m.yzy + 10000 * m.zv; tiles4[3] = (m.staged ? -1 : 1) * (m.rpb + 100 * m.xv);
    return 0;
}

int bm_debug_kernels(bm_ctx *c, int mesh, double *K6)
{
    if (int rc = check_mesh(c, mesh)) return rc;
    Mesh &m = c->meshes[mesh];
    cudaSetDevice(c->device);
    int Nx = 2 * nice_size(m.nx), Ny = 2 * nice_size(m.ny), Nz = m.nz > 1 ? 2 * nice_size(m.nz) : 1;
    size_t nk = (size_t)(Nx / 2 + 1) * (Ny / 2 + 1) * (Nz / 2 + 1);
    double *K = nullptr;
    void *tx = nullptr, *ty = nullptr, *tz = nullptr;
    CK(cudaMalloc(&K, sizeof(double) * 6 * nk));
    int rc = 0;
    if ((rc = upload_table<double>(&tx, Nx, true, c->stream)) || (rc = upload_table<double>(&ty, Ny, true, c->stream)) ||
        (rc = upload_table<double>(&tz, Nz, true, c->stream))) { cudaFree(K); return rc; }
    double hm = std::fmax(m.h[0], std::fmax(m.h[1], m.h[2]));
    std::vector<double> fq(6 * BM_FARQ_PER_COMP);
    bm_far_coeffs(m.h[0] / hm, m.h[1] / hm, m.h[2] / hm, fq.data());
    CK(cudaMemcpy(c->farq, fq.data(), sizeof(double) * fq.size(), cudaMemcpyHostToDevice));
    rc = build_kernels_device<double>(K, m.nx, m.ny, m.nz, Nx, Ny, Nz, m.h[0], m.h[1], m.h[2], c->farq,
                                      (const cpx<double> *)tx, (const cpx<double> *)ty, (const cpx<double> *)tz, c->stream,
                                      m.pbc);
    cudaFree(tx); cudaFree(ty); cudaFree(tz);
    if (rc) { cudaFree(K); return fail(BM_ECUDA, "kernel build failed"); }
    CK(cudaMemcpy(K6, K, sizeof(double) * 6 * nk, cudaMemcpyDeviceToHost));
    cudaFree(K);
    return 0;
}

int bm_debug_tensor(int device, int nx, int ny, int nz, double hx, double hy, double hz, double *oct6)
{
    return bm_debug_tensor_pbc(device, nx, ny, nz, hx, hy, hz, nullptr, oct6);
}

int bm_debug_tensor_pbc(int device, int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc3, double *oct6)
{
    if (nx < 1 || ny < 1 || nz < 1 || !oct6) return fail(BM_EINVAL, "args");
    CK(cudaSetDevice(device));
    size_t np = (size_t)nx * ny * nz;
    double *d = nullptr, *fq_d = nullptr;
    CK(cudaMalloc(&d, sizeof(double) * 6 * np));
    CK(cudaMalloc(&fq_d, sizeof(double) * 6 * BM_FARQ_PER_COMP));
    double hm = std::fmax(hx, std::fmax(hy, hz));
    std::vector<double> fq(6 * BM_FARQ_PER_COMP);
    bm_far_coeffs(hx / hm, hy / hm, hz / hm, fq.data());
    CK(cudaMemcpy(fq_d, fq.data(), sizeof(double) * fq.size(), cudaMemcpyHostToDevice));
    int rc = tensor_octant_device(d, nx, ny, nz, hx, hy, hz, fq_d, 0, pbc3);
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(oct6, d, sizeof(double) * 6 * np, cudaMemcpyDeviceToHost));
    cudaFree(d);
    cudaFree(fq_d);
    return rc ? fail(BM_ECUDA, "tensor launch") : 0;
}

int bm_debug_fft(int device, int L, int howmany, int precision, int inverse, double *data)
{
    if (L < 1 || howmany < 1 || !data) return fail(BM_EINVAL, "args");
    FFTPlan P;
    if (!bm_make_plan(L, P)) return fail(BM_EUNSUPPORTED, "length");
    CK(cudaSetDevice(device));
    size_t nv = 2 * (size_t)L * howmany;
    double *d64 = nullptr;
    CK(cudaMalloc(&d64, sizeof(double) * nv));
    CK(cudaMemcpy(d64, data, sizeof(double) * nv, cudaMemcpyHostToDevice));
    int rc = 0;
    void *tw = nullptr;
    if (precision == BM_FP64) {
        if ((rc = upload_table<double>(&tw, L, false, 0))) { cudaFree(d64); return rc; }
        rc = launch_fft_strided<double>((cpx<double> *)d64, P, (const cpx<double> *)tw, 1, L, howmany, 0, 1, inverse != 0, 0);
    } else {
        float *d32 = nullptr;
        CK(cudaMalloc(&d32, sizeof(float) * nv));
        launch_convert<float>(d32, d64, (long long)nv, 0);
        if ((rc = upload_table<float>(&tw, L, false, 0))) { cudaFree(d64); cudaFree(d32); return rc; }
        rc = launch_fft_strided<float>((cpx<float> *)d32, P, (const cpx<float> *)tw, 1, L, howmany, 0, 1, inverse != 0, 0);
        launch_convert_back<float>(d64, d32, (long long)nv, 0);
        cudaDeviceSynchronize();
        cudaFree(d32);
    }
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(data, d64, sizeof(double) * nv, cudaMemcpyDeviceToHost));
    cudaFree(d64);
    cudaFree(tw);
    return rc ? fail(BM_ECUDA, "fft launch failed " + std::to_string(rc)) : 0;
}

}  // extern "C"
