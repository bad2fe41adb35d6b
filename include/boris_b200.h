/*
 * boris_b200 — C ABI of the B200-native micromagnetic field-and-integrate path.
 *
 * Plain C: opaque context, plain pointers and sizes, int status (0 = ok, otherwise an
 * error code; bm_last_error() gives the text). Host arrays of vectors are AoS doubles
 * (x, y, z per cell), cells ordered x fastest, then y, then z — the layout of the
 * reference's VEC<DBL3> (BorisLib/VEC.h). One context per host thread; all work goes
 * to one internal CUDA stream.
 *
 * Each entry point names the reference interface it replaces (paths in the reference tree).
 */
#ifndef BORIS_B200_H
#define BORIS_B200_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct bm_ctx bm_ctx;

/* modules (the reference's MOD_ values for the FM mesh modules on this path) */
#define BM_DEMAG   1   /* Boris/Demag.h            MOD_DEMAG */
#define BM_EXCH    2   /* Boris/Exchange.h         MOD_EXCHANGE (Exch_6ngbr_Neu) */
#define BM_IDMI    4   /* Boris/iDMExchange.h      MOD_IDMEXCHANGE (replaces BM_EXCH) */
#define BM_ANIUNI  8   /* Boris/Anisotropy.h       MOD_ANIUNI */
#define BM_ZEEMAN 16   /* Boris/Zeeman.h           MOD_ZEEMAN */

/* evaluation methods (Boris/DiffEq_Defs.h EVAL_RK4, EVAL_RKDP54) */
#define BM_RK4    0
#define BM_RKDP54 1

/* precision */
#define BM_FP64   0   /* plain form: every array and transform in FP64 */
#define BM_MIXED  1   /* FP32 FFTs, convolution and stages; FP64 tensor build and RKDP54 error norm */

/* error codes */
#define BM_OK          0
#define BM_EINVAL      1
#define BM_ECUDA       2
#define BM_ENOMEM      3
#define BM_ESTATE      4
#define BM_EUNSUPPORTED 5
#define BM_ENONFINITE  6

typedef struct {
    long long accepted;    /* accepted steps since creation (the reference's iteration counter) */
    long long rejected;    /* RKDP54 rejections */
    long long attempts;    /* RKDP54 stage-0 evaluations */
    double time;           /* simulated time, s */
    double dT;             /* current time step, s */
    double last_lte;       /* last RKDP54 error estimate (max over cells of |M - M4| / |M|) */
} bm_stats;

/* Context (one device). Replaces the reference's SuperMesh/ODECommon ownership of meshes
 * (Boris/SuperMesh.h, Boris/DiffEq_CommonBase.h). */
int bm_create(int device, bm_ctx **out);
int bm_destroy(bm_ctx *ctx);
const char *bm_last_error(void);
int bm_version(void);

/* Add a ferromagnetic mesh: n cells, cellsize h (m), origin (m).
 * Replaces Mesh creation + MeshBase::n / h / meshRect (Boris/MeshBase.h). */
int bm_add_mesh(bm_ctx *ctx, int nx, int ny, int nz, double hx, double hy, double hz,
                double ox, double oy, double oz, int *mesh_id);

/* Material parameters (Boris/MeshParams.h: Ms, A, D, alpha, grel, K1, K2, mcanis_ea1).
 * grel is the relative gyromagnetic ratio (gamma / 2.212761569e5). */
int bm_set_material(bm_ctx *ctx, int mesh, double Ms, double A, double alpha, double grel,
                    double K1, double K2, const double *ea3, double D);

/* Per-cell maps of Ms and K1 (absolute values, one per cell), or NULL for uniform.
 * Replaces the spatial scaling of MaterialParameter (Boris/MaterialParameter.h:805,
 * setparamvar) read through update_parameters_mcoarse (Boris/MeshParamsControl.h:56). */
int bm_set_material_maps(bm_ctx *ctx, int mesh, const double *Ms_map, const double *K1_map);

/* Module set for a mesh (bitmask of BM_*). Replaces MeshBase::AddModule / DelModule
 * (Boris/MeshBaseModules.cpp); BM_IDMI and BM_EXCH are exclusive as in the reference
 * (Boris/SimSharedData.cpp:179). */
int bm_set_modules(bm_ctx *ctx, int mesh, int modules);

/* Periodic boundary conditions of a mesh: the number of images summed along each axis (0: the axis
 * is not periodic; at most BM_PBC_MAX_IMAGES in magnitude). Replaces Demag::Set_PBC
 * (Boris/Demag.cpp:137) with Mesh::Set_Magnetic_PBC (Boris/MeshControl.cpp:49), which the "pbc"
 * command reaches through SuperMesh::Set_PBC (Boris/SuperMeshMeshes_Settings.cpp:659):
 *   - demag: along a periodic axis the convolution is cyclic over the mesh's n cells with the
 *     tensor summed over +-|images| periods (Boris/DemagTFunc_PBC.cpp:5,97,185,300,
 *     Boris/ConvolutionData.cpp:115-145); the evaluation speedup's self term adds the images'
 *     far field (DemagTFunc::SelfDemag_PBC, Boris/DemagTFunc_Self.cpp:57);
 *   - exchange / iDMI: a cell on a periodic face takes the cell on the opposite face as its missing
 *     neighbour, times the sign of images (a negative count wraps with -1, as the reference's
 *     differential operators do, BorisLib/VEC_VC_Del.h:141, BorisLib/VEC_VC_Grad.h:139).
 * Not combined with the multilayered modes of bm_set_multiconvolution (BM_EUNSUPPORTED at set-up);
 * with the supermesh mode the supermesh convolution takes its images from bm_set_supermesh_pbc. */
#define BM_PBC_MAX_IMAGES 1000
int bm_set_pbc(bm_ctx *ctx, int mesh, int x_images, int y_images, int z_images);
int bm_get_pbc(bm_ctx *ctx, int mesh, int *images3);

/* Applied field: nsamples piecewise-constant 3-vectors (A/m) over [0, t_span); with
 * nsamples == 1 the field is constant. Replaces Zeeman::SetField / H_equation
 * (Boris/Zeeman.cpp:164); as there, the field is evaluated at the step start time. */
int bm_set_field(bm_ctx *ctx, int mesh, const double *Ha, int nsamples, double t_span);

/* ODE: evaluation method and time step. Replaces SetODE (Boris/DiffEq_Common.cpp:79,
 * "setode LLG RK4|RKDP54") and SetdT ("setdt", Boris/Commands.cpp:1914). Selecting an
 * evaluation method loads its defaults (Boris/DiffEq_CommonBase_Control.cpp:9). */
int bm_set_ode(bm_ctx *ctx, int eval, double dt);

/* Adaptive step control for RKDP54. Replaces SetAdaptiveTimeStepCtrl ("astepctrl",
 * Boris/Commands.cpp:1931, Boris/DiffEq_CommonBase.h:236): err_fail = relative error
 * tolerance, dT_incr = maximum increase factor, dT_min / dT_max = step limits. */
int bm_set_astepctrl(bm_ctx *ctx, double err_fail, double dT_incr, double dT_min, double dT_max);

/* Many independent meshes per launch (batching): with on != 0, every pass of a field evaluation
 * runs as one launch over a work list of (mesh, tile) items covering all meshes of the context
 * (uneven sizes allowed), and a step is one CUDA graph of those launches. The meshes are
 * independent systems sharing the time step, as meshes of one reference simulation do
 * (ODECommon); without it every mesh gets its own launches. Not combined with
 * bm_set_multiconvolution. */
int bm_set_batched(bm_ctx *ctx, int on);

/* Device-memory limit of the context, in bytes (0, the default: the free device memory). Before it
 * allocates anything, the set-up of a context compares the bytes its meshes need (every buffer plus
 * the scratch of the kernel-spectrum build) with the lower of this limit and the free device memory
 * and refuses with BM_ENOMEM, naming both figures, when they do not fit; the context stays usable
 * (raise the limit or shrink the meshes and call again). The reference checks for room before it
 * builds its kernels on the GPU and falls back to a CPU build (Boris/DemagKernelCUDA.cpp:357-369);
 * this path has no CPU fallback, so it refuses. */
int bm_set_memory_limit(bm_ctx *ctx, long long bytes);

/* Precision: BM_FP64 or BM_MIXED (default BM_MIXED). Must be set before the first run. */
int bm_set_precision(bm_ctx *ctx, int precision);

/* Multilayered convolution (SDemag in multilayer mode). The demag modules of all meshes with
 * BM_DEMAG become the layers of one convolution on a common grid: each layer's M is moved to the
 * common grid by the reference's weighted mesh transfer, the layers' spectra are combined by an
 * L x L set of kernels (self, z-shifted, full), and the field is moved back into every mesh.
 * Mesh positions come from the origins given to bm_add_mesh.
 *   mode BM_ML_OFF   every mesh its own demag convolution (default)
 *        BM_ML_3D    `multiconvolution 1`: 3D common grid (2D when every mesh is one cell thick)
 *        BM_ML_2D    `2dmulticonvolution 1`: n_common.z = 1, each mesh one layer
 *        BM_ML_2D_LAYERED `2dmulticonvolution 2`: n_common.z = 1, every z cell layer its own layer
 *   n_common NULL for the default (largest cell count of the meshes per axis, `ncommonauto`),
 *        else 3 ints (`ncommon`; n_common.z = 1 then selects 2D).
 * Replaces SDemag::Set_Multilayered_Convolution / Set_2D_Multilayered_Convolution / Set_n_common
 * (Boris/SDemag.cpp:323,341,362; commands Boris/Commands.cpp:1704,1720). At most 8 layers;
 * n_common.z at most 32. */
#define BM_ML_OFF (-1)
#define BM_ML_3D 0
#define BM_ML_2D 1
#define BM_ML_2D_LAYERED 2
#define BM_ML_SUPERMESH 3   /* supermesh demag, below (n_common unused) */
int bm_set_multiconvolution(bm_ctx *ctx, int mode, const int *n_common);

/* Supermesh demag (mode BM_ML_SUPERMESH): the reference's SDemag module with the multilayered
 * convolution off (Boris/SDemag.cpp:737-760, `multiconvolution 0` with the supermesh demag module
 * added). One demag convolution runs on a grid over the bounding box of every mesh with BM_DEMAG:
 * the meshes' M are moved onto it by the weighted mesh transfer (a supermesh cell takes the
 * covered-volume ratio times the reciprocal-distance weights over every mesh it overlaps,
 * BorisLib/VEC_MeshTransfer.h:901), convolved with the supermesh's own kernel, and the field is
 * moved back into every mesh (VEC_MeshTransfer.h:1221). The grid has round(size / h) cells per axis
 * (at least 1) and cellsize size / cells (SuperMesh::UpdateConfiguration,
 * Boris/SuperMeshControl.cpp:22-44). As in the reference there is no evaluation speedup for it
 * (bm_set_evalspeedup is refused) and it is not combined with bm_set_batched or the adjoint.
 *   bm_set_supermesh_cellsize  requested cellsize (SuperMesh::SetFMSMeshCellsize, `fmscellsize`,
 *                              Boris/SuperMeshSettings.cpp:79; default 5 nm, Boris/SuperMesh.h:117)
 *   bm_set_supermesh_pbc       PBC images of the supermesh convolution, also set as every mesh's
 *                              stencil PBC (SDemag::Set_PBC / Set_Magnetic_PBC, Boris/SDemag.cpp:404)
 *   bm_supermesh_info          cells, cellsize, rectangle (start, end) and the count of supermesh
 *                              cells covered by a mesh (the reference's non_empty_cells) */
int bm_set_supermesh_cellsize(bm_ctx *ctx, double hx, double hy, double hz);
int bm_set_supermesh_pbc(bm_ctx *ctx, int x_images, int y_images, int z_images);
int bm_supermesh_info(bm_ctx *ctx, int *n3, double *h3, double *rect6, long long *nonempty);

/* Geometry of the multilayered convolution once prepared (after a run or field call, or
 * bm_prepare): layer count, n_common, and per layer the mesh, whether it is moved by mesh
 * transfer, the convolution rectangle (start, end; 6 doubles) and per (layer, source) pair the
 * kernel kind (1 self, 2 z-shifted, 3 z-shifted reused for the opposite shift, 4 full). Arrays
 * sized for 8 layers may be passed; any pointer may be NULL. */
int bm_ml_info(bm_ctx *ctx, int *L, int *nc3, int *layer_mesh, int *transfer, double *rects6, int *kinds);

/* Device time (ms per launch sequence, CUDA events) and algorithmic bytes of the parts of one
 * multilayer demag evaluation: [0] transfer in + x forward, [1] y forward, [2] z pass with the
 * L x L products, [3] y inverse, [4] x inverse + transfer out, [5] the whole evaluation. */
int bm_ml_time_kernels(bm_ctx *ctx, int reps, double *ms6, double *bytes6);

/* Columns per block of the fused multilayer z pass (chosen by timing at setup). */
int bm_ml_tile(bm_ctx *ctx, int *W);

/* Discrete adjoint of RK4 (no counterpart in the reference): from the current state, run `steps`
 * RK4 steps (a checkpoint of M every ckpt_every steps), evaluate the loss
 * L = (1/n) sum_i |M_i(T)/Ms_i - target_i|^2 (target: AoS unit vectors, 3n doubles) and its exact
 * gradients by reverse mode through every stage: dMs (n, per-cell Ms), dK1 (n, per-cell K1 of the
 * uniaxial anisotropy) and dHa (3 * nsamples of bm_set_field). m0_scales_with_Ms: the initial M is
 * Ms * m0, so L also depends on Ms through it. One mesh; modules demag, exchange, anisotropy
 * (K2 = 0) and Zeeman; steps a multiple of ckpt_every. times_ms (optional, 2 doubles): device time
 * of the forward run and of the backward sweep. The context is left at the end of the run.
 * Any output pointer except loss may be NULL. */
int bm_adjoint_rk4(bm_ctx *ctx, int steps, int ckpt_every, const double *target, int m0_scales_with_Ms, double *loss,
                   double *dMs, double *dK1, double *dHa, double *times_ms);

/* Allocate and build everything for the current configuration now (kernels, tiles). */
int bm_prepare(bm_ctx *ctx);

/* Evaluation speedup, the reference's `evalspeedup` command (Boris/Simulation.cpp:551,
 * Boris/DemagCUDA.cpp:106): level 0 off, 1 step, 2 linear, 3 quadratic, 4 cubic, 5 quartic,
 * 6 quintic. A computed demag field is saved without its self term; other evaluations extrapolate
 * it from the last `level` saved fields (polynomial in time) plus the self term of the current M.
 * RK4: the field is computed and saved at the first evaluation of every step, the other
 * evaluations extrapolate once `level` fields are saved. RKDP54: the reference's rule, decided on
 * the device per evaluation: compute and save at the first evaluation of an attempt that follows a
 * completed step, and at every evaluation while fewer than `level` are saved; extrapolate otherwise
 * (so after a rejected step the repeated first evaluation extrapolates). With the multilayered
 * convolution every layer's field is saved and extrapolated on its common grid with the layer's own
 * self term, as SDemagCUDA::UpdateField does (Boris/SDemagCUDA.cpp:587-930); not with the supermesh
 * demag (BM_EUNSUPPORTED at set-up). With batched meshes the y/z passes stay batched and the speedup
 * kernels cover every mesh in one launch. Setting M drops the saved fields. */
int bm_set_evalspeedup(bm_ctx *ctx, int level);
/* The self term of the evaluation speedup: 0 (default) -N of the cell on its cellsize normalised by
 * the largest, the tensor's own self term; 1 as the reference computes it, DemagTFunc::SelfDemag on
 * the cellsize in metres (Boris/DemagCUDA.cpp:39, Boris/SDemag_Demag.cpp:328). For nanometre cells
 * the reference's Newell f then drops terms under its 1e-12 zero threshold (Boris/DemagTFunc_fg.cpp:10),
 * so its coefficients differ (5 x 5 x 3 nm: (-0.232, -0.232, -0.535) against (-0.274, -0.274, -0.452));
 * 1 follows the reference's trajectories with the speedup on. */
int bm_set_evalspeedup_self(bm_ctx *ctx, int metres);
/* Self-demagnetising coefficients -N (x, y, z) of one cell of size hx, hy, hz (DemagTFunc::SelfDemag,
 * Boris/DemagTFunc_Self.cpp:6); host only. */
int bm_self_demag(double hx, double hy, double hz, double *out3);
/* The same on the cellsize in metres as DemagTFunc::SelfDemag computes it there (the speedup's self term
 * with bm_set_evalspeedup_self(ctx, 1)); host only. */
int bm_self_demag_metres(double hx, double hy, double hz, double *out3);

/* Magnetization M (A/m, |M| = Ms), AoS doubles, 3 * n values. Replaces writes/reads of
 * MeshBase::M (VEC_VC<DBL3>, Boris/Mesh.h). Setting M un-primes RKDP54 as a restart does. */
int bm_set_m(bm_ctx *ctx, int mesh, const double *M);
int bm_get_m(bm_ctx *ctx, int mesh, double *M);

/* OOMMF OVF 2.0 files of vector data (rectangular, valuedim 3; "binary 4", "binary 8" or "text").
 * bm_ovf2_read replaces OVF2::Read_OVF2_VEC (Boris/OVF2_Handlers.cpp:364): it fills n3 (nodes),
 * h3 (cellsize, m), rect6 (xmin, ymin, zmin, xmax, ymax, zmax, m) where given, and, when data is
 * not NULL, 3 * n values (AoS, x fastest) into data, which must hold `capacity` >= 3 * n doubles
 * (call once with data = NULL to learn n). A file whose first line is not "# OOMMF OVF 2.0" gives
 * BM_EUNSUPPORTED; a malformed or truncated file BM_EINVAL.
 * bm_ovf2_write replaces OVF2::Write_OVF2_VEC (Boris/OVF2_Handlers.cpp:701): data_type "bin4",
 * "bin8" or "text", every value divided by norm, the rectangle from origin3 (NULL: 0) and n3 * h3. */
int bm_ovf2_read(const char *path, int *n3, double *h3, double *rect6, double *data, long long capacity);
int bm_ovf2_write(const char *path, const int *n3, const double *h3, const double *origin3, const double *data,
                  const char *data_type, double norm);
/* Nearest-cell remap of AoS vectors from src_n3 to dst_n3 cells: VEC::mapmesh_newdims
 * (BorisLib/VEC_mng.h:9). Scale every vector longer than 1e-12 to `length`: VEC::renormalize
 * (BorisLib/VEC_oper.h:45). */
int bm_map_cells(const double *src, const int *src_n3, double *dst, const int *dst_n3);
int bm_renormalize(double *data, long long ncell, double length);
/* The reference's loadovf2mag / saveovf2mag commands (Boris/Commands.cpp:5025, 5192): load a file
 * into a mesh's M, renormalised to `renormalize` when it is non-zero, mapped to the mesh's cell
 * counts; save a mesh's M with the mesh's origin and cellsize, divided by the mesh's Ms when
 * normalize != 0. A file that puts a zero-length value on a cell (an empty cell of the reference's
 * mesh shape) gives BM_EUNSUPPORTED: every cell here carries Ms > 0. */
int bm_load_ovf2_mag(bm_ctx *ctx, int mesh, const char *path, double renormalize);
int bm_save_ovf2_mag(bm_ctx *ctx, int mesh, const char *path, const char *data_type, int normalize);

/* Demagnetising field of the current M into H (3 * n doubles) and the demag energy
 * density -mu0/(2 n) sum M.H. Replaces Demag::UpdateField (Boris/Demag.cpp:170) /
 * DemagCUDA::UpdateField (Boris/DemagCUDA.cpp:106). */
int bm_compute_hdemag(bm_ctx *ctx, int mesh, double *H, double *energy);

/* Device-resident variants for a caller that keeps its vectors on the GPU as AoS arrays of
 * float (elem_bytes 4) or double (8), x, y, z per cell, cells x fastest: the data of the
 * reference's cuVEC<cuReal3> (BorisCUDALib/cuVEC.h). `stream` (a cudaStream_t, NULL for the
 * default stream) is synchronised first, so the caller's pending writes to its arrays land before
 * they are read; each call returns with its results written.
 * bm_demag_field_device: the mesh's M becomes the given M, and its demag field is set (add = 0) or
 * added (add = 1) into H; energy (optional) receives -mu0/(2 n) sum M.H_demag. Replaces the
 * Convolute call of DemagCUDA::UpdateField (Boris/DemagCUDA.cpp:106-121), which adds into Heff.
 * bm_set_m_device / bm_get_m_device: bm_set_m / bm_get_m with device arrays (the ODE state
 * exchange of a forwarder of ODECommon_Base::IterateCUDA, Boris/DiffEq_CommonBase_IterateCUDA.cpp:13). */
int bm_demag_field_device(bm_ctx *ctx, int mesh, const void *M, void *H, int elem_bytes, int add, double *energy,
                          void *stream);
int bm_set_m_device(bm_ctx *ctx, int mesh, const void *M, int elem_bytes, void *stream);
int bm_get_m_device(bm_ctx *ctx, int mesh, void *M, int elem_bytes, void *stream);

/* Effective field of the current M with all modules of the mesh (Zeeman, demag,
 * exchange / iDMI, anisotropy), as MeshBase::UpdateModules leaves Heff
 * (Boris/MeshBaseModules.cpp:76). */
int bm_compute_heff(bm_ctx *ctx, int mesh, double *H);

/* Advance until `steps` more steps are accepted. Replaces the AdvanceTime loop
 * (Boris/SuperMeshSimulation.cpp:84,122) over ODECommon_Base::Iterate[CUDA]
 * (Boris/DiffEq_CommonBase_Iterate.cpp:63, Boris/DiffEq_CommonBase_IterateCUDA.cpp:13).
 * A stage that produces a NaN or infinite M (or RKDP54 error estimate) sets a device flag that is
 * read after every batch of steps: bm_run then returns BM_ENONFINITE. Under RKDP54 the step that
 * produced the state is not accepted, whatever dT is; under RK4 the steps of the batch are counted.
 * The flag stays set, and bm_run refuses, until bm_set_m gives a new M. (The reference has no such
 * check: a NaN state propagates.) */
int bm_run(bm_ctx *ctx, int steps, bm_stats *out);
int bm_get_stats(bm_ctx *ctx, bm_stats *out);

/* The torque and dm/dt diagnostics of the evaluators, replacing ODECommon_Base::Get_mxh / Get_dmdt
 * (Boris/DiffEq_CommonBase_Get.cpp:7,19; reductions in Boris/DiffEqFM_EvalsLLGCUDA.cu:416-640 for
 * RK4 and Boris/DiffEqFM_EvalsCUDA_RKDP54.cu:15-53,188-232 for RKDP54). mxh: the maximum over the
 * cells of |M x Heff| / |M|^2 at the step's first evaluation; dmdt: the maximum of
 * |M - M_step_start| / (dT GAMMA |M|^2) after its last stage (GAMMA = 2.212761569e5); both over the
 * meshes whose grel is non-zero. As in the reference a call returns the value of the last step that
 * computed it (0 before any) and asks the next step to compute it, so a value runs one step behind
 * the call that asked for it. */
int bm_get_mxh(bm_ctx *ctx, double *mxh);
int bm_get_dmdt(bm_ctx *ctx, double *dmdt);

/* Number of cells of a mesh and the FFT sizes its demag convolution uses. */
int bm_mesh_info(bm_ctx *ctx, int mesh, int *n3, int *N3);

/* Device-resident access for benchmarks and wrappers: the device pointer of the
 * current M planes ([3][n] of float (BM_MIXED) or double (BM_FP64)) and a
 * synchronisation point. */
int bm_device_m(bm_ctx *ctx, int mesh, void **dptr, int *elem_bytes);
int bm_sync(bm_ctx *ctx);
/* Number of kernels one bm_run step enqueues (for launch accounting). */
int bm_kernels_per_step(bm_ctx *ctx, int *count);

/* bm_run with its device time (CUDA events on the context's stream around the whole run). */
int bm_run_timed(bm_ctx *ctx, int steps, bm_stats *out, double *device_ms);

/* Time each kernel of one field evaluation of a mesh separately (reps launches each, CUDA
 * events on the context's stream) and report the average ms per launch and the algorithmic
 * bytes each launch must move: index 0 = y/z pass 1 (2D: ymid2d, 3D: yfwd), 1 = zmid (3D),
 * 2 = yinv (3D), 3 = fused stage kernel (inverse x FFT, fields, LLG, update, forward x FFT).
 * Unused slots are 0. Leaves the spectrum buffers stale (the next run re-primes them). */
int bm_time_kernels(bm_ctx *ctx, int mesh, int reps, double *ms4, double *bytes4);

/* Run `steps` steps (RKDP54: attempts) of every mesh eagerly, with the launches, buffers and
 * arguments of the captured step graph, recording a CUDA event after every launch, and report
 * per kernel kind the summed device ms, the summed algorithmic bytes (what each launch must read
 * and write once, from its arguments) and the launch count, in arrays of 8: [0] fused stage kernel,
 * [1] y forward, [2] z pass, [3] y inverse, [4] 2D y pass, [5] other (restore launches, timed, no
 * bytes), [6] fused y -> z -> y cluster pass, [7] unused. The simulation advances. Not for batched meshes, the multilayered convolution or the evaluation
 * speedup (BM_EUNSUPPORTED). No counterpart in the reference (measurement). */
int bm_time_step(bm_ctx *ctx, int steps, double *ms6, double *bytes6, int *launches6);

/* Device time (ms, CUDA events, average of reps) of one demag field evaluation of a mesh as the
 * pipeline runs it: x transform of M, the y / z passes with the kernel product, inverse x transform
 * into H (the demag term alone). The counterpart of one Convolute call of the reference's
 * ConvolutionCUDA (Boris/ConvolutionCUDA.h:478), for the same-box comparison. */
int bm_time_demag(bm_ctx *ctx, int mesh, int reps, double *ms);

/* Tile shapes the autotuner chose for a mesh: [2D y-pass width, 3D y-pass width (plus 100
 * when the 3D y passes use the radix-16 Stockham transform, plus 200 when they are the persistent
 * kernels fed by pipelined bulk tensor copies),
 * z-pass width (plus 1000 when the fused y -> z -> y cluster pass replaces the three 3D passes,
 * plus 10000 when the z pass is the parity split: two threads per pencil line), stage rows per block (plus 100 when the stage kernel uses the radix-8
 * Stockham x transform, 200 the radix-16 one, 300 the radix-16 one at the lower FP32 register
 * cap; negative when it prefetches its per-cell rows into shared memory)]. Valid after the first
 * compute or run. */
int bm_tiles(bm_ctx *ctx, int mesh, int *tiles4);

/* Test hooks (used by the test suite only). */
/* FP64 demag kernel spectra (octant (Nx/2+1)(Ny/2+1)(Nz/2+1), 6 components xx,yy,zz,xy,xz,yz). */
int bm_debug_kernels(bm_ctx *ctx, int mesh, double *K6);
/* Raw FP64 tensor octant values D(i,j,k) for i<nx, j<ny, k<nz: 6 per point. */
int bm_debug_tensor(int device, int nx, int ny, int nz, double hx, double hy, double hz, double *oct6);
/* As bm_debug_tensor for a mesh of nx x ny x nz cells with pbc3 images per axis (NULL: none): along
 * a periodic axis the octant holds the image-summed tensor made even (xx, yy, zz) or odd (the
 * off-diagonal components odd in that axis) about the origin with period n. */
int bm_debug_tensor_pbc(int device, int nx, int ny, int nz, double hx, double hy, double hz, const int *pbc3,
                        double *oct6);
/* Batched complex FFT on the device of `howmany` contiguous lines of length L (in place,
 * interleaved re/im doubles on the host); precision BM_FP64 or BM_MIXED; inverse != 0
 * uses exp(+2 pi i ...), unnormalised. */
int bm_debug_fft(int device, int L, int howmany, int precision, int inverse, double *data);

/* Allocation-free batched FFT, for callers that cannot allocate device memory when they need
 * the transform (a host that has handed the rest of the GPU's memory to other work, or a
 * solver in the middle of an asynchronous step where a cudaMalloc/cudaFree, which may
 * synchronise the device, would stall it). This entry point has no counterpart in the
 * reference. It transforms `howmany` contiguous lines of L complex FP64 values (interleaved
 * re/im) from the device buffer `in` into the device buffer `out` (in == out transforms in
 * place), on `stream` (a cudaStream_t; NULL for the default stream), unnormalised, with
 * exp(+2 pi i ...) when inverse != 0. It calls no cudaMalloc/cudaFree: its only scratch, the
 * twiddle table, lives in a fixed device array of 4096 complex doubles (64 KiB) that every GPU
 * loading the library keeps until exit, so L is limited to 1..4096 (2^p or 3*2^p). Every call
 * made outside stream capture looks up that array's device address on `device`; a call under
 * capture reuses the address of the last uncaptured call, so make the first call on a device
 * before any stream capture (a captured first call gives BM_ESTATE). The caller's current
 * device is restored on return. The table is rewritten by every call, so calls that overlap on
 * the GPU (different streams, or concurrent host threads) race on it and must be serialised. */
int bm_fft_noalloc(int device, int L, int howmany, int inverse, const double *in, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
