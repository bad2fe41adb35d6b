// Boris-side DemagB200 / ODEB200 (see DemagB200.h).
#include "DemagB200.h"

namespace {

// device address of a cuVEC's data: the cuVEC object itself lives in device memory (cu_obj), so
// its data pointer is read on the device
template <typename V>
__global__ void k_vec_data(V &v, cuReal3 **out)
{
    *out = v.data();
}

template <typename V>
cuReal3 *vec_data(cu_obj<V> &v)
{
    cuReal3 **d = nullptr;
    cuReal3 *h = nullptr;
    if (cudaMalloc(&d, sizeof(cuReal3 *)) != cudaSuccess) return nullptr;
    k_vec_data<V><<<1, 1>>>(v, d);
    cudaMemcpy(&h, d, sizeof(cuReal3 *), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return h;
}

int add_mesh_like(bm_ctx *ctx, cuSZ3 n, cuReal3 h)
{
    int id = -1;
    if (bm_add_mesh(ctx, (int)n.x, (int)n.y, (int)n.z, (double)h.x, (double)h.y, (double)h.z, 0, 0, 0, &id)) return -1;
    return id;
}

}  // namespace

//------------------------------------------------------------------ DemagB200

DemagB200::DemagB200(cu_obj<cuVEC_VC<cuReal3>> &M_, cu_obj<cuVEC<cuReal3>> &Heff_, int device) : M(M_), Heff(Heff_)
{
    if (bm_create(device, &ctx)) { error_on_create(BERROR_OUTOFGPUMEMORY_CRIT); return; }
    own_ctx = true;
    mesh = add_mesh_like(ctx, M()->size_cpu(), M()->cellsize_cpu());
    if (mesh < 0 || bm_set_modules(ctx, mesh, BM_DEMAG) ||
        bm_set_precision(ctx, sizeof(cuBReal) == 8 ? BM_FP64 : BM_MIXED)) error_on_create(BERROR_INCORRECTVALUE);
    else error_on_create = Initialize();
}

DemagB200::~DemagB200()
{
    if (own_ctx && ctx) bm_destroy(ctx);
}

BError DemagB200::Initialize(void)
{
    BError error(CLASS_STR(DemagB200));
    M_data = vec_data(M);
    H_data = vec_data(Heff);
    if (!M_data || !H_data) return error(BERROR_OUTOFGPUMEMORY_CRIT);
    if (bm_prepare(ctx)) return error(BERROR_OUTOFGPUMEMORY_CRIT);
    initialized = true;
    return error;
}

BError DemagB200::UpdateConfiguration(UPDATECONFIG_ cfgMessage)
{
    // a changed mesh means new cuVEC storage: look the data pointers up again
    Uninitialize();
    return Initialize();
}

BError DemagB200::Set_PBC(INT3 demag_pbc_images)
{
    BError error(CLASS_STR(DemagB200));
    if (bm_set_pbc(ctx, mesh, demag_pbc_images.x, demag_pbc_images.y, demag_pbc_images.z))
        return error(BERROR_INCORRECTVALUE);
    pbc = demag_pbc_images;
    Uninitialize();
    return Initialize();
}

void DemagB200::UpdateField(void)
{
    double e = 0.0;
    if (bm_demag_field_device(ctx, mesh, M_data, H_data, (int)sizeof(cuBReal), 1, &e, nullptr)) return;
    last_energy = e;
    energy.from_cpu((cuBReal)e);
}

//------------------------------------------------------------------ ODEB200

ODEB200::ODEB200(cu_obj<cuVEC_VC<cuReal3>> &M_, int device) : M(M_)
{
    if (bm_create(device, &ctx)) return;
    own_ctx = true;
    add_mesh_like(ctx, M()->size_cpu(), M()->cellsize_cpu());
    bm_set_precision(ctx, sizeof(cuBReal) == 8 ? BM_FP64 : BM_MIXED);
    M_data = vec_data(M);
}

ODEB200::~ODEB200()
{
    if (own_ctx && ctx) bm_destroy(ctx);
}

BError ODEB200::SetODE(ODE_ setOde, EVAL_ evalMethod)
{
    BError error(CLASS_STR(ODEB200));
    if (setOde != ODE_LLG || (evalMethod != EVAL_RK4 && evalMethod != EVAL_RKDP54)) return error(BERROR_INCORRECTVALUE);
    eval = evalMethod == EVAL_RK4 ? BM_RK4 : BM_RKDP54;
    if (bm_set_ode(ctx, eval, dT)) return error(BERROR_INCORRECTVALUE);
    return error;
}

void ODEB200::SetdT(double dT_)
{
    dT = dT_;
    bm_set_ode(ctx, eval, dT);
}

void ODEB200::SetAdaptiveTimeStepCtrl(double err_fail, double dT_incr, double dT_min, double dT_max)
{
    bm_set_astepctrl(ctx, err_fail, dT_incr, dT_min, dT_max);
}

BError ODEB200::Iterate(int steps)
{
    BError error(CLASS_STR(ODEB200));
    if (!M_data) return error(BERROR_OUTOFGPUMEMORY_CRIT);
    // the context's state is the mesh's M on the first call; afterwards it stays on the device in the
    // context between calls, and M receives a copy after each
    if (!ready) {
        if (bm_set_m_device(ctx, 0, M_data, (int)sizeof(cuBReal), nullptr)) return error(BERROR_INCORRECTVALUE);
        ready = true;
    }
    if (bm_run(ctx, steps, &st)) return error(BERROR_INCORRECTVALUE);
    if (bm_get_m_device(ctx, 0, M_data, (int)sizeof(cuBReal), nullptr)) return error(BERROR_INCORRECTVALUE);
    return error;
}
