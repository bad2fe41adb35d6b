// Test entry points over the Boris-side shim (used by tests/test_gpu_shim.py): a mesh's vectors held
// the way the reference holds them (cu_obj<cuVEC_VC<cuReal3>> M, cu_obj<cuVEC<cuReal3>> Heff, filled
// from CPU VEC_VC / VEC), driven through DemagB200 and ODEB200 exactly as the reference's module and
// ODE code would call them.
#include "DemagB200.h"
#include "BorisCUDALib.cuh"
#include "BorisLib.h"

#include <cstring>

namespace {
struct ShimMesh {
    VEC_VC<DBL3> Mc;
    VEC<DBL3> Hc;
    cu_obj<cuVEC_VC<cuReal3>> M;
    cu_obj<cuVEC<cuReal3>> Heff;
    int n = 0;
    ShimMesh(int nx, int ny, int nz, double hx, double hy, double hz)
    {
        n = nx * ny * nz;
        Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
        Mc.assign(DBL3(hx, hy, hz), r, DBL3(1, 0, 0));
        Hc.assign(DBL3(hx, hy, hz), r, DBL3(0, 0, 0));
        M()->set_from_cpuvec(Mc);
        Heff()->set_from_cpuvec(Hc);
    }
    void set_m(const double *Mh)
    {
        memcpy(Mc.data(), Mh, sizeof(double) * 3 * n);
        M()->copy_from_cpuvec(Mc);
    }
    void get_m(double *Mh)
    {
        M()->copy_to_cpuvec(Mc);
        memcpy(Mh, Mc.data(), sizeof(double) * 3 * n);
    }
};
struct ShimDemag {
    ShimMesh mesh;
    DemagB200 *mod = nullptr;
    ShimDemag(int nx, int ny, int nz, double hx, double hy, double hz) : mesh(nx, ny, nz, hx, hy, hz) {}
};
struct ShimODE {
    ShimMesh mesh;
    ODEB200 *ode = nullptr;
    ShimODE(int nx, int ny, int nz, double hx, double hy, double hz) : mesh(nx, ny, nz, hx, hy, hz) {}
};
}  // namespace

extern "C" {

int shim_real_bytes(void) { return (int)sizeof(cuBReal); }

void *shim_demag_create(int nx, int ny, int nz, double hx, double hy, double hz, int device)
{
    ShimDemag *s = new ShimDemag(nx, ny, nz, hx, hy, hz);
    s->mod = new DemagB200(s->mesh.M, s->mesh.Heff, device);
    if (s->mod->Error_On_Create()) { delete s->mod; delete s; return nullptr; }
    return s;
}

// Heff preset to Hpre (host), then one UpdateField (which adds H_demag), then Heff and the energy back
int shim_demag_update(void *h, const double *M, const double *Hpre, double *Heff, double *energy)
{
    ShimDemag *s = (ShimDemag *)h;
    s->mesh.set_m(M);
    memcpy(s->mesh.Hc.data(), Hpre, sizeof(double) * 3 * s->mesh.n);
    s->mesh.Heff()->copy_from_cpuvec(s->mesh.Hc);
    s->mod->UpdateField();
    cudaDeviceSynchronize();
    s->mesh.Heff()->copy_to_cpuvec(s->mesh.Hc);
    memcpy(Heff, s->mesh.Hc.data(), sizeof(double) * 3 * s->mesh.n);
    *energy = s->mod->GetLastEnergyDensity();
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// DemagB200::Set_PBC, then the images it reports
int shim_demag_set_pbc(void *h, int x, int y, int z, int *out3)
{
    ShimDemag *s = (ShimDemag *)h;
    int rc = (int)s->mod->Set_PBC(INT3(x, y, z)).code();
    INT3 p = s->mod->Get_PBC();
    out3[0] = p.x; out3[1] = p.y; out3[2] = p.z;
    return rc;
}

void shim_demag_destroy(void *h)
{
    ShimDemag *s = (ShimDemag *)h;
    if (!s) return;
    delete s->mod;
    delete s;
}

void *shim_ode_create(int nx, int ny, int nz, double hx, double hy, double hz, int device)
{
    ShimODE *s = new ShimODE(nx, ny, nz, hx, hy, hz);
    s->ode = new ODEB200(s->mesh.M, device);
    if (!s->ode->Context()) { delete s->ode; delete s; return nullptr; }
    return s;
}

// the forwarder's context, to describe the mesh's material, modules and field through the C ABI
void *shim_ode_context(void *h) { return ((ShimODE *)h)->ode->Context(); }

int shim_ode_setode(void *h, int eval, double dt)
{
    ShimODE *s = (ShimODE *)h;
    s->ode->SetdT(dt);
    return (int)s->ode->SetODE(ODE_LLG, eval ? EVAL_RKDP54 : EVAL_RK4).code();
}

void shim_ode_astepctrl(void *h, double err_fail, double dT_incr, double dT_min, double dT_max)
{
    ((ShimODE *)h)->ode->SetAdaptiveTimeStepCtrl(err_fail, dT_incr, dT_min, dT_max);
}

void shim_ode_set_m(void *h, const double *M) { ((ShimODE *)h)->mesh.set_m(M); }
void shim_ode_get_m(void *h, double *M) { ((ShimODE *)h)->mesh.get_m(M); }

int shim_ode_iterate(void *h, int steps, double *time)
{
    ShimODE *s = (ShimODE *)h;
    BError e = s->ode->Iterate(steps);
    *time = s->ode->GetTime();
    return (int)e.code();
}

void shim_ode_destroy(void *h)
{
    ShimODE *s = (ShimODE *)h;
    if (!s) return;
    delete s->ode;
    delete s;
}

}  // extern "C"
