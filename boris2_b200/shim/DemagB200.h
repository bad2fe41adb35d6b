// Boris-side drop-in for the demag module and the ODE iteration of one ferromagnetic mesh, compiled
// against the reference's own headers (it is the code a Boris maintainer adds to the reference
// tree; boris2_b200/shim/Makefile builds it here). Both forward to the C ABI of include/boris_b200.h
// with the mesh's vectors left on the GPU.
//
//   DemagB200   a ModulesCUDA (Boris/ModulesCUDA.h:15-114) in place of DemagCUDA
//               (Boris/DemagCUDA.h): UpdateField adds H_demag of the mesh's M into its Heff, as
//               DemagCUDA::UpdateField does (Boris/DemagCUDA.cpp:106-121), through
//               bm_demag_field_device, and keeps the energy density in the module's `energy`.
//   ODEB200     the setode / setdt / astepctrl settings and the Iterate step of ODECommon_Base
//               (Boris/DiffEq_Common.cpp:79, Boris/Commands.cpp:1914,1931,
//               Boris/DiffEq_CommonBase_IterateCUDA.cpp:13) for LLG with RK4 or RKDP54: the mesh's
//               M goes into a context, bm_run advances it, M comes back.
#pragma once

#include "Boris_Enums_Defs.h"
#include "ModulesCUDA.h"
#include "DiffEq_Defs.h"
#include "../../include/boris_b200.h"

class DemagB200 : public ModulesCUDA {
    bm_ctx *ctx = nullptr;
    int mesh = 0;
    cu_obj<cuVEC_VC<cuReal3>> &M;
    cu_obj<cuVEC<cuReal3>> &Heff;
    cuReal3 *M_data = nullptr, *H_data = nullptr;
    bool own_ctx = false;
    double last_energy = 0.0;
    INT3 pbc;

public:
    // M and Heff: the mesh's vectors (MeshCUDA::M, MeshCUDA::Heff); h the cellsize (m). The module
    // owns a context on `device` with one mesh of M's dimensions and the demag module only.
    DemagB200(cu_obj<cuVEC_VC<cuReal3>> &M_, cu_obj<cuVEC<cuReal3>> &Heff_, int device = 0);
    ~DemagB200();

    BError Initialize(void);
    void Uninitialize(void) { initialized = false; }
    BError UpdateConfiguration(UPDATECONFIG_ cfgMessage);
    void UpdateConfiguration_Values(UPDATECONFIG_ cfgMessage) {}
    void UpdateField(void);

    // DemagBase::Set_PBC / Get_PBC (Boris/DemagBase.h:55, Boris/Demag.cpp:137): images per axis of the
    // periodic demag, also the periodic neighbours of the library's stencils (bm_set_pbc); the kernels
    // are rebuilt by the following Initialize, as UpdateConfiguration(UPDATECONFIG_DEMAG_CONVCHANGE) does
    BError Set_PBC(INT3 demag_pbc_images);
    INT3 Get_PBC(void) const { return pbc; }

    // the energy density of the last UpdateField (also in the module's device `energy`)
    double GetLastEnergyDensity(void) const { return last_energy; }
    // the library's last error text
    static const char *LastError(void) { return bm_last_error(); }
};

class ODEB200 {
    bm_ctx *ctx = nullptr;
    cu_obj<cuVEC_VC<cuReal3>> &M;
    cuReal3 *M_data = nullptr;
    int eval = BM_RK4;
    double dT = 1e-13;
    bool own_ctx = false;
    bool ready = false;
    bm_stats st = {};

public:
    // M: the mesh's magnetization; the caller describes the mesh's material and modules on
    // Context() before the first Iterate (bm_set_material, bm_set_modules, bm_set_field).
    ODEB200(cu_obj<cuVEC_VC<cuReal3>> &M_, int device = 0);
    ~ODEB200();
    bm_ctx *Context(void) { return ctx; }

    // setode LLG RK4|RKDP54 (other equations and evaluators: BERROR_INCORRECTVALUE)
    BError SetODE(ODE_ setOde, EVAL_ evalMethod);
    // setdt
    void SetdT(double dT_);
    // astepctrl
    void SetAdaptiveTimeStepCtrl(double err_fail, double dT_incr, double dT_min, double dT_max);
    // advance `steps` accepted steps (the reference's Iterate loop of AdvanceTime) and leave the
    // new M in the mesh's vector
    BError Iterate(int steps = 1);

    double GetTime(void) const { return st.time; }
    double GetdT(void) const { return st.dT; }
    long long GetIteration(void) const { return st.accepted; }
};
