/*
 * Same-box reference GPU bar (measurement infrastructure; never linked into the product):
 * a thin extern "C" harness over the reference's own GPU demag convolution,
 * ConvolutionCUDA<., DemagKernelCUDA> (Boris/ConvolutionCUDA.h:478 Convolute_3D, :383 Convolute_2D)
 * with its cuFFT plans (Boris/ConvolutionDataCUDA.cpp:24,130-306), transposes and fused q2D
 * product kernels (Boris/DemagKernelCUDA.cu:93-803), compiled unmodified for sm_100a by
 * baseline/Makefile into baseline/_ref/librefgpu_f32.so (SINGLEPRECISION 1) and
 * librefgpu_f64.so (SINGLEPRECISION 0).
 *
 *   refgpu_create    build the convolution and its kernels for an n, h mesh
 *                    (Calculate_Demag_Kernels(true, on_gpu), Boris/DemagKernelCUDA.cpp:358,603)
 *   refgpu_set_m     M (host AoS doubles) into the GPU cuVEC_VC, as MeshCUDA does
 *   refgpu_eval      `reps` evaluations Convolute(M, Heff, energy, false, false) as
 *                    DemagCUDA::UpdateField issues them (Boris/DemagCUDA.cpp:121), timed with CUDA
 *                    events on the default stream (the one the reference uses); returns ms per call
 *   refgpu_get_h     H_demag of the current M (host AoS doubles)
 */
#include "stdafx.h"
#include "ConvolutionCUDA.h"
#include "DemagKernelCUDA.h"
#include "BorisCUDALib.cuh"
#include "BorisLib.h"

#include <vector>
#include <cstring>

namespace {

struct RefDemagGPU : public ConvolutionCUDA<RefDemagGPU, DemagKernelCUDA> {
    RefDemagGPU(cuSZ3 n_, cuReal3 h_) : ConvolutionCUDA<RefDemagGPU, DemagKernelCUDA>(n_, h_) {}
    BError calc(bool on_gpu) { return Calculate_Demag_Kernels(true, on_gpu); }
    bool failed(void) { return (bool)Convolution_Error_on_Create(); }
    void conv(cu_obj<cuVEC_VC<cuReal3>> &In, cu_obj<cuVEC<cuReal3>> &Out, cu_obj<cuBReal> &energy, bool clear)
    {
        Convolute(In, Out, energy, false, clear);
    }
};

struct refgpu_s {
    RefDemagGPU *conv = nullptr;
    VEC_VC<DBL3> Mc;
    VEC<DBL3> Hc;
    cu_obj<cuVEC_VC<cuReal3>> M;
    cu_obj<cuVEC<cuReal3>> H;
    cu_obj<cuBReal> energy;
    int n = 0;
};

}  // namespace

extern "C" {

int refgpu_precision_bytes(void) { return (int)sizeof(cuBReal); }

void *refgpu_create(int nx, int ny, int nz, double hx, double hy, double hz, int on_gpu)
{
    refgpu_s *s = new refgpu_s();
    s->n = nx * ny * nz;
    Rect r(DBL3(0, 0, 0), DBL3(hx * nx, hy * ny, hz * nz));
    s->Mc.assign(DBL3(hx, hy, hz), r, DBL3(1, 0, 0));
    s->Hc.assign(DBL3(hx, hy, hz), r, DBL3(0, 0, 0));
    if (!s->M()->set_from_cpuvec(s->Mc) || !s->H()->set_from_cpuvec(s->Hc)) { delete s; return nullptr; }
    s->conv = new RefDemagGPU(cuSZ3(nx, ny, nz), cuReal3(hx, hy, hz));
    if (s->conv->failed() || s->conv->calc(on_gpu != 0)) { delete s->conv; delete s; return nullptr; }
    cudaDeviceSynchronize();
    return s;
}

int refgpu_set_m(void *h, const double *M)
{
    refgpu_s *s = (refgpu_s *)h;
    memcpy(s->Mc.data(), M, sizeof(double) * 3 * s->n);
    return s->M()->copy_from_cpuvec(s->Mc) ? 0 : 1;
}

double refgpu_eval(void *h, int reps)
{
    refgpu_s *s = (refgpu_s *)h;
    s->conv->conv(s->M, s->H, s->energy, true);   // warm-up
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    for (int i = 0; i < reps; i++) s->conv->conv(s->M, s->H, s->energy, false);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? (double)ms / reps : -1.0;
}

int refgpu_get_h(void *h, double *H)
{
    refgpu_s *s = (refgpu_s *)h;
    s->conv->conv(s->M, s->H, s->energy, true);
    if (!s->H()->copy_to_cpuvec(s->Hc)) return 1;
    memcpy(H, s->Hc.data(), sizeof(double) * 3 * s->n);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

void refgpu_destroy(void *h)
{
    refgpu_s *s = (refgpu_s *)h;
    if (!s) return;
    delete s->conv;
    delete s;
}

}  // extern "C"
