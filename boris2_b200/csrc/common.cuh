// Common device/host helpers for the B200 micromagnetic path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define BM_HD __host__ __device__ __forceinline__

template <typename T> struct cpx_t;
template <> struct alignas(8) cpx_t<float> { float x, y; };
template <> struct alignas(16) cpx_t<double> { double x, y; };
template <typename T> using cpx = cpx_t<T>;

template <typename T> BM_HD cpx<T> mk(T a, T b) { cpx<T> r; r.x = a; r.y = b; return r; }
template <typename T> BM_HD cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> BM_HD cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> BM_HD cpx<T> cmul(cpx<T> a, cpx<T> b) { return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename T> BM_HD cpx<T> cscale(cpx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
template <typename T> BM_HD cpx<T> conj(cpx<T> a) { return mk<T>(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse): s = -1 gives -i*a, s = +1 gives +i*a
template <typename T> BM_HD cpx<T> mul_i(cpx<T> a) { return mk<T>(-a.y, a.x); }
template <typename T> BM_HD cpx<T> mul_mi(cpx<T> a) { return mk<T>(a.y, -a.x); }

#ifdef __CUDACC__
// Asynchronous global -> shared copy of one element (4, 8 or 16 bytes); when !valid the
// destination is zero-filled and nothing is read (src must still be a mapped address).
template <int BYTES>
__device__ __forceinline__ void cp_async_el(void *smem, const void *gmem, bool valid)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int src = valid ? BYTES : 0;
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N committed groups of this thread are still in flight
template <int N> __device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
template <typename T>
__device__ __forceinline__ void cp_async_cpx(cpx<T> *smem, const cpx<T> *gmem, bool valid)
{
    cp_async_el<sizeof(cpx<T>)>(smem, gmem, valid);
}
template <typename T>
__device__ __forceinline__ void cp_async_real(T *smem, const T *gmem, bool valid)
{
    cp_async_el<sizeof(T)>(smem, gmem, valid);
}
#endif

// Physical constants (the reference's BorisLib/Funcs_Math_base.h:9,16)
#define BM_MU0 1.256637061435916e-6
#define BM_GAMMA 2.212761569e5
// StageArgs::diag bits: the step's first evaluation (|M x Heff| / |M|^2), its last stage
// (|M - M_start| / (dT GAMMA |M|^2)), and the set's last launch (publishes the maxima)
#define BM_DIAG_MXH 1
#define BM_DIAG_DMDT 2
#define BM_DIAG_PUBLISH 4

// module bits
#define BM_MOD_DEMAG 1
#define BM_MOD_EXCH 2
#define BM_MOD_IDMI 4
#define BM_MOD_ANIUNI 8
#define BM_MOD_ZEEMAN 16

// StepState.error bits (sticky until the next bm_set_m)
#define BM_ERR_NONFINITE 1   // a stage produced a NaN or infinite M or error estimate
#define BM_ERR_WAIT 2        // a kernel's bounded wait on its own bulk copies gave up

// device-resident step state shared by all kernels of a solver
struct StepState {
    double time, stagetime, dT, dT_last;
    double lte, last_lte;
    double tol, dT_incr, dT_min, dT_max;
    long long accepted, rejected, attempts;
    int primed, reject_flag, need_restore, error;
    unsigned long long lte_bits;   // running max of lte (non-negative doubles order like their bits)
    unsigned int blocks_done;      // last-block-done counter for grid reductions
    unsigned int restore_done;
    int eval_order;
    int pad_;
    // evaluation speedup: fields saved so far (<= es_K) and the times they were saved at
    int es_saved, es_K;
    double es_t[6];
    // evaluation speedup under RKDP54: the decision for the current evaluation (0 none, 1 compute and
    // save into es_slot at time es_tnew, 2 extrapolate with the weights es_a), whether that save
    // replaces the field of an already saved time (es_pad 1), and the reference's `available` flag
    // (the previous step completed)
    int es_mode, es_slot, es_available, es_pad;
    double es_tnew;
    double es_a[6];
    // torque and dm/dt diagnostics (the reference's Get_mxh / Get_dmdt): calc_* are requests from the
    // host; the launches that evaluate them take running maxima into *_acc (non-negative doubles as
    // bits), and the last block of the set's last launch publishes mxh / dmdt and clears both
    int calc_mxh, calc_dmdt;
    unsigned long long mxh_acc, dmdt_acc;
    double mxh, dmdt;
};
