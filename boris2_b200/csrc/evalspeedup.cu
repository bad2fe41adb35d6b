// Evaluation speedup of RK4 (the reference's `evalspeedup` levels 1..6: step, linear, quadratic,
// cubic, quartic, quintic), following DemagCUDA::UpdateField (Boris/DemagCUDA.cpp:106-470) with
// ODECommon_Base::Check_Step_Update / Get_EvalStep_Time (Boris/DiffEq_CommonBase_Iterate.cpp:1536,1639;
// dTspeedup linked to dT, so the field is computed at the first evaluation of every step):
//   - the first evaluation of a step computes the demag field and saves H - S M (S the self-demag
//     coefficients, Demag_EvalSpeedup_AddField_SubSelf, Boris/DemagCUDA.cu:46) in the next free slot,
//     then in the slot holding the earliest time;
//   - the other evaluations compute the field in full until es_K fields are saved, then use
//     sum_k a_k (H_k - S M_k) + S M with the Lagrange weights a_k of the saved times at the
//     evaluation time (Demag_EvalSpeedup_AddExtrapField_AddSelf, Boris/DemagCUDA.cu:64-265).
// The reference does this on the real-space field; here it is done on S1, the x spectrum the y/z
// passes consume and produce. Every step of it is linear and S is diagonal, so the field the stage
// kernel transforms back is the same: an extrapolating evaluation replaces the y forward, z and y
// inverse passes with one pass over S1 and the saved slots.
#include "kernels.h"

namespace {

__device__ __forceinline__ int es_slot(const StepState *st)
{
    int K = st->es_K, saved = st->es_saved;
    if (saved < K) return saved;
    int slot = 0;
    for (int k = 1; k < K; k++)
        if (st->es_t[k] < st->es_t[slot]) slot = k;
    return slot;
}

// grid: x covers one component plane (capped, grid-stride), y = the 3 components
dim3 es_grid(long long plane)
{
    long long b = (plane + 255) / 256;
    long long cap = 148LL * 4;
    return dim3((unsigned)(b < cap ? (b < 1 ? 1 : b) : cap), 3);
}

__device__ __forceinline__ double es_coef(int c, double c0, double c1, double c2)
{
    return c == 0 ? c0 : (c == 1 ? c1 : c2);
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_pre(const cpx<T> *__restrict__ S1, cpx<T> *__restrict__ G, long long plane,
                                                double c0, double c1, double c2, const StepState *st)
{
    const int c = blockIdx.y;
    const T f = (T)es_coef(c, c0, c1, c2);
    const cpx<T> *src = S1 + c * plane;
    cpx<T> *g = G + ((long long)es_slot(st) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> v = src[i];
        g[i] = mk<T>(f * v.x, f * v.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_post(const cpx<T> *__restrict__ S1, cpx<T> *__restrict__ G, long long plane,
                                                 const StepState *st)
{
    const int c = blockIdx.y;
    const cpx<T> *src = S1 + c * plane;
    cpx<T> *g = G + ((long long)es_slot(st) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> h = src[i], s = g[i];
        g[i] = mk<T>(h.x - s.x, h.y - s.y);
    }
}

__global__ void k_es_commit(StepState *st)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int slot = es_slot(st);
        st->es_t[slot] = st->time;
        if (st->es_saved < st->es_K) st->es_saved++;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_extrap(cpx<T> *__restrict__ S1, const cpx<T> *__restrict__ G, long long plane,
                                                   double c0, double c1, double c2, const StepState *st, double c_eval)
{
    const int K = st->es_K;
    if (st->es_saved < K) return;
    // Lagrange weights of the saved times at the evaluation time
    const double t = st->time + c_eval * st->dT;
    T a[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double w = 0.0;
        if (k < K) {
            w = 1.0;
            for (int j = 0; j < K; j++)
                if (j != k) w *= (t - st->es_t[j]) / (st->es_t[k] - st->es_t[j]);
        }
        a[k] = (T)w;
    }
    const int c = blockIdx.y;
    const T f = (T)es_coef(c, c0, c1, c2);
    cpx<T> *dst = S1 + c * plane;
    const long long slot_stride = 3 * plane;
    const cpx<T> *g = G + c * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> m = dst[i];
        T x = f * m.x, y = f * m.y;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            if (k < K) {
                cpx<T> v = g[k * slot_stride + i];
                x += a[k] * v.x;
                y += a[k] * v.y;
            }
        }
        dst[i] = mk<T>(x, y);
    }
}

// batched: blockIdx.y = 3 * mesh + component; blocks beyond a mesh's plane do nothing
dim3 es_grid_batch(long long max_plane, int nmesh)
{
    long long b = (max_plane + 255) / 256;
    long long cap = 64;
    return dim3((unsigned)(b < cap ? (b < 1 ? 1 : b) : cap), 3 * nmesh);
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_pre_batch(const EsMesh *__restrict__ tab, const StepState *st)
{
    const EsMesh &e = tab[blockIdx.y / 3];
    const int c = blockIdx.y % 3;
    const long long plane = e.plane;
    const T f = (T)e.cs[c];
    const cpx<T> *src = (const cpx<T> *)e.S1 + c * plane;
    cpx<T> *g = (cpx<T> *)e.G + ((long long)es_slot(st) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> v = src[i];
        g[i] = mk<T>(f * v.x, f * v.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_post_batch(const EsMesh *__restrict__ tab, const StepState *st)
{
    const EsMesh &e = tab[blockIdx.y / 3];
    const int c = blockIdx.y % 3;
    const long long plane = e.plane;
    const cpx<T> *src = (const cpx<T> *)e.S1 + c * plane;
    cpx<T> *g = (cpx<T> *)e.G + ((long long)es_slot(st) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> h = src[i], s = g[i];
        g[i] = mk<T>(h.x - s.x, h.y - s.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_extrap_batch(const EsMesh *__restrict__ tab, const StepState *st, double c_eval)
{
    const int K = st->es_K;
    if (st->es_saved < K) return;
    const double t = st->time + c_eval * st->dT;
    T a[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double w = 0.0;
        if (k < K) {
            w = 1.0;
            for (int j = 0; j < K; j++)
                if (j != k) w *= (t - st->es_t[j]) / (st->es_t[k] - st->es_t[j]);
        }
        a[k] = (T)w;
    }
    const EsMesh &e = tab[blockIdx.y / 3];
    const int c = blockIdx.y % 3;
    const long long plane = e.plane;
    const T f = (T)e.cs[c];
    cpx<T> *dst = (cpx<T> *)e.S1 + c * plane;
    const long long slot_stride = 3 * plane;
    const cpx<T> *g = (const cpx<T> *)e.G + c * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> m = dst[i];
        T x = f * m.x, y = f * m.y;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            if (k < K) {
                cpx<T> v = g[k * slot_stride + i];
                x += a[k] * v.x;
                y += a[k] * v.y;
            }
        }
        dst[i] = mk<T>(x, y);
    }
}

}  // namespace

template <typename T>
int launch_es_pre_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, cudaStream_t s)
{
    k_es_pre_batch<T><<<es_grid_batch(max_plane, nmesh), 256, 0, s>>>(tab, st);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_post_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, cudaStream_t s)
{
    k_es_post_batch<T><<<es_grid_batch(max_plane, nmesh), 256, 0, s>>>(tab, st);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_extrap_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, double c_eval,
                           cudaStream_t s)
{
    k_es_extrap_batch<T><<<es_grid_batch(max_plane, nmesh), 256, 0, s>>>(tab, st, c_eval);
    return (int)cudaGetLastError();
}

template int launch_es_pre_batch<float>(const EsMesh *, int, long long, const StepState *, cudaStream_t);
template int launch_es_pre_batch<double>(const EsMesh *, int, long long, const StepState *, cudaStream_t);
template int launch_es_post_batch<float>(const EsMesh *, int, long long, const StepState *, cudaStream_t);
template int launch_es_post_batch<double>(const EsMesh *, int, long long, const StepState *, cudaStream_t);
template int launch_es_extrap_batch<float>(const EsMesh *, int, long long, const StepState *, double, cudaStream_t);
template int launch_es_extrap_batch<double>(const EsMesh *, int, long long, const StepState *, double, cudaStream_t);


template <typename T>
int launch_es_pre(const cpx<T> *S1, cpx<T> *G, long long plane, const double *cs, const StepState *st, cudaStream_t s)
{
    k_es_pre<T><<<es_grid(plane), 256, 0, s>>>(S1, G, plane, cs[0], cs[1], cs[2], st);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_post(const cpx<T> *S1, cpx<T> *G, long long plane, const StepState *st, cudaStream_t s)
{
    k_es_post<T><<<es_grid(plane), 256, 0, s>>>(S1, G, plane, st);
    return (int)cudaGetLastError();
}

int launch_es_commit(StepState *st, cudaStream_t s)
{
    k_es_commit<<<1, 32, 0, s>>>(st);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_extrap(cpx<T> *S1, const cpx<T> *G, long long plane, const double *cs, const StepState *st, double c_eval,
                     cudaStream_t s)
{
    k_es_extrap<T><<<es_grid(plane), 256, 0, s>>>(S1, G, plane, cs[0], cs[1], cs[2], st, c_eval);
    return (int)cudaGetLastError();
}

template int launch_es_pre<float>(const cpx<float> *, cpx<float> *, long long, const double *, const StepState *, cudaStream_t);
template int launch_es_pre<double>(const cpx<double> *, cpx<double> *, long long, const double *, const StepState *, cudaStream_t);
template int launch_es_post<float>(const cpx<float> *, cpx<float> *, long long, const StepState *, cudaStream_t);
template int launch_es_post<double>(const cpx<double> *, cpx<double> *, long long, const StepState *, cudaStream_t);
template int launch_es_extrap<float>(cpx<float> *, const cpx<float> *, long long, const double *, const StepState *, double,
                                     cudaStream_t);
template int launch_es_extrap<double>(cpx<double> *, const cpx<double> *, long long, const double *, const StepState *,
                                      double, cudaStream_t);
