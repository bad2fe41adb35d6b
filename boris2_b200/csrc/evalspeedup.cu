// Evaluation speedup (the reference's `evalspeedup` levels 1..6: step, linear, quadratic, cubic,
// quartic, quintic), following DemagCUDA::UpdateField (Boris/DemagCUDA.cpp:106-470) with
// ODECommon_Base::Check_Step_Update / Get_EvalStep_Time (Boris/DiffEq_CommonBase_Iterate.cpp:1536,1639;
// dTspeedup linked to dT):
//   - an evaluation that computes the demag field saves H - S M (S the self-demag coefficients,
//     Demag_EvalSpeedup_AddField_SubSelf, Boris/DemagCUDA.cu:46) in the next free slot while fewer than
//     es_K are saved, then in the slot the reference's ordering rule picks (Boris/DemagCUDA.cpp:180-280:
//     the first slot when the saved times increase, else the first slot whose time is below its
//     predecessor's, else the last), with its evaluation time;
//   - an evaluation that extrapolates uses sum_k a_k (H_k - S M_k) + S M with the Lagrange weights a_k
//     of the saved times at the evaluation time (Demag_EvalSpeedup_AddExtrapField_AddSelf,
//     Boris/DemagCUDA.cu:64-265).
// Which evaluation does which:
//   RK4     (sel 0) the first evaluation of a step saves, the others compute in full until es_K are
//           saved and extrapolate after (two captured step graphs chosen on the host). The reference
//           also saves at the other evaluations while fewer than es_K are saved; under RK4 its second
//           and third evaluations share the time t + dT/2, which for es_K >= 3 would give two equal
//           saved times (a zero Lagrange denominator), so saves are kept to the step starts here.
//   RKDP54  (sel 1) the reference's rule as is, decided on the device per evaluation by k_es_decide:
//           compute and save when the previous step completed (`available`: evaluation 0 of an attempt
//           that follows an accepted step) or fewer than es_K are saved, else extrapolate. A rejected
//           step clears `available`, so the repeated evaluation 0 extrapolates, with the field saved at
//           the rejected step's end kept in its slot, as in the reference. One deviation: a save at a
//           time already saved replaces that slot (the last stage, c = 1, and the next step's first
//           evaluation share t + dT; at level 6 the reference's rule keeps both, a zero Lagrange
//           denominator).
// The reference does this on the real-space field; here it is done on S1, the x spectrum the y/z
// passes consume and produce. Every step of it is linear and S is diagonal, so the field the stage
// kernel transforms back is the same: an extrapolating evaluation replaces the y forward, z and y
// inverse passes with one pass over S1 and the saved slots.
#include "kernels.h"

namespace {

// the slot the next saved field goes to (Boris/DemagCUDA.cpp:158-280)
__device__ __forceinline__ int es_slot_rule(const StepState *st)
{
    const int K = st->es_K, saved = st->es_saved;
    if (saved < K) return saved;
    if (K == 1) return 0;
    bool inc = true;
    for (int k = 1; k < K; k++) inc = inc && (st->es_t[k] > st->es_t[k - 1]);
    if (inc) return 0;
    for (int j = 1; j < K - 1; j++)
        if (st->es_t[j - 1] > st->es_t[j]) return j;
    return K - 1;
}

// slot of the field being saved: RK4 (sel 0) from the rule, RKDP54 (sel 1) as decided
__device__ __forceinline__ int es_slot(const StepState *st, int sel) { return sel ? st->es_slot : es_slot_rule(st); }

// whether a save kernel (want 1) or the extrapolation (want 2) runs for this evaluation (sel 1)
__device__ __forceinline__ bool es_off(const StepState *st, int sel, int want)
{
    return sel && *((volatile const int *)&st->es_mode) != want;
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
                                                double c0, double c1, double c2, const StepState *st, int sel)
{
    if (es_off(st, sel, 1)) return;
    const int c = blockIdx.y;
    const T f = (T)es_coef(c, c0, c1, c2);
    const cpx<T> *src = S1 + c * plane;
    cpx<T> *g = G + ((long long)es_slot(st, sel) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> v = src[i];
        g[i] = mk<T>(f * v.x, f * v.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_post(const cpx<T> *__restrict__ S1, cpx<T> *__restrict__ G, long long plane,
                                                 const StepState *st, int sel)
{
    if (es_off(st, sel, 1)) return;
    const int c = blockIdx.y;
    const cpx<T> *src = S1 + c * plane;
    cpx<T> *g = G + ((long long)es_slot(st, sel) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> h = src[i], s = g[i];
        g[i] = mk<T>(h.x - s.x, h.y - s.y);
    }
}

__global__ void k_es_commit(StepState *st, int sel)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        if (es_off(st, sel, 1)) return;
        if (sel && st->es_pad) return;   // replaced the field of an already saved time
        const int slot = es_slot(st, sel);
        // the reference keeps the time of a level-1 (step) cycling save unchanged
        if (!(sel && st->es_K == 1 && st->es_saved >= 1)) st->es_t[slot] = sel ? st->es_tnew : st->time;
        if (st->es_saved < st->es_K) st->es_saved++;
    }
}

// RKDP54: the decision of one evaluation (eval 0..5 at time + c_eval dT): compute and save
// (es_mode 1, slot and time recorded) when the previous step completed and this is evaluation 0, or
// while fewer than es_K are saved; else extrapolate (es_mode 2, Lagrange weights recorded). Evaluations
// 1..5 of a rejected attempt do nothing (es_mode 0; their other launches are skipped as well).
__global__ void k_es_decide(StepState *st, int eval, double c_eval)
{
    if (threadIdx.x || blockIdx.x) return;
    if (eval > 0 && st->reject_flag) { st->es_mode = 0; return; }
    const int K = st->es_K, saved = st->es_saved;
    const double t = st->time + c_eval * st->dT;
    if ((eval == 0 && st->es_available) || saved < K) {
        st->es_mode = 1;
        st->es_tnew = t;
        // a save at a time already saved replaces that slot (the last stage and the next step's first
        // evaluation share t + dT; two fields at one time would give a zero Lagrange denominator)
        for (int k = 0; k < saved; k++)
            if (st->es_t[k] == t) {
                st->es_slot = k;
                st->es_pad = 1;   // no new slot
                return;
            }
        st->es_slot = es_slot_rule(st);
        st->es_pad = 0;
        return;
    }
    st->es_mode = 2;
    for (int k = 0; k < 6; k++) {
        double w = 0.0;
        if (k < K) {
            w = 1.0;
            for (int j = 0; j < K; j++)
                if (j != k) w *= (t - st->es_t[j]) / (st->es_t[k] - st->es_t[j]);
        }
        st->es_a[k] = w;
    }
}

// Lagrange weights of the saved times at the evaluation time: computed here (RK4, sel 0) or recorded by
// k_es_decide (RKDP54, sel 1)
template <typename T>
__device__ __forceinline__ void es_weights(const StepState *st, int sel, double c_eval, T a[6])
{
    bm_es_weights<T>(st, sel, c_eval, a);
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_extrap(cpx<T> *__restrict__ S1, const cpx<T> *__restrict__ G, long long plane,
                                                   double c0, double c1, double c2, const StepState *st, double c_eval,
                                                   int sel)
{
    const int K = st->es_K;
    if (sel ? es_off(st, sel, 2) : st->es_saved < K) return;
    T a[6];
    es_weights<T>(st, sel, c_eval, a);
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
__global__ void __launch_bounds__(256) k_es_pre_batch(const EsMesh *__restrict__ tab, const StepState *st, int sel)
{
    if (es_off(st, sel, 1)) return;
    const EsMesh &e = tab[blockIdx.y / 3];
    const int c = blockIdx.y % 3;
    const long long plane = e.plane;
    const T f = (T)e.cs[c];
    const cpx<T> *src = (const cpx<T> *)e.S1 + c * plane;
    cpx<T> *g = (cpx<T> *)e.G + ((long long)es_slot(st, sel) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> v = src[i];
        g[i] = mk<T>(f * v.x, f * v.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_post_batch(const EsMesh *__restrict__ tab, const StepState *st, int sel)
{
    if (es_off(st, sel, 1)) return;
    const EsMesh &e = tab[blockIdx.y / 3];
    const int c = blockIdx.y % 3;
    const long long plane = e.plane;
    const cpx<T> *src = (const cpx<T> *)e.S1 + c * plane;
    cpx<T> *g = (cpx<T> *)e.G + ((long long)es_slot(st, sel) * 3 + c) * plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane; i += (long long)gridDim.x * blockDim.x) {
        cpx<T> h = src[i], s = g[i];
        g[i] = mk<T>(h.x - s.x, h.y - s.y);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_es_extrap_batch(const EsMesh *__restrict__ tab, const StepState *st, double c_eval,
                                                         int sel)
{
    const int K = st->es_K;
    if (sel ? es_off(st, sel, 2) : st->es_saved < K) return;
    T a[6];
    es_weights<T>(st, sel, c_eval, a);
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
int launch_es_pre_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, cudaStream_t s, int sel)
{
    k_es_pre_batch<T><<<es_grid_batch(max_plane, nmesh), 256, 0, s>>>(tab, st, sel);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_post_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, cudaStream_t s, int sel)
{
    k_es_post_batch<T><<<es_grid_batch(max_plane, nmesh), 256, 0, s>>>(tab, st, sel);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_extrap_batch(const EsMesh *tab, int nmesh, long long max_plane, const StepState *st, double c_eval,
                           cudaStream_t s, int sel)
{
    k_es_extrap_batch<T><<<es_grid_batch(max_plane, nmesh), 256, 0, s>>>(tab, st, c_eval, sel);
    return (int)cudaGetLastError();
}

template int launch_es_pre_batch<float>(const EsMesh *, int, long long, const StepState *, cudaStream_t, int);
template int launch_es_pre_batch<double>(const EsMesh *, int, long long, const StepState *, cudaStream_t, int);
template int launch_es_post_batch<float>(const EsMesh *, int, long long, const StepState *, cudaStream_t, int);
template int launch_es_post_batch<double>(const EsMesh *, int, long long, const StepState *, cudaStream_t, int);
template int launch_es_extrap_batch<float>(const EsMesh *, int, long long, const StepState *, double, cudaStream_t, int);
template int launch_es_extrap_batch<double>(const EsMesh *, int, long long, const StepState *, double, cudaStream_t, int);


template <typename T>
int launch_es_pre(const cpx<T> *S1, cpx<T> *G, long long plane, const double *cs, const StepState *st, cudaStream_t s, int sel)
{
    k_es_pre<T><<<es_grid(plane), 256, 0, s>>>(S1, G, plane, cs[0], cs[1], cs[2], st, sel);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_post(const cpx<T> *S1, cpx<T> *G, long long plane, const StepState *st, cudaStream_t s, int sel)
{
    k_es_post<T><<<es_grid(plane), 256, 0, s>>>(S1, G, plane, st, sel);
    return (int)cudaGetLastError();
}

int launch_es_commit(StepState *st, cudaStream_t s, int sel)
{
    k_es_commit<<<1, 32, 0, s>>>(st, sel);
    return (int)cudaGetLastError();
}

int launch_es_decide(StepState *st, int eval, double c_eval, cudaStream_t s)
{
    k_es_decide<<<1, 32, 0, s>>>(st, eval, c_eval);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_es_extrap(cpx<T> *S1, const cpx<T> *G, long long plane, const double *cs, const StepState *st, double c_eval,
                     cudaStream_t s, int sel)
{
    k_es_extrap<T><<<es_grid(plane), 256, 0, s>>>(S1, G, plane, cs[0], cs[1], cs[2], st, c_eval, sel);
    return (int)cudaGetLastError();
}

template int launch_es_pre<float>(const cpx<float> *, cpx<float> *, long long, const double *, const StepState *, cudaStream_t, int);
template int launch_es_pre<double>(const cpx<double> *, cpx<double> *, long long, const double *, const StepState *, cudaStream_t,
                                   int);
template int launch_es_post<float>(const cpx<float> *, cpx<float> *, long long, const StepState *, cudaStream_t, int);
template int launch_es_post<double>(const cpx<double> *, cpx<double> *, long long, const StepState *, cudaStream_t, int);
template int launch_es_extrap<float>(cpx<float> *, const cpx<float> *, long long, const double *, const StepState *, double,
                                     cudaStream_t, int);
template int launch_es_extrap<double>(cpx<double> *, const cpx<double> *, long long, const double *, const StepState *,
                                      double, cudaStream_t, int);
