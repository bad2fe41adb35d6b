// 3D y passes (S1 -> S2 forward, S2 -> S1 inverse) as a persistent kernel whose input tiles arrive by
// bulk tensor copies (TMA) into a two-stage shared-memory ring: while a block transforms one column
// tile, the next tile of its work list is already in flight, so the loads of a block no longer wait
// behind its own transforms and stores (the one-shot kernels of demag.cu keep at most their own
// tile's loads in flight).
//
// Work item (column tile bx, plane z, component c), items bx fastest; a block takes items
// blockIdx.x, + gridDim.x, ... The input plane of an item is a [R_in][LX] block of complex values
// (R_in = n.y forward, Ny inverse); a tensor map over the whole array viewed as 2D rows x LX (in
// 4-byte words: 2 per FP32 complex, 4 per FP64) copies its [R_in][W] column tile in boxes of at most
// 256 rows. The transform is the two-level register FFT of k_ypass_reg (Ny = P * Q): stage 1 reads
// x[n1 + P n2] from the staged tile instead of global memory, one shared transpose, stage 2 stores
// straight to global memory (forward: all Ny rows; inverse: rows < n.y).
#include "kernels.h"
#include "regfft.cuh"
#include "tma.cuh"

#include <cudaTypedefs.h>

namespace {

template <typename T>
__device__ __forceinline__ bool yt_gated_out(const StepState *st, int gate)
{
    if (gate == BM_GATE_ALWAYS || st == nullptr) return false;
    if (gate == BM_GATE_ACCEPTED) return *((volatile const int *)&st->reject_flag) != 0;
    if (gate == BM_GATE_ES || gate == BM_GATE_ES_ACC)
        return *((volatile const int *)&st->es_mode) != 1 ||
               (gate == BM_GATE_ES_ACC && *((volatile const int *)&st->reject_flag) != 0);
    return *((volatile const int *)&st->need_restore) == 0;
}

struct YTmaGeom {
    int R_in;    // input rows per plane
    int BR;      // rows per box (<= 256)
    int nbox;    // boxes per tile
    int bufel;   // complex values per ring buffer (nbox * BR * W rounded up to 128 bytes)
};

constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s per bulk-copy wait

template <typename T, int P, int Q, bool INV>
__global__ void __launch_bounds__(yreg_maxt<T>::v) k_ypass_tma(YZArgs<T> a, const __grid_constant__ CUtensorMap map,
                                                               YTmaGeom g)
{
    if (yt_gated_out<T>(a.st, a.gate)) return;
    extern __shared__ __align__(128) unsigned char smraw[];
    constexpr int L = P * Q;
    constexpr int EF = (int)(sizeof(cpx<T>) / 4);   // 4-byte words per complex value
    const int W = a.W, ny = a.ny, LX = a.LX, nz = a.nz;
    const int lw = __ffs(W) - 1;
    const int tid = threadIdx.x;
    const int w = tid & (W - 1), r = tid >> lw;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw);
    const size_t bufel = (size_t)g.bufel;   // both ring buffers start on 128-byte boundaries
    cpx<T> *buf0 = reinterpret_cast<cpx<T> *>(smraw + 128);
    cpx<T> *buf1 = buf0 + bufel;
    cpx<T> *sm = buf0 + 2 * bufel;   // transpose tile [L][W]
    const int nbx = (LX + W - 1) / W;
    const int nitems = nbx * nz * 3;
    // every box counts in full, the rows past the end of the array included
    const uint32_t tx_bytes = (uint32_t)((size_t)g.nbox * g.BR * W * sizeof(cpx<T>));
    int it = blockIdx.x;
    if (it >= nitems) return;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](int item, int sb) {
        const int bx = item % nbx, zc = item / nbx;   // zc = z + nz * c: the plane's row block
        cpx<T> *dstb = sb ? buf1 : buf0;
        mbar_arrive_expect_tx(&bar[sb], tx_bytes);
        for (int b = 0; b < g.nbox; b++)
            tma_load_2d(dstb + (size_t)b * g.BR * W, &map, bx * W * EF, zc * g.R_in + b * g.BR, &bar[sb]);
    };
    if (tid == 0) issue(it, 0);
    for (int k = 0; it < nitems; it += gridDim.x, k++) {
        const int sb = k & 1;
        const int nxt = it + (int)gridDim.x;
        // the other buffer was read in the previous item, before its trailing barrier
        if (tid == 0 && nxt < nitems) issue(nxt, sb ^ 1);
        const bool ok = mbar_wait_bounded(&bar[sb], (uint32_t)((k >> 1) & 1), kWaitNs);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) {
                if (a.st) atomicOr(&a.st->error, BM_ERR_WAIT);
                // the prefetch issued above must land before the block's shared memory goes away
                if (nxt < nitems) mbar_wait_bounded(&bar[sb ^ 1], (uint32_t)(((k + 1) >> 1) & 1), kWaitNs);
            }
            __syncthreads();
            return;
        }
        const cpx<T> *tile = sb ? buf1 : buf0;
        const int bx = it % nbx, zc = it / nbx;
        const int kx = bx * W + w;
        const bool colok = kx < LX;
        cpx<T> *dst = INV ? a.S1 + (long long)zc * ny * LX + kx : a.S2 + (long long)zc * L * LX + kx;
        if (r < P) {
            const int n1 = r;
            cpx<T> v[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; n2++) {
                const int e = n1 + P * n2;
                if (!INV) v[n2] = (n2 < Q / 2 && e < ny) ? tile[e * W + w] : mk<T>(0, 0);
                else v[n2] = tile[e * W + w];
            }
            RegFFT<T, Q, INV>::run(v, a.twy, P);
#pragma unroll
            for (int k2 = 0; k2 < Q; k2++) {
                cpx<T> t = v[k2];
                if (k2 > 0 && n1 > 0) {
                    cpx<T> tw = a.twy[n1 * k2];
                    if (INV) tw.y = -tw.y;
                    t = cmul(t, tw);
                }
                sm[(k2 * P + n1) * W + w] = t;
            }
        }
        __syncthreads();
        if (r < Q) {
            const int k2 = r;
            cpx<T> u[P];
#pragma unroll
            for (int n1 = 0; n1 < P; n1++) u[n1] = sm[(k2 * P + n1) * W + w];
            RegFFT<T, P, INV>::run(u, a.twy, Q);
            if (colok) {
#pragma unroll
                for (int k1 = 0; k1 < P; k1++) {
                    const int e = k2 + Q * k1;
                    if (!INV) dst[(long long)e * LX] = u[k1];
                    else if (k1 < P / 2 && e < ny) dst[(long long)e * LX] = u[k1];
                }
            }
        }
        __syncthreads();
    }
}

template <int L> struct yt_split {
    static constexpr int q = (L >= 1024) ? 32 : (L >= 256) ? 16 : (L >= 64) ? 8 : (L >= 16) ? 4 : 2;
    static constexpr int p = L / q;
};

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

template <typename T> size_t ytma_smem_bytes(int L, int W, const YTmaGeom &g)
{
    return 128 + (size_t)2 * g.bufel * sizeof(cpx<T>) + (size_t)L * W * sizeof(cpx<T>);
}

template <typename T, bool INV> YTmaGeom ytma_geom(const YZArgs<T> &a)
{
    YTmaGeom g;
    g.R_in = INV ? a.Ny : a.ny;
    g.BR = g.R_in < 256 ? g.R_in : 256;
    g.nbox = (g.R_in + g.BR - 1) / g.BR;
    const size_t bytes = ((size_t)g.nbox * g.BR * a.W * sizeof(cpx<T>) + 127) & ~(size_t)127;
    g.bufel = (int)(bytes / sizeof(cpx<T>));
    return g;
}

bool ypass_has_tma(int Ny)
{
    return Ny == 8 || Ny == 16 || Ny == 32 || Ny == 64 || Ny == 128 || Ny == 256 || Ny == 512 || Ny == 1024;
}

template <typename T, int Lc, bool INV>
int launch_ytma_len(const YZArgs<T> &a, cudaStream_t s)
{
    constexpr int P = yt_split<Lc>::p, Q = yt_split<Lc>::q;
    const YTmaGeom g = ytma_geom<T, INV>(a);
    const size_t smem = ytma_smem_bytes<T>(Lc, a.W, g);
    int nt = a.W * (P > Q ? P : Q);
    if (nt < 32) nt = 32;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return -1;
    // the array as 2D: rows of LX complex values (EF words each), 3 * nz planes of R_in rows
    constexpr int EF = (int)(sizeof(cpx<T>) / 4);
    CUtensorMap map;
    cuuint64_t dims[2] = {(cuuint64_t)a.LX * EF, (cuuint64_t)3 * a.nz * g.R_in};
    cuuint64_t strides[1] = {(cuuint64_t)a.LX * EF * 4};
    cuuint32_t box[2] = {(cuuint32_t)(a.W * EF), (cuuint32_t)g.BR};
    cuuint32_t estr[2] = {1, 1};
    void *base = INV ? (void *)a.S2 : (void *)a.S1;
    CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return 120;
    auto kern = k_ypass_tma<T, P, Q, INV>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem);
    if (e != cudaSuccess || per_sm < 1) return 121;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int nitems = ((a.LX + a.W - 1) / a.W) * a.nz * 3;
    int grid = per_sm * nsm;
    if (grid > nitems) grid = nitems;
    kern<<<grid, nt, smem, s>>>(a, map, g);
    return (int)cudaGetLastError();
}

}  // namespace

// whether both pipelined y passes apply to these arguments: transform length, a power-of-two tile
// width of at least 2 (a box row and its start are then multiples of 16 bytes), a row pitch that is
// a multiple of 16 bytes, the block size and the shared memory of the ring
template <typename T> bool ypass_tma_fits(const YZArgs<T> &a)
{
    if (!ypass_has_tma(a.Ny) || a.W < 2 || (a.W & (a.W - 1)) != 0 || a.nz < 1 || a.ny < 1) return false;
    if (((size_t)a.LX * sizeof(cpx<T>)) % 16 != 0) return false;
    const int q = (a.Ny >= 1024) ? 32 : (a.Ny >= 256) ? 16 : (a.Ny >= 64) ? 8 : (a.Ny >= 16) ? 4 : 2;
    const int p = a.Ny / q;
    if (a.W * (p > q ? p : q) > yreg_maxt<T>::v) return false;
    return ytma_smem_bytes<T>(a.Ny, a.W, ytma_geom<T, false>(a)) <= BM_SMEM_CAP &&
           ytma_smem_bytes<T>(a.Ny, a.W, ytma_geom<T, true>(a)) <= BM_SMEM_CAP;
}

// -1 when the pipelined y pass does not apply (ypass_tma_fits), else the launch status
template <typename T, bool INV>
int launch_ypass_tma(const YZArgs<T> &a, cudaStream_t s)
{
    if (!ypass_tma_fits<T>(a)) return -1;
    switch (a.Ny) {
    case 8: return launch_ytma_len<T, 8, INV>(a, s);
    case 16: return launch_ytma_len<T, 16, INV>(a, s);
    case 32: return launch_ytma_len<T, 32, INV>(a, s);
    case 64: return launch_ytma_len<T, 64, INV>(a, s);
    case 128: return launch_ytma_len<T, 128, INV>(a, s);
    case 256: return launch_ytma_len<T, 256, INV>(a, s);
    case 512: return launch_ytma_len<T, 512, INV>(a, s);
    case 1024: return launch_ytma_len<T, 1024, INV>(a, s);
    default: return -1;
    }
}

template bool ypass_tma_fits<float>(const YZArgs<float> &);
template bool ypass_tma_fits<double>(const YZArgs<double> &);
template int launch_ypass_tma<float, false>(const YZArgs<float> &, cudaStream_t);
template int launch_ypass_tma<float, true>(const YZArgs<float> &, cudaStream_t);
template int launch_ypass_tma<double, false>(const YZArgs<double> &, cudaStream_t);
template int launch_ypass_tma<double, true>(const YZArgs<double> &, cudaStream_t);
