// Allocation-free batched line FFT (bm_fft_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a transform:
// code running while another component holds a fixed, pre-reserved device-memory budget,
// or a solver that is in the middle of an asynchronous step where a cudaMalloc/cudaFree
// (which may synchronise the device) would stall or break its pipeline. For them this entry
// point runs the same batched FFT kernel as the rest of the library on buffers the caller
// already owns, and keeps its only scratch (the twiddle table) in a file-scope device array
// that every GPU loading the library holds until the process exits.
#include "kernels.h"
#include <string>

// records the library's last-error text (defined with the rest of the C ABI in api.cu)
int bm_set_error(int code, const std::string &msg);

#define BM_NOALLOC_MAX_L 4096   // longest supported line: 4096 complex FP64 twiddles = 64 KiB

// Scratch for the twiddle table. In host code this name is only a stand-in for the device
// symbol: its device address is looked up with cudaGetSymbolAddress once per device.
static __device__ __align__(256) cpx<double> g_noalloc_tw[BM_NOALLOC_MAX_L];

#define BM_NOALLOC_MAX_DEV 64
static cpx<double> *s_tw_dev[BM_NOALLOC_MAX_DEV];   // device address per device ordinal (null until set up)

// tw[m] = exp(-2 pi i m / L), rebuilt on every call because calls share the array
__global__ void k_noalloc_twiddles(cpx<double> *tw, int L)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < L; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)m / (double)L, &s, &c);
        tw[m] = mk<double>(c, -s);
    }
}

extern "C" int bm_fft_noalloc(int device, int L, int howmany, int inverse, const double *in, double *out, void *stream)
{
    if (device < 0 || device >= BM_NOALLOC_MAX_DEV) return bm_set_error(1, "bm_fft_noalloc: bad device index");
    if (L < 1 || L > BM_NOALLOC_MAX_L)
        return bm_set_error(1, "bm_fft_noalloc: line length must be in [1, 4096] (the scratch twiddle table holds 4096 entries)");
    if (howmany < 1) return bm_set_error(1, "bm_fft_noalloc: howmany must be >= 1");
    if (!in || !out) return bm_set_error(1, "bm_fft_noalloc: null device buffer");
    FFTPlan P;
    if (!bm_make_plan(L, P)) return bm_set_error(5, "bm_fft_noalloc: line length must be 2^p or 3*2^p");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bm_set_error(2, std::string("bm_fft_noalloc: cudaSetDevice: ") + cudaGetErrorString(e));
    // one-time set-up on this device (with it current): the device address of the scratch array
    if (!s_tw_dev[device]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_tw);
        if (e != cudaSuccess || !p)
            return bm_set_error(2, std::string("bm_fft_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        s_tw_dev[device] = (cpx<double> *)p;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cpx<double> *tw = s_tw_dev[device];
    k_noalloc_twiddles<<<(L + 255) / 256, 256, 0, s>>>(tw, L);
    e = cudaGetLastError();
    if (e != cudaSuccess) return bm_set_error(2, std::string("bm_fft_noalloc: twiddle kernel: ") + cudaGetErrorString(e));
    if ((const void *)in != (const void *)out) {
        e = cudaMemcpyAsync(out, in, sizeof(double) * 2 * (size_t)L * howmany, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return bm_set_error(2, std::string("bm_fft_noalloc: copy: ") + cudaGetErrorString(e));
    }
    int rc = launch_fft_strided<double>((cpx<double> *)out, P, tw, 1, L, howmany, 0, 1, inverse != 0, s);
    if (rc) return bm_set_error(2, "bm_fft_noalloc: FFT launch failed (" + std::to_string(rc) + ")");
    return 0;
}
