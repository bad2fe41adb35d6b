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
// symbol: its device address is looked up with cudaGetSymbolAddress, with the device current,
// and only that address is passed to the kernels.
static __device__ __align__(256) cpx<double> g_noalloc_tw[BM_NOALLOC_MAX_L];

#define BM_NOALLOC_MAX_DEV 64
// device address per device ordinal, for calls made while the stream is being captured (where a
// symbol lookup, which may load the module, is not allowed); refreshed by every uncaptured call
static cpx<double> *s_tw_dev[BM_NOALLOC_MAX_DEV];

// tw[m] = exp(-2 pi i m / L), rebuilt on every call because calls share the array
__global__ void k_noalloc_twiddles(cpx<double> *tw, int L)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < L; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)m / (double)L, &s, &c);
        tw[m] = mk<double>(c, -s);
    }
}

namespace {
// the body of bm_fft_noalloc, run with `device` current
int fft_noalloc_on_device(int device, const FFTPlan &P, int L, int howmany, int inverse, const double *in, double *out,
                          cudaStream_t s)
{
    // The scratch array's device address. Outside stream capture it is looked up on every call
    // (cheap, allocates nothing), so a context that was reset and re-created since the last call
    // gets the address in its new module; under capture the address recorded by the last
    // uncaptured call on this device is used.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return bm_set_error(2, std::string("bm_fft_noalloc: cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    if (cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_tw);
        if (e != cudaSuccess || !p)
            return bm_set_error(2, std::string("bm_fft_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        s_tw_dev[device] = (cpx<double> *)p;
    } else if (!s_tw_dev[device]) {
        return bm_set_error(4, "bm_fft_noalloc: the first call on a device must come before any stream capture");
    }
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
}  // namespace

extern "C" int bm_fft_noalloc(int device, int L, int howmany, int inverse, const double *in, double *out, void *stream)
{
    if (device < 0 || device >= BM_NOALLOC_MAX_DEV) return bm_set_error(1, "bm_fft_noalloc: bad device index");
    if (L < 1 || L > BM_NOALLOC_MAX_L)
        return bm_set_error(1, "bm_fft_noalloc: line length must be in [1, 4096] (the scratch twiddle table holds 4096 entries)");
    if (howmany < 1) return bm_set_error(1, "bm_fft_noalloc: howmany must be >= 1");
    if (!in || !out) return bm_set_error(1, "bm_fft_noalloc: null device buffer");
    FFTPlan P;
    if (!bm_make_plan(L, P)) return bm_set_error(5, "bm_fft_noalloc: line length must be 2^p or 3*2^p");
    // the caller's current device is restored before returning, on every path
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return bm_set_error(2, std::string("bm_fft_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    if (prev != device) {
        e = cudaSetDevice(device);
        if (e != cudaSuccess) return bm_set_error(2, std::string("bm_fft_noalloc: cudaSetDevice: ") + cudaGetErrorString(e));
    }
    int rc = fft_noalloc_on_device(device, P, L, howmany, inverse, in, out, (cudaStream_t)stream);
    if (prev != device) {
        e = cudaSetDevice(prev);
        if (e != cudaSuccess && rc == 0)
            return bm_set_error(2, std::string("bm_fft_noalloc: restoring the caller's device: ") + cudaGetErrorString(e));
    }
    return rc;
}
