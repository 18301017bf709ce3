// noalloc.cu -- filter design into caller memory, without allocating.
//
// Some callers of this library cannot call cudaMalloc: a data-acquisition
// pipeline that reserves all of its device memory when an observation starts
// and forbids allocation while samples stream in (an allocation can block
// behind running work, or fail once the reservation holds the device), a host
// framework whose own allocator owns the device and must account for every
// byte, or code that re-designs one trial's filter in the middle of a
// dedispersion pass and cannot afford the device-wide synchronisation that
// cudaMalloc/cudaFree bring.  msosm_prepare_dedisp_params_noalloc serves
// them: the caller passes the output (a device buffer of 2M complex values);
// the design kernel's scratch (twiddle tables and the trial's chirp
// parameters) lives in the fixed file-scope device array below instead of in
// allocated memory.
#include "msosm_b200.h"

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "host_prepare.hpp"
#include "kernels.hpp"

namespace {

using namespace msosm;

// Largest filter order served: M = 8192 (FFT 16384 points).
constexpr unsigned long kNoAllocMaxM = 8192;
// Scratch layout: [M twiddles exp(+2 pi i e/M)] [2M twiddles exp(-2 pi i e/(2M))]
// [ChirpParams], for the largest M.
constexpr size_t kTwiddleBytes = 3 * kNoAllocMaxM * sizeof(float2);
constexpr size_t kScratchBytes = kTwiddleBytes + 256;

// 196,864 bytes.  Every GPU that loads this library holds them until the
// process exits; all calls on one device share them.
static __device__ __align__(256) unsigned char g_design_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch[kMaxDevices] = {};  // device address of the array, per device

msosm_status fail(msosm_status st, const char *fmt, ...)
{
    char buf[320];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_error_message(buf);
    return st;
}

// Writes the twiddle tables and the chirp parameters.  Every byte of scratch
// that the design kernel reads is rewritten by each call, so nothing has to
// start at zero and nothing carries over from the previous call.
__global__ void fill_design_scratch(float2 *tw_m, int m, float2 *tw_n, int n, ChirpParams *cp, ChirpParams p)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)e / (double)n, &s, &c);
        tw_n[e] = make_float2((float)c, (float)-s);
        if (e < m) {
            sincospi(2.0 * (double)e / (double)m, &s, &c);
            tw_m[e] = make_float2((float)c, (float)s);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *cp = p;
}

}  // namespace

extern "C" MSOSM_API msosm_status msosm_prepare_dedisp_params_noalloc(float bw, float dm, float f0, unsigned long M,
                                                                      msosm_complex *H_device, void *stream)
{
    if (!H_device || !(bw > 0) || !(f0 > 0) || !(dm >= 0))
        return fail(MSOSM_ERR_BAD_ARG, "msosm_prepare_dedisp_params_noalloc: null output, or bw/f0 <= 0, or dm < 0");
    if (M < 32 || M > kNoAllocMaxM || (M & (M - 1)) != 0)
        return fail(MSOSM_ERR_BAD_ARG,
                    "msosm_prepare_dedisp_params_noalloc: M = %lu is not a power of two in 32..%lu "
                    "(FFT 64..%lu points); use msosm_prepare_dedisp_params for other sizes",
                    M, kNoAllocMaxM, 2 * kNoAllocMaxM);
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, H_device) != cudaSuccess ||
        (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        return fail(MSOSM_ERR_BAD_ARG, "msosm_prepare_dedisp_params_noalloc: H must point to device memory");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(MSOSM_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    // the design kernel runs on the current device and writes H there
    if (at.type == cudaMemoryTypeDevice && at.device != dev)
        return fail(MSOSM_ERR_BAD_ARG,
                    "msosm_prepare_dedisp_params_noalloc: H is memory of device %d, the current device is %d",
                    at.device, dev);
    if (dev < 0 || dev >= kMaxDevices)
        return fail(MSOSM_ERR_UNSUPPORTED, "device ordinal %d above %d", dev, kMaxDevices - 1);
    void *base = nullptr;
    {
        // Once per device, with that device current: the device address of
        // the array.  In host code the array's name is only a host-side
        // stand-in; kernels must be given this address.
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_design_scratch);
            if (e != cudaSuccess)
                return fail(MSOSM_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_scratch[dev] = p;
        }
        base = g_scratch[dev];
    }
    const unsigned long N = 2 * M;
    int log2n = 0;
    while ((1ul << log2n) < N)
        ++log2n;
    float2 *tw_m = static_cast<float2 *>(base);
    float2 *tw_n = tw_m + M;
    ChirpParams *cp = reinterpret_cast<ChirpParams *>(static_cast<unsigned char *>(base) + kTwiddleBytes);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fill_design_scratch<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(tw_m, (int)M, tw_n, (int)N, cp,
                                                                    chirp_params(bw, dm, f0, M));
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        DesignArgs a;
        a.chirp = cp;
        a.D = 1;
        a.tw_inv_m = tw_m;
        a.tw_fwd_n = tw_n;
        a.H = reinterpret_cast<float2 *>(H_device);
        a.scale = 1.0f;
        a.sign = -1;
        e = launch_design(log2n, a, st);
    }
    if (e != cudaSuccess)
        return fail(MSOSM_ERR_CUDA, "msosm_prepare_dedisp_params_noalloc: %s", cudaGetErrorString(e));
    return MSOSM_OK;
}
