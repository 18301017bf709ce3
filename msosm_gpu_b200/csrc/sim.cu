// sim.cu -- the signal simulator on the device (msosm_sim_* of msosm_b200.h).
//
// Random numbers: the counter-based generator Philox4x32-10 (Salmon, Moraes,
// Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC11, 2011).
// Sample i draws one block at counter (lo(i), hi(i), tag, 0) under the key
// (lo(seed), hi(seed)), so every sample's numbers are fixed by (seed, i, tag)
// whatever the launch shape or chunking, and a CPU implementation of the
// same arithmetic reproduces them.  The four words become two complex unit
// normals by the Box-Muller transform, evaluated in double precision and
// rounded to float.
//
// Two generators use them:
//  * the reference's SimulatedComplexSignal::generate_pulsar_signal
//    (simulated_pulsar/simulated_complex_signal.cpp:40-236): one period of two
//    unit deltas at Np/2 and Np/2 + 2 dispersed by the +phase chirp filter of
//    order 2^ceil(log2(range Np)) and summed over the `range` periods the
//    smear spans, tiled `repeat` times, plus AWGN at an SNR in dB relative to
//    the measured signal power (AWGN.cpp:20-46), and the uint16 codec of
//    :209-228.  The filter is applied by index arithmetic on the impulse
//    response (the circular convolution of deltas), its inverse DFT computed
//    by the library's chirp transform.
//  * a streaming Gaussian-profile pulsar: x(t) = disperse(a(t) z1(t)) + z2(t),
//    a(t) = sqrt(snr g(phase(t))), z1, z2 complex normals of variance 1/2 per
//    component, the dispersion run through the library's overlap-save path
//    with the +phase chirp filter (MSOSM_FLAG_OSM | MSOSM_FLAG_DISPERSE).
#include "msosm_b200.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "host_prepare.hpp"
#include "kernels.hpp"

using namespace msosm;

namespace {

constexpr unsigned kTagPulsar = 0, kTagAwgn = 1;

// ---------------------------------------------------------------------------
// device: generator
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

__device__ __forceinline__ uint4 block_at(unsigned long long seed, unsigned long long i, unsigned tag)
{
    return philox4x32_10(make_uint4((unsigned)i, (unsigned)(i >> 32), tag, 0u),
                         make_uint2((unsigned)seed, (unsigned)(seed >> 32)));
}

// u1 = (a + 1) 2^-32 in (0, 1], u2 = b 2^-32: (r cos, r sin)(2 pi u2),
// r = sqrt(-2 ln u1), in double, each rounded once to float
__device__ __forceinline__ float2 box_muller(unsigned a, unsigned b)
{
    const double u1 = __dmul_rn((double)a + 1.0, 0x1p-32);
    const double u2 = __dmul_rn((double)b, 0x1p-32);
    const double r = sqrt(__dmul_rn(-2.0, log(u1)));
    const double ang = __dmul_rn(2.0 * kPi, u2);
    double s, c;
    sincos(ang, &s, &c);
    return make_float2((float)__dmul_rn(r, c), (float)__dmul_rn(r, s));
}

__global__ void normals_kernel(unsigned long long seed, unsigned long long start, long long n, unsigned tag,
                               float2 *z1, float2 *z2)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    const uint4 w = block_at(seed, start + (unsigned long long)j, tag);
    if (z1)
        z1[j] = box_muller(w.x, w.y);
    if (z2)
        z2[j] = box_muller(w.z, w.w);
}

// ---------------------------------------------------------------------------
// device: the reference simulator (two deltas per period)
// ---------------------------------------------------------------------------

// period[j] = sum over i < range, p in {Np/2, Np/2 + 2} of hbuf[(j - i Np - p)
// mod 2 order], hbuf the zero buffer of 2 order points holding h (already / order)
// in its upper half (simulated_complex_signal.cpp:115-159)
__global__ void two_spike_period_kernel(const float2 *h, long long order, long long Np, long long range,
                                        float2 *period)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= Np)
        return;
    const long long F = 2 * order;
    double re = 0.0, im = 0.0;
    for (long long i = 0; i < range; ++i) {
        for (int q = 0; q < 2; ++q) {
            const long long p = i * Np + Np / 2 + 2 * q;
            long long n = (j - p) % F;
            if (n < 0)
                n += F;
            if (n >= order) {
                const float2 v = h[n - order];
                re += (double)v.x;
                im += (double)v.y;
            }
        }
    }
    period[j] = make_float2((float)re, (float)im);
}

// (v == 0) ? 0 : uint16(v * 32767 + 32768), float arithmetic, truncation,
// modulo 2^16 (simulated_complex_signal.cpp:213-214, 225-226)
__device__ __forceinline__ unsigned ref_u16(float v)
{
    if (v == 0.f)
        return 0u;
    const float f = __fadd_rn(__fmul_rn(v, 32767.f), 32768.f);
    return (unsigned)(int)truncf(f) & 0xFFFFu;
}

// signal[i] = period[i mod Np] (+ AWGN), and its uint16 pairs
// (simulated_complex_signal.cpp:203-230; the noise of AWGN.cpp:38-46)
__global__ void two_spike_tile_kernel(const float2 *period, long long Np, long long total, int add_noise,
                                      double noise_scale, unsigned long long seed, float2 *signal,
                                      unsigned *u16)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total)
        return;
    float2 v = period[i % Np];
    if (add_noise) {
        const uint4 w = block_at(seed, (unsigned long long)i, kTagAwgn);
        const float2 z = box_muller(w.x, w.y);
        v.x = __fadd_rn(v.x, (float)__dmul_rn(noise_scale, (double)z.x));
        v.y = __fadd_rn(v.y, (float)__dmul_rn(noise_scale, (double)z.y));
    }
    if (signal)
        signal[i] = v;
    if (u16)
        u16[i] = ref_u16(v.x) | (ref_u16(v.y) << 16);
}

// AWGN::generateNoiseSamples (AWGN.cpp:29-58): snr mode sigma/sqrt(2) z in
// double rounded to float; else normal_distribution(mean, variance): z *
// variance + mean in float (the reference passes the variance as the
// standard deviation)
__global__ void awgn_kernel(unsigned long long seed, long long n, int snr_mode, double snr_scale, float mean,
                            float stddev, float2 *out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint4 w = block_at(seed, (unsigned long long)i, kTagAwgn);
    const float2 z = box_muller(w.x, w.y);
    if (snr_mode)
        out[i] = make_float2((float)__dmul_rn(snr_scale, (double)z.x), (float)__dmul_rn(snr_scale, (double)z.y));
    else
        out[i] = make_float2(__fadd_rn(__fmul_rn(z.x, stddev), mean), __fadd_rn(__fmul_rn(z.y, stddev), mean));
}

// ---------------------------------------------------------------------------
// device: the Gaussian-profile pulsar
// ---------------------------------------------------------------------------

struct PulsarArgs {
    unsigned long long seed;
    double bw, period, sigma, centre, snr;
};

// a(t) = sqrt(snr exp(-(d / sigma)^2 / 2)), d the phase offset from the
// pulse centre wrapped to [-1/2, 1/2), phase = frac(t / bw / period)
__device__ __forceinline__ float amplitude(const PulsarArgs &a, unsigned long long t)
{
    double ph = __ddiv_rn(__ddiv_rn((double)t, a.bw), a.period);
    ph = __dadd_rn(ph, -floor(ph));
    double x = __dadd_rn(__dadd_rn(ph, -a.centre), 0.5);
    const double d = __dadd_rn(__dadd_rn(x, -floor(x)), -0.5);
    const double q = __ddiv_rn(d, a.sigma);
    const double g = exp(__dmul_rn(-0.5, __dmul_rn(q, q)));
    return (float)sqrt(__dmul_rn(a.snr, g));
}

constexpr float kInvSqrt2f = 0.70710678118654752f;

// e(t) = a(t) z1(t) / sqrt(2)
__global__ void emit_kernel(PulsarArgs a, unsigned long long t0, long long n, float2 *e)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    const unsigned long long t = t0 + (unsigned long long)j;
    const uint4 w = block_at(a.seed, t, kTagPulsar);
    const float2 z = box_muller(w.x, w.y);
    const float amp = amplitude(a, t);
    e[j] = make_float2(__fmul_rn(__fmul_rn(z.x, kInvSqrt2f), amp), __fmul_rn(__fmul_rn(z.y, kInvSqrt2f), amp));
}

// x(t) = gain y(t) + z2(t) / sqrt(2); optional offset-binary uint16 of
// rint(x scale) + 32768 clipped to [1, 65535] (0 is the blank value)
__global__ void finish_kernel(PulsarArgs a, unsigned long long t0, long long n, const float2 *y, float gain,
                              float2 *out, unsigned *u16, double qscale)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n)
        return;
    const unsigned long long t = t0 + (unsigned long long)j;
    const uint4 w = block_at(a.seed, t, kTagPulsar);
    const float2 z = box_muller(w.z, w.w);
    const float2 v = y[j];
    const float2 x = make_float2(__fadd_rn(__fmul_rn(gain, v.x), __fmul_rn(z.x, kInvSqrt2f)),
                                 __fadd_rn(__fmul_rn(gain, v.y), __fmul_rn(z.y, kInvSqrt2f)));
    if (out)
        out[j] = x;
    if (u16) {
        double qr = rint(__dmul_rn((double)x.x, qscale)) + 32768.0;
        double qi = rint(__dmul_rn((double)x.y, qscale)) + 32768.0;
        qr = fmin(fmax(qr, 1.0), 65535.0);
        qi = fmin(fmax(qi, 1.0), 65535.0);
        u16[j] = (unsigned)qr | ((unsigned)qi << 16);
    }
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

msosm_status sim_fail(msosm_status s, const char *msg)
{
    set_error_message(msg);
    return s;
}

msosm_status sim_cuda_fail(cudaError_t e, const char *what)
{
    cudaGetLastError();
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    set_error_message(buf);
    if (e == cudaErrorMemoryAllocation)
        return MSOSM_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return MSOSM_ERR_NO_DEVICE;
    return MSOSM_ERR_CUDA;
}

bool device_ptr(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Output destination: the caller's device buffer, or a device temporary
// copied to the caller's host buffer afterwards.
struct Out {
    void *user = nullptr, *dev = nullptr;
    size_t bytes = 0;
    bool own = false;
    cudaError_t init(void *p, size_t b)
    {
        user = p;
        bytes = b;
        if (!p)
            return cudaSuccess;
        if (device_ptr(p)) {
            dev = p;
            return cudaSuccess;
        }
        own = true;
        return cudaMalloc(&dev, b + 16);
    }
    cudaError_t finish(cudaStream_t st)
    {
        if (own && user)
            return cudaMemcpyAsync(user, dev, bytes, cudaMemcpyDeviceToHost, st);
        return cudaSuccess;
    }
    ~Out()
    {
        if (own && dev)
            cudaFree(dev);
    }
};

struct Stream {
    cudaStream_t s = nullptr;
    cudaError_t init() { return cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking); }
    ~Stream()
    {
        if (s)
            cudaStreamDestroy(s);
    }
};

int ceil_log2(unsigned long long v)
{
    int l = 0;
    while ((1ull << l) < v)
        ++l;
    return l;
}

// SimulatedComplexSignal's derived sizes (simulated_complex_signal.cpp:21-25,
// 52, 65-71); a smear shorter than one period still spans one period.
msosm_status two_spike_shape(float bw, float dm, float f0, float period, msosm_sim_two_spike_info *info)
{
    if (!(bw > 0) || !(f0 > 0) || !(dm >= 0) || !(period > 0) || !std::isfinite(dm))
        return sim_fail(MSOSM_ERR_BAD_ARG, "bw, f0, period must be > 0 and dm >= 0");
    const float fs = bw;
    info->Np = (unsigned long)(period * fs);
    info->Nd = dispersion_smear(bw, dm, f0);
    if (info->Np < 4)
        return sim_fail(MSOSM_ERR_BAD_ARG, "period shorter than 4 samples");
    unsigned long range = (unsigned long)std::ceil((float)info->Nd / (float)info->Np);
    if (range == 0)
        range = 1;
    info->range = range;
    info->order = 1ul << ceil_log2((unsigned long long)range * info->Np);
    return MSOSM_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

struct msosm_sim {
    PulsarArgs args{};
    msosm_sim_pulsar_params params{};
    msosm_dedisp *osm = nullptr;  // null at DM 0 (no dispersion)
    unsigned long chunk = 0, M = 0, Nd = 0;
    unsigned long long t0 = 0;
    cudaStream_t stream = nullptr;
    float2 *e = nullptr, *x = nullptr;
    unsigned *u16 = nullptr;
};

extern "C" {

msosm_status msosm_host_alloc(size_t bytes, int pinned, void **out)
{
    if (!out)
        return sim_fail(MSOSM_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    if (pinned) {
        cudaError_t e = cudaMallocHost(out, bytes ? bytes : 1);
        if (e != cudaSuccess) {
            *out = nullptr;
            return sim_cuda_fail(e, "cudaMallocHost");
        }
        return MSOSM_OK;
    }
    *out = std::malloc(bytes ? bytes : 1);
    return *out ? MSOSM_OK : sim_fail(MSOSM_ERR_OOM, "host allocation");
}

msosm_status msosm_host_free(void *p, int pinned)
{
    if (!p)
        return MSOSM_OK;
    if (pinned) {
        cudaError_t e = cudaFreeHost(p);
        return e == cudaSuccess ? MSOSM_OK : sim_cuda_fail(e, "cudaFreeHost");
    }
    std::free(p);
    return MSOSM_OK;
}

msosm_status msosm_sim_normals(unsigned long long seed, unsigned long long start, unsigned long n, unsigned tag,
                               msosm_complex *z1, msosm_complex *z2)
{
    if (!z1 && !z2)
        return sim_fail(MSOSM_ERR_BAD_ARG, "both outputs null");
    if (n == 0)
        return MSOSM_OK;
    Stream st;
    Out o1, o2;
    cudaError_t e = st.init();
    if (e == cudaSuccess)
        e = o1.init(z1, sizeof(float2) * n);
    if (e == cudaSuccess)
        e = o2.init(z2, sizeof(float2) * n);
    if (e == cudaSuccess) {
        normals_kernel<<<nblk((long long)n, 256), 256, 0, st.s>>>(seed, start, (long long)n, tag, (float2 *)o1.dev,
                                                                  (float2 *)o2.dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = o1.finish(st.s);
    if (e == cudaSuccess)
        e = o2.finish(st.s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st.s);
    return e == cudaSuccess ? MSOSM_OK : sim_cuda_fail(e, "msosm_sim_normals");
}

msosm_status msosm_sim_awgn(unsigned long long seed, unsigned long n, int snr_mode, float mean, float variance,
                            float snr_db, msosm_complex *out)
{
    if (!out)
        return sim_fail(MSOSM_ERR_BAD_ARG, "null output");
    if (n == 0)
        return MSOSM_OK;
    // AWGN.cpp:20-26, 43-44: sigma = sqrt(10^(-SNR/10)) stored in float,
    // then sigma / sqrt(2) in double
    const float sigma = (float)std::sqrt(std::pow(10.0, (double)(-snr_db / 10.0f)));
    const double scale = (double)sigma / std::sqrt(2.0);
    Stream st;
    Out o;
    cudaError_t e = st.init();
    if (e == cudaSuccess)
        e = o.init(out, sizeof(float2) * n);
    if (e == cudaSuccess) {
        awgn_kernel<<<nblk((long long)n, 256), 256, 0, st.s>>>(seed, (long long)n, snr_mode, scale, mean, variance,
                                                               (float2 *)o.dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = o.finish(st.s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st.s);
    return e == cudaSuccess ? MSOSM_OK : sim_cuda_fail(e, "msosm_sim_awgn");
}

msosm_status msosm_sim_two_spike_shape(float bw, float dm, float f0, float period, msosm_sim_two_spike_info *info)
{
    if (!info)
        return sim_fail(MSOSM_ERR_BAD_ARG, "null argument");
    return two_spike_shape(bw, dm, f0, period, info);
}

msosm_status msosm_sim_two_spike(float bw, float dm, float f0, float period, unsigned long repeat, int add_noise,
                                 float snr_db, unsigned long long seed, msosm_complex *signal,
                                 msosm_uint16_pair *signal_u16, float *signal_power_db)
{
    msosm_sim_two_spike_info info{};
    msosm_status s = two_spike_shape(bw, dm, f0, period, &info);
    if (s != MSOSM_OK)
        return s;
    if (repeat < 1)
        return sim_fail(MSOSM_ERR_BAD_ARG, "repeat must be >= 1");
    const int log2o = ceil_log2(info.order);
    ChirpIdft idft;
    Stream st;
    cudaError_t e = st.init();
    if (e != cudaSuccess)
        return sim_cuda_fail(e, "stream");
    if ((s = idft.init(log2o, st.s)) != MSOSM_OK)
        return s;
    const unsigned long long total = (unsigned long long)repeat * info.Np;
    float2 *h = nullptr, *per = nullptr;
    Out osig, ou16;
    e = cudaMalloc((void **)&h, sizeof(float2) * info.order);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&per, sizeof(float2) * info.Np);
    if (e == cudaSuccess)
        e = osig.init(signal, sizeof(float2) * total);
    if (e == cudaSuccess)
        e = ou16.init(signal_u16, sizeof(unsigned) * total);
    // h = IDFT_order(+chirp) / order (simulated_complex_signal.cpp:91-113)
    if (e == cudaSuccess)
        e = idft.run(chirp_params(bw, dm, f0, info.order), +1, h, (long long)info.order, st.s);
    if (e == cudaSuccess)
        e = launch_conj_scale(h, (long long)info.order, 1.0f / (float)info.order, 0, st.s);
    if (e == cudaSuccess) {
        two_spike_period_kernel<<<nblk((long long)info.Np, 256), 256, 0, st.s>>>(
            h, (long long)info.order, (long long)info.Np, (long long)info.range, per);
        e = cudaGetLastError();
    }
    // measured power of one period, accumulated in float as :169-174
    std::vector<float2> hp(info.Np);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hp.data(), per, sizeof(float2) * info.Np, cudaMemcpyDeviceToHost, st.s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st.s);
    float power = 0.f;
    if (e == cudaSuccess) {
        for (unsigned long i = 0; i < info.Np; ++i)
            power = power + hp[i].x * hp[i].x + hp[i].y * hp[i].y;
        power = 10 * std::log10(power / (float)info.Np);
        if (signal_power_db)
            *signal_power_db = power;
    }
    if (e == cudaSuccess && (osig.dev || ou16.dev)) {
        // AWGN g(SNR - power): sigma = sqrt(10^(-(SNR - power)/10))
        const float sigma = (float)std::sqrt(std::pow(10.0, (double)(-(snr_db - power) / 10.0f)));
        const double scale = (double)sigma / std::sqrt(2.0);
        two_spike_tile_kernel<<<nblk((long long)total, 256), 256, 0, st.s>>>(
            per, (long long)info.Np, (long long)total, add_noise, scale, seed, (float2 *)osig.dev,
            (unsigned *)ou16.dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = osig.finish(st.s);
    if (e == cudaSuccess)
        e = ou16.finish(st.s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st.s);
    idft.release();
    if (h)
        cudaFree(h);
    if (per)
        cudaFree(per);
    return e == cudaSuccess ? MSOSM_OK : sim_cuda_fail(e, "msosm_sim_two_spike");
}

msosm_status msosm_sim_pulsar_destroy(msosm_sim *s)
{
    if (!s)
        return MSOSM_OK;
    if (s->stream)
        cudaStreamSynchronize(s->stream);
    if (s->osm)
        msosm_dedisp_destroy(s->osm);
    void *bufs[] = {s->e, s->x, s->u16};
    for (void *b : bufs)
        if (b)
            cudaFree(b);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    delete s;
    return MSOSM_OK;
}

msosm_status msosm_sim_pulsar_create(const msosm_sim_pulsar_params *p, unsigned long min_chunk, msosm_sim **out)
{
    if (!p || !out)
        return sim_fail(MSOSM_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    if (!(p->bw > 0) || !(p->f0 > 0) || !(p->dm >= 0) || !std::isfinite(p->dm) || !(p->period > 0) ||
        !(p->fwhm > 0) || !(p->snr >= 0) || !std::isfinite(p->centre))
        return sim_fail(MSOSM_ERR_BAD_ARG, "bw, f0, period, fwhm must be > 0; dm, snr >= 0");
    msosm_sim *s = new (std::nothrow) msosm_sim;
    if (!s)
        return sim_fail(MSOSM_ERR_OOM, "host allocation");
    s->params = *p;
    s->args.seed = p->seed;
    s->args.bw = (double)p->bw;
    s->args.period = p->period;
    s->args.sigma = p->fwhm / (2.0 * std::sqrt(2.0 * std::log(2.0)));
    s->args.centre = p->centre;
    s->args.snr = p->snr;
    s->Nd = dispersion_smear(p->bw, p->dm, p->f0);
    if (min_chunk == 0)
        min_chunk = 1ul << 22;
    msosm_status st = MSOSM_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        msosm_sim_pulsar_destroy(s);
        return sim_cuda_fail(e, "stream");
    }
    if (s->Nd > 0) {
        s->M = osm_min_order(s->Nd);
        const unsigned long count = (min_chunk + s->M - 1) / s->M;
        s->chunk = count * s->M;
        const float bw = p->bw, dm = p->dm, f0 = p->f0;
        st = msosm_dedisp_create(&bw, &dm, &f0, 1, 0, (int)count, 0, MSOSM_FLAG_OSM | MSOSM_FLAG_DISPERSE, &s->osm);
        if (st == MSOSM_OK)
            st = msosm_dedisp_set_stream(s->osm, s->stream);
    } else {
        s->M = 0;
        s->chunk = min_chunk;
    }
    if (st == MSOSM_OK) {
        e = cudaMalloc((void **)&s->e, sizeof(float2) * s->chunk + 16);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&s->x, sizeof(float2) * s->chunk + 16);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&s->u16, sizeof(unsigned) * s->chunk + 16);
        if (e != cudaSuccess)
            st = sim_cuda_fail(e, "simulator buffers");
    }
    if (st != MSOSM_OK) {
        msosm_sim_pulsar_destroy(s);
        return st;
    }
    *out = s;
    return MSOSM_OK;
}

msosm_status msosm_sim_pulsar_get_info(const msosm_sim *s, msosm_sim_pulsar_info *info)
{
    if (!s || !info)
        return sim_fail(MSOSM_ERR_BAD_ARG, "null argument");
    info->chunk = s->chunk;
    info->M = s->M;
    info->Nd = s->Nd;
    info->next_sample = s->t0;
    return MSOSM_OK;
}

msosm_status msosm_sim_pulsar_next(msosm_sim *s, msosm_complex *out, msosm_uint16_pair *u16, double u16_scale)
{
    if (!s)
        return sim_fail(MSOSM_ERR_BAD_ARG, "null handle");
    if (!out && !u16)
        return sim_fail(MSOSM_ERR_BAD_ARG, "both outputs null");
    const long long n = (long long)s->chunk;
    cudaError_t e = cudaSuccess;
    msosm_status st = MSOSM_OK;
    const float2 *y = s->e;
    float gain = 1.f;
    emit_kernel<<<nblk(n, 256), 256, 0, s->stream>>>(s->args, s->t0, n, s->e);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return sim_cuda_fail(e, "emit");
    if (s->osm) {
        // the overlap-save output is half the dispersed emission
        if ((st = msosm_dedisp_filter_block_c64(s->osm, (const msosm_complex *)s->e)) != MSOSM_OK)
            return st;
        msosm_complex *yp = nullptr;
        if ((st = msosm_dedisp_output_device_ptr(s->osm, &yp)) != MSOSM_OK)
            return st;
        y = (const float2 *)yp;
        gain = 2.f;
    }
    const bool out_dev = out && device_ptr(out), u16_dev = u16 && device_ptr(u16);
    float2 *xo = out ? (out_dev ? (float2 *)out : s->x) : nullptr;
    unsigned *uo = u16 ? (u16_dev ? (unsigned *)u16 : s->u16) : nullptr;
    finish_kernel<<<nblk(n, 256), 256, 0, s->stream>>>(s->args, s->t0, n, y, gain, xo, uo, u16_scale);
    e = cudaGetLastError();
    if (e == cudaSuccess && out && !out_dev)
        e = cudaMemcpyAsync(out, s->x, sizeof(float2) * n, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && u16 && !u16_dev)
        e = cudaMemcpyAsync(u16, s->u16, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess)
        return sim_cuda_fail(e, "msosm_sim_pulsar_next");
    s->t0 += (unsigned long long)n;
    return MSOSM_OK;
}

}  // extern "C"
