// api.cu -- the C ABI (include/msosm_b200.h) over the sm_100a kernels.
#include "msosm_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "host_prepare.hpp"
#include "kernels.hpp"
#include "tc_layout.hpp"

using namespace msosm;

namespace {

thread_local std::string g_err;

msosm_status fail(msosm_status s, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

msosm_status cuda_fail(cudaError_t e, const char *what)
{
    cudaGetLastError();  // clear a non-sticky error
    if (e == cudaErrorMemoryAllocation)
        return fail(MSOSM_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return fail(MSOSM_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return fail(MSOSM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return cuda_fail(e_, #call);                                                               \
    } while (0)

int ilog2_exact(unsigned long n)
{
    if (n == 0 || (n & (n - 1)) != 0)
        return -1;
    int l = 0;
    while ((1ul << l) < n)
        ++l;
    return l;
}

bool is_device_ptr(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// exp(sign * 2 pi i e / n), e < n, computed in double on the host
std::vector<float2> twiddle_table(int n, int sign)
{
    std::vector<float2> t(n);
    for (int e = 0; e < n; ++e) {
        const double a = sign * 2.0 * kPi * (double)e / (double)n;
        t[e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    return t;
}

template <typename T>
cudaError_t dalloc(T **p, size_t count, size_t &total)
{
    total += count * sizeof(T);
    return cudaMalloc((void **)p, count * sizeof(T) + 16);
}

// The tensor-core kernel's limit on each wait for one of its GEMMs (which
// take microseconds): 1 s of global timer.
constexpr long long kTcWaitLimitDefaultNs = 1000000000ll;

}  // namespace

namespace msosm {
void set_error_message(const char *msg) { g_err = msg; }
}  // namespace msosm

struct msosm_dedisp {
    // configuration
    int D = 0, count = 0, log2n = 0, S = 0, R = 1, grid = 1, max_dc = 0, max_delay = 0;
    unsigned long M = 0, N = 0, M_min = 0;
    unsigned int flags = 0;
    bool series = true;
    bool pingpong = false;  // tuning: MSOSM_DEDISP_PINGPONG=1 selects the two-buffer kernel
    std::vector<unsigned long> Nd;
    std::vector<int> dc;
    std::vector<int> delays;  // D x N (host copy)
    unsigned long long calls = 0;
    size_t device_bytes = 0;
    // streams and events
    cudaStream_t stream = nullptr, own_stream = nullptr, copy_stream = nullptr;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_consumed[2] = {nullptr, nullptr};
    cudaEvent_t ev_spans[2] = {nullptr, nullptr};
    // device buffers
    float2 *ring = nullptr, *H = nullptr, *hist = nullptr, *series_buf = nullptr;
    uint16_t *delays_d = nullptr;
    float2 *tw_fwd = nullptr, *tw_inv = nullptr, *tw_inv_m = nullptr;
    void *staging[2] = {nullptr, nullptr};
    uint32_t *u16_out = nullptr;
    // folding
    bool fold = false;
    int detect = 0, nbins = 0, bpt = 1, span_cap = 0, win_cap = 64;
    unsigned long ps = 0;
    double out_scale = 1.0;
    FoldPlanner *planner = nullptr;
    std::vector<FoldSpan> spans;
    float *part_main = nullptr, *part_pend = nullptr, *prof_out = nullptr;
    double *acc_main = nullptr, *acc_pend = nullptr;
    long long *span_a_d = nullptr, *span_b_d = nullptr;
    int *span_p_d = nullptr, *span_dest_d = nullptr;
    // pinned span staging: [2][cap] of a, b, phase0, dest
    long long *span_host = nullptr;
    // inverse transforms on the tensor cores (MSOSM_FLAG_TENSOR_F16): ring,
    // H and delays in tensor-core order (tc_layout.hpp); status_d != 0 after
    // a timed-out wait in the kernel
    bool tc = false, tc_bf16 = false;
    int *status_d = nullptr;
    long long tc_wait_limit_ns = kTcWaitLimitDefaultNs;  // each wait of the kernel on a GEMM
    float *row_max = nullptr;  // [S] largest |component| of each ring row
    float *h_max = nullptr;    // [D] largest |component| of each trial's H
    int *delay_max_d = nullptr; // [D] largest block delay of each trial
    // FFT above one thread block: four-step N = N1*N2, spectra in [k1][k2] order
    bool large = false;
    int log2n1 = 0, log2n2 = 0;
    float2 *lA = nullptr, *lB = nullptr;         // column-pass and row-pass scratch
    float *lI = nullptr;                         // intensities for folding
    float2 *tw1f = nullptr, *tw1i = nullptr, *tw2f = nullptr, *tw2i = nullptr;
    // timing: events per timed call: e0 [forward] e1 [fold prep] e2 [dedisp] e3
    // [fold reduce] e6; e4 [h2d] e5 on the copy stream
    bool timing = false;
    struct CallEvents {
        cudaEvent_t e[7];
        bool h2d;
    };
    std::vector<CallEvents> timed;
    unsigned long long launches = 0, timed_launches = 0;
};

namespace {

void release(msosm_dedisp *d)
{
    if (!d)
        return;
    if (d->stream)
        cudaStreamSynchronize(d->stream);
    if (d->copy_stream)
        cudaStreamSynchronize(d->copy_stream);
    void *bufs[] = {d->ring, d->H, d->hist, d->series_buf, d->delays_d, d->tw_fwd, d->tw_inv, d->tw_inv_m,
                    d->staging[0], d->staging[1], d->u16_out, d->part_main, d->part_pend, d->prof_out,
                    d->acc_main, d->acc_pend, d->span_a_d, d->span_b_d, d->span_p_d, d->span_dest_d,
                    d->lA, d->lB, d->lI, d->tw1f, d->tw1i, d->tw2f, d->tw2i, d->status_d,
                    d->row_max, d->h_max, d->delay_max_d};
    for (void *p : bufs)
        if (p)
            cudaFree(p);
    if (d->span_host)
        cudaFreeHost(d->span_host);
    for (int i = 0; i < 2; ++i) {
        if (d->ev_copied[i])
            cudaEventDestroy(d->ev_copied[i]);
        if (d->ev_consumed[i])
            cudaEventDestroy(d->ev_consumed[i]);
        if (d->ev_spans[i])
            cudaEventDestroy(d->ev_spans[i]);
    }
    for (auto &c : d->timed)
        for (cudaEvent_t e : c.e)
            cudaEventDestroy(e);
    if (d->copy_stream)
        cudaStreamDestroy(d->copy_stream);
    if (d->own_stream)
        cudaStreamDestroy(d->own_stream);
    delete d->planner;
    delete d;
}

msosm_status upload_table(float2 **dst, int n, int sign, size_t &total, cudaStream_t st)
{
    std::vector<float2> t = twiddle_table(n, sign);
    CK(dalloc(dst, (size_t)n, total));
    CK(cudaMemcpyAsync(*dst, t.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return MSOSM_OK;
}

// H of every trial on the device: H_ref * scale into H[D][N]
msosm_status design_filters(int log2n, const std::vector<ChirpParams> &cp, float scale, int sign,
                            const float2 *tw_inv_m, const float2 *tw_fwd, float2 *H, cudaStream_t st)
{
    ChirpParams *cp_d = nullptr;
    CK(cudaMalloc((void **)&cp_d, sizeof(ChirpParams) * cp.size()));
    cudaError_t e = cudaMemcpyAsync(cp_d, cp.data(), sizeof(ChirpParams) * cp.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        DesignArgs a;
        a.chirp = cp_d;
        a.D = (int)cp.size();
        a.tw_inv_m = tw_inv_m;
        a.tw_fwd_n = tw_fwd;
        a.H = H;
        a.scale = scale;
        a.sign = sign;
        e = launch_design(log2n, a, st);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaFree(cp_d);
    if (e != cudaSuccess)
        return cuda_fail(e, "filter design");
    return MSOSM_OK;
}

// Whether the fused kernel keeps a work item's two profiles in shared memory
// (else in the global partial rows): up to kMaxSmemBins bins, and in the
// tensor-core kernels only when they fit beside the tables, operand buffers
// and span window in the device's per-block limit (at 8192 points that is
// 1024 bins with the usual 64-span window; at 16384, 2048).
bool prof_in_smem(const msosm_dedisp *d)
{
    if (d->nbins > kMaxSmemBins)
        return false;
    if (!d->tc)
        return true;
    const size_t need = tc_smem_base(d->log2n) + fold_smem_bytes(d->nbins, d->win_cap, true, tc_threads(d->log2n));
    return need <= tc_smem_limit();
}

// Persistent grid of the dedispersion kernel: work items (block range,
// trial), about eight per resident CTA, spread evenly over the waves.
cudaError_t plan_grid(msosm_dedisp *d)
{
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
        return e;
    const int threads = d->tc ? tc_threads(d->log2n) : (int)(d->N / 16);
    const size_t extra = d->fold ? fold_smem_bytes(d->nbins, d->win_cap, prof_in_smem(d), threads) : 0;
    int per_sm = d->tc ? tc_blocks_per_sm(d->log2n, d->tc_bf16, d->series, d->fold, extra)
                       : dedisp_blocks_per_sm(d->log2n, d->pingpong, d->series, d->fold, extra);
    if (per_sm < 1)
        per_sm = 1;
    const long long resident = (long long)per_sm * sms;
    long long R = (8 * resident + d->D - 1) / d->D;
    // the tensor-core kernel works in steps of a pair of blocks (one block at 16384)
    const int bps = d->tc ? tc_blocks_per_step(d->log2n) : 1;
    const long long units = (d->count + bps - 1) / bps;
    if (R > units)
        R = units;
    if (R < 1)
        R = 1;
    d->R = (int)R;
    const long long items = (long long)d->D * R;
    const long long waves = (items + resident - 1) / resident;
    d->grid = (int)((items + waves - 1) / waves);
    if (std::getenv("MSOSM_DEBUG_GRID"))
        std::fprintf(stderr, "msosm plan_grid: tc=%d fold=%d series=%d extra=%zu per_sm=%d R=%d grid=%d\n",
                     (int)d->tc, (int)d->fold, (int)d->series, extra, per_sm, d->R, d->grid);
    return cudaSuccess;
}

}  // namespace

// ---------------------------------------------------------------------------
// Inverse M-point DFT of the reference chirp on the device (filter design and
// the signal simulator)
// ---------------------------------------------------------------------------

namespace msosm {

int ChirpIdft::init(int log2m_, cudaStream_t st)
{
    log2m = log2m_;
    large = log2m > kMaxLog2N;
    if (log2m < kMinLog2N || (large && !large_supported(log2m)))
        return fail(MSOSM_ERR_UNSUPPORTED, "chirp transform of 2^%d points outside 2^%d .. 2^24", log2m, kMinLog2N);
    const long long M = 1ll << log2m;
    size_t tot = 0;
    cudaError_t e = cudaMalloc((void **)&cp_d, sizeof(ChirpParams));
    if (e == cudaSuccess)
        e = dalloc(&V, (size_t)M, tot);
    if (e == cudaSuccess)
        e = dalloc(&W, (size_t)M, tot);
    if (e == cudaSuccess && large)
        e = dalloc(&A, (size_t)M, tot);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "chirp transform scratch");
    }
    msosm_status s;
    if (large) {
        large_split(log2m, m1l, m2l);
        s = upload_table(&tw1, 1 << m1l, -1, tot, st);
        if (s == MSOSM_OK)
            s = upload_table(&tw2, 1 << m2l, -1, tot, st);
    } else {
        s = upload_table(&tw1, 1 << log2m, -1, tot, st);
    }
    if (s != MSOSM_OK)
        release();
    return s;
}

// conj(chirp) -> FFT_M -> un-permute + conj: the unnormalised inverse DFT
cudaError_t ChirpIdft::run(const ChirpParams &cp, int sign, float2 *P, long long len_out, cudaStream_t st)
{
    const long long M = 1ll << log2m;
    cudaError_t e = cudaMemcpyAsync(cp_d, &cp, sizeof(ChirpParams), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_chirp_conj(cp_d, V, M, sign, st);
    if (e != cudaSuccess)
        return e;
    if (!large) {
        e = launch_vec_fft(log2m, -1, V, W, tw1, 1, st);
        if (e == cudaSuccess)
            e = launch_unpermute_conj(W, P, M, 1, M, len_out, st);
        return e;
    }
    LargeColArgs ca{};
    ca.input = V;
    ca.out = A;
    ca.N = M;
    ca.N2 = 1ll << m2l;
    ca.len = M;
    ca.log2n = log2m;
    ca.count = 1;
    ca.tw1 = tw1;
    e = launch_large_col_fwd(m1l, 2, ca, 1, st);
    if (e == cudaSuccess) {
        LargeRowArgs ra{};
        ra.in = A;
        ra.out = W;
        ra.N = M;
        ra.log2n = log2m;
        ra.tw2 = tw2;
        ra.count = 1;
        e = launch_large_row(m2l, 2, ra, 1 << m1l, 1, 1, st);
    }
    if (e == cudaSuccess)
        e = launch_unpermute_conj(W, P, M, 1ll << m1l, 1ll << m2l, len_out, st);
    return e;
}

void ChirpIdft::release()
{
    void *bufs[] = {cp_d, V, W, A, tw1, tw2};
    for (void *b : bufs)
        if (b)
            cudaFree(b);
    cp_d = nullptr;
    V = W = A = tw1 = tw2 = nullptr;
}

}  // namespace msosm

namespace {

// H of every trial for N above one thread block, in the permuted [k1][k2]
// order of the four-step spectra, scaled by `scale`:
//   the unnormalised inverse M-point DFT of the chirp (the reference's h)
//   -> zero pad to N -> FFT_N (permuted) -> x scale.
msosm_status design_filters_large(int log2n, const std::vector<ChirpParams> &cp, float scale, int sign, float2 *Hp,
                                  cudaStream_t st)
{
    const long long N = 1ll << log2n;
    int n1l, n2l;
    large_split(log2n, n1l, n2l);
    size_t tot = 0;
    ChirpIdft idft;
    float2 *P = nullptr, *A = nullptr, *twn1 = nullptr, *twn2 = nullptr;
    msosm_status s = idft.init(log2n - 1, st);
    cudaError_t e = cudaSuccess;
    if (s == MSOSM_OK) {
        e = dalloc(&P, (size_t)N, tot);
        if (e == cudaSuccess)
            e = dalloc(&A, (size_t)N, tot);
        if (e != cudaSuccess)
            s = cuda_fail(e, "design scratch");
    }
    if (s == MSOSM_OK)
        s = upload_table(&twn1, 1 << n1l, -1, tot, st);
    if (s == MSOSM_OK)
        s = upload_table(&twn2, 1 << n2l, -1, tot, st);
    if (s == MSOSM_OK) {
        for (size_t i = 0; i < cp.size() && e == cudaSuccess; ++i) {
            e = idft.run(cp[i], sign, P, N, st);
            if (e == cudaSuccess) {
                LargeColArgs ca{};
                ca.input = P;
                ca.out = A;
                ca.N = N;
                ca.N2 = 1ll << n2l;
                ca.len = N;
                ca.log2n = log2n;
                ca.count = 1;
                ca.tw1 = twn1;
                e = launch_large_col_fwd(n1l, 2, ca, 1, st);
            }
            if (e == cudaSuccess) {
                LargeRowArgs ra{};
                ra.in = A;
                ra.out = Hp + i * (size_t)N;
                ra.N = N;
                ra.log2n = log2n;
                ra.tw2 = twn2;
                ra.count = 1;
                e = launch_large_row(n2l, 2, ra, 1 << n1l, 1, 1, st);
            }
            if (e == cudaSuccess)
                e = launch_conj_scale(Hp + i * (size_t)N, N, scale, 0, st);
        }
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            s = cuda_fail(e, "large filter design");
    }
    idft.release();
    void *bufs[] = {P, A, twn1, twn2};
    for (void *b : bufs)
        if (b)
            cudaFree(b);
    return s;
}

}  // namespace

namespace msosm {
cudaStream_t dedisp_stream(const msosm_dedisp *d) { return d->stream; }
}  // namespace msosm

namespace {

msosm_status check_handle(const msosm_dedisp *d)
{
    if (!d)
        return fail(MSOSM_ERR_BAD_ARG, "null handle");
    return MSOSM_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char *msosm_last_error(void) { return g_err.c_str(); }
int msosm_version(void) { return 100; }

int msosm_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

msosm_status msosm_prepare_nd(float bw, float dm, float f0, unsigned long *Nd)
{
    if (!Nd || !(bw > 0) || !(f0 > 0))
        return fail(MSOSM_ERR_BAD_ARG, "msosm_prepare_nd: bw and f0 must be positive");
    *Nd = dispersion_smear(bw, dm, f0);
    return MSOSM_OK;
}

msosm_status msosm_prepare_min_order_msosm(unsigned long Nd, unsigned long *M_min)
{
    if (!M_min)
        return fail(MSOSM_ERR_BAD_ARG, "null output");
    *M_min = msosm_min_order(Nd);
    return MSOSM_OK;
}

msosm_status msosm_prepare_min_order_osm(unsigned long Nd, unsigned long *M_min)
{
    if (!M_min)
        return fail(MSOSM_ERR_BAD_ARG, "null output");
    *M_min = osm_min_order(Nd);
    return MSOSM_OK;
}

msosm_status msosm_prepare_segmentation(float bw, float dm, float f0, unsigned long M, int *delaycount,
                                        int *delay_points)
{
    if (!delaycount || !delay_points || M == 0 || !(bw > 0) || !(f0 > 0))
        return fail(MSOSM_ERR_BAD_ARG, "msosm_prepare_segmentation: bad arguments");
    *delaycount = segment_delays(bw, dm, f0, dispersion_smear(bw, dm, f0), M, delay_points);
    return MSOSM_OK;
}

msosm_status msosm_prepare_dedisp_params(float bw, float dm, float f0, unsigned long M, msosm_complex *H)
{
    if (!H || !(bw > 0) || !(f0 > 0) || !(dm >= 0))
        return fail(MSOSM_ERR_BAD_ARG, "msosm_prepare_dedisp_params: null output, or bw/f0 <= 0, or dm < 0");
    const int log2n = ilog2_exact(2 * M);
    if (log2n < 0)
        return fail(MSOSM_ERR_BAD_ARG, "M must be a power of two");
    if (!log2n_supported(log2n))
        return fail(MSOSM_ERR_UNSUPPORTED, "FFT size %lu outside 64..16384", 2 * M);
    if (msosm_device_count() == 0)
        return fail(MSOSM_ERR_NO_DEVICE, "no CUDA device");
    size_t total = 0;
    cudaStream_t st = nullptr;
    float2 *tw_m = nullptr, *tw_n = nullptr, *Hd = nullptr;
    msosm_status s = MSOSM_OK;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if ((s = upload_table(&tw_m, (int)M, +1, total, st)) == MSOSM_OK &&
        (s = upload_table(&tw_n, (int)(2 * M), -1, total, st)) == MSOSM_OK) {
        cudaError_t e = cudaMalloc((void **)&Hd, sizeof(float2) * 2 * M);
        if (e != cudaSuccess) {
            s = cuda_fail(e, "cudaMalloc");
        } else {
            std::vector<ChirpParams> cp(1, chirp_params(bw, dm, f0, M));
            s = design_filters(log2n, cp, 1.0f, -1, tw_m, tw_n, Hd, st);
            if (s == MSOSM_OK) {
                e = cudaMemcpy(H, Hd, sizeof(float2) * 2 * M, cudaMemcpyDeviceToHost);
                if (e != cudaSuccess)
                    s = cuda_fail(e, "cudaMemcpy");
            }
        }
    }
    cudaFree(Hd);
    cudaFree(tw_m);
    cudaFree(tw_n);
    cudaStreamDestroy(st);
    return s;
}

msosm_status msosm_dedisp_create(const float *bw, const float *dm, const float *f0, int numDMs,
                                 unsigned long fftpoint, int count, unsigned long input_size,
                                 unsigned int flags, msosm_dedisp **out)
{
    if (!out || !bw || !dm || !f0 || numDMs < 1)
        return fail(MSOSM_ERR_BAD_ARG, "msosm_dedisp_create: null argument or numDMs < 1");
    *out = nullptr;
    if (flags & ~(MSOSM_FLAG_OSM | MSOSM_FLAG_NO_SERIES | MSOSM_FLAG_TENSOR_F16 | MSOSM_FLAG_TENSOR_BF16 |
                  MSOSM_FLAG_DISPERSE))
        return fail(MSOSM_ERR_BAD_ARG, "unknown flags 0x%x", flags);
    // the per-bin block delays of MS-OSM follow the dedispersion chirp
    if ((flags & MSOSM_FLAG_DISPERSE) && !(flags & MSOSM_FLAG_OSM))
        return fail(MSOSM_ERR_BAD_ARG, "MSOSM_FLAG_DISPERSE needs MSOSM_FLAG_OSM");
    for (int i = 0; i < numDMs; ++i)
        if (!(bw[i] > 0) || !(f0[i] > 0) || !(dm[i] >= 0) || !std::isfinite(dm[i]))
            return fail(MSOSM_ERR_BAD_ARG, "trial %d: bw, f0 must be > 0 and dm >= 0", i);
    const bool osm = (flags & MSOSM_FLAG_OSM) != 0;
    msosm_dedisp *d = new (std::nothrow) msosm_dedisp;
    if (!d)
        return fail(MSOSM_ERR_OOM, "host allocation");
    d->D = numDMs;
    d->flags = flags;
    d->series = (flags & MSOSM_FLAG_NO_SERIES) == 0;
    d->Nd.resize(numDMs);
    d->dc.assign(numDMs, 0);
    // minimum orders, common order (msosm_prepare_dm_concurrent.cpp:31-49,
    // msosm_gpu_dm_concurrent.cpp:29-42)
    unsigned long Mc = 0;
    for (int i = 0; i < numDMs; ++i) {
        d->Nd[i] = dispersion_smear(bw[i], dm[i], f0[i]);
        const unsigned long m = osm ? osm_min_order(d->Nd[i]) : msosm_min_order(d->Nd[i]);
        Mc = m > Mc ? m : Mc;
    }
    d->M_min = Mc;
    unsigned long M = Mc;
    if (fftpoint != 0) {
        M = fftpoint / 2;
        if (M < Mc)
            M = Mc;  // the reference warns and raises the FFT to the minimum
    }
    const int log2n = ilog2_exact(2 * M);
    if (log2n < 0) {
        release(d);
        return fail(MSOSM_ERR_BAD_ARG, "FFT size %lu is not a power of two", 2 * M);
    }
    if (!log2n_supported(log2n) && !large_supported(log2n)) {
        release(d);
        return fail(MSOSM_ERR_UNSUPPORTED, "FFT size %lu outside the supported 64..2^24", 2 * M);
    }
    d->large = !log2n_supported(log2n);
    d->tc = (flags & (MSOSM_FLAG_TENSOR_F16 | MSOSM_FLAG_TENSOR_BF16)) != 0;
    d->tc_bf16 = (flags & MSOSM_FLAG_TENSOR_BF16) != 0;
    if ((flags & MSOSM_FLAG_TENSOR_F16) && d->tc_bf16) {
        release(d);
        return fail(MSOSM_ERR_BAD_ARG, "MSOSM_FLAG_TENSOR_F16 and MSOSM_FLAG_TENSOR_BF16 exclude each other");
    }
    if (d->tc && !tc_supported(log2n)) {
        release(d);
        return fail(MSOSM_ERR_UNSUPPORTED, "the tensor-core path needs FFT size 4096, 8192 or 16384 (got %lu)", 2 * M);
    }
    if (input_size != 0)
        count = (int)(input_size / M);
    if (count < 1) {
        release(d);
        return fail(MSOSM_ERR_BAD_ARG, "count must be >= 1");
    }
    if ((unsigned long long)count * M >= (1ull << 31)) {
        release(d);
        return fail(MSOSM_ERR_BAD_ARG, "count*M = %llu samples per call exceeds 2^31 - 1",
                    (unsigned long long)count * M);
    }
    d->M = M;
    d->N = 2 * M;
    d->log2n = log2n;
    d->count = count;
    const unsigned long N = d->N;
    d->delays.assign((size_t)numDMs * N, 0);
    if (!osm) {
        for (int i = 0; i < numDMs; ++i)
            d->dc[i] = segment_delays(bw[i], dm[i], f0[i], d->Nd[i], M, d->delays.data() + (size_t)i * N);
    }
    for (int i = 0; i < numDMs; ++i) {
        d->max_dc = d->dc[i] > d->max_dc ? d->dc[i] : d->max_dc;
        for (unsigned long b = 0; b < N; ++b)
            d->max_delay = d->delays[(size_t)i * N + b] > d->max_delay ? d->delays[(size_t)i * N + b] : d->max_delay;
    }
    if (d->max_delay > 65535) {
        release(d);
        return fail(MSOSM_ERR_UNSUPPORTED, "block delay %d exceeds 65535", d->max_delay);
    }
    if (msosm_device_count() == 0) {
        release(d);
        return fail(MSOSM_ERR_NO_DEVICE, "no CUDA device");
    }
    // spectra of blocks [k0 - max_delay, k0 + count) must be resident; a
    // power-of-two depth turns the slot arithmetic into a mask
    {
        long long need = (long long)count + d->max_delay, S = 1;
        while (S < need)
            S <<= 1;
        if (S > (1ll << 30)) {
            release(d);
            return fail(MSOSM_ERR_BAD_ARG, "count + max delay too large");
        }
        d->S = (int)S;
    }
    if (const char *pp = std::getenv("MSOSM_DEDISP_PINGPONG"))
        d->pingpong = std::atoi(pp) != 0;

#define CKD(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            msosm_status s_ = cuda_fail(e_, #call);                                                    \
            release(d);                                                                                \
            return s_;                                                                                 \
        }                                                                                              \
    } while (0)

    CKD(cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking));
    CKD(cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking));
    d->stream = d->own_stream;
    for (int i = 0; i < 2; ++i) {
        CKD(cudaEventCreateWithFlags(&d->ev_copied[i], cudaEventDisableTiming));
        CKD(cudaEventCreateWithFlags(&d->ev_consumed[i], cudaEventDisableTiming));
        CKD(cudaEventCreateWithFlags(&d->ev_spans[i], cudaEventDisableTiming));
    }
    size_t &tot = d->device_bytes;
    CKD(dalloc(&d->ring, (size_t)d->S * N, tot));
    CKD(dalloc(&d->H, (size_t)numDMs * N, tot));
    CKD(dalloc(&d->delays_d, (size_t)numDMs * N, tot));
    CKD(dalloc(&d->hist, 2 * (size_t)M, tot));
    CKD(cudaMemsetAsync(d->hist, 0, sizeof(float2) * 2 * M, d->stream));
    for (int i = 0; i < 2; ++i)
        CKD(dalloc((float2 **)&d->staging[i], (size_t)count * M, tot));
    if (d->series)
        CKD(dalloc(&d->series_buf, (size_t)numDMs * count * M + 1, tot));
    if (d->large)
        large_split(log2n, d->log2n1, d->log2n2);
    {
        // per-bin delays on the device; for the four-step layout permuted to
        // position k1*N2 + k2 of bin k1 + N1*k2, for the tensor-core kernel
        // to tc_pos(bin)
        std::vector<uint16_t> dl(d->delays.size());
        const unsigned long N1 = 1ul << d->log2n1, N2 = 1ul << d->log2n2;
        for (int t = 0; t < numDMs; ++t)
            for (unsigned long p = 0; p < N; ++p) {
                const unsigned long b = d->large ? (p / N2) + N1 * (p % N2) : p;
                const unsigned long q = d->tc ? (unsigned long)tc::tc_pos((int)p, log2n) : p;
                dl[(size_t)t * N + q] = (uint16_t)d->delays[(size_t)t * N + b];
            }
        CKD(cudaMemcpy(d->delays_d, dl.data(), sizeof(uint16_t) * dl.size(), cudaMemcpyHostToDevice));
    }
    msosm_status s;
    std::vector<ChirpParams> cp(numDMs);
    for (int i = 0; i < numDMs; ++i)
        cp[i] = chirp_params(bw[i], dm[i], f0[i], M);
    // 1/N^2: the reference's /N before and /(2M) after the inverse FFT
    const float scale = 1.0f / ((float)N * (float)N);
    // the dispersion filter (+phase chirp) of MSOSM_FLAG_DISPERSE
    const int sign = (flags & MSOSM_FLAG_DISPERSE) ? +1 : -1;
    if (!d->large) {
        if ((s = upload_table(&d->tw_fwd, (int)N, -1, tot, d->stream)) != MSOSM_OK ||
            (s = upload_table(&d->tw_inv, (int)N, +1, tot, d->stream)) != MSOSM_OK ||
            (s = upload_table(&d->tw_inv_m, (int)M, +1, tot, d->stream)) != MSOSM_OK) {
            release(d);
            return s;
        }
        if ((s = design_filters(log2n, cp, scale, sign, d->tw_inv_m, d->tw_fwd, d->H, d->stream)) != MSOSM_OK) {
            release(d);
            return s;
        }
        if (d->tc) {
            float2 *tmp = nullptr;
            CKD(cudaMalloc((void **)&tmp, sizeof(float2) * (size_t)numDMs * N));
            cudaError_t e = launch_tc_permute_rows(d->H, tmp, numDMs, log2n, d->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d->H, tmp, sizeof(float2) * (size_t)numDMs * N, cudaMemcpyDeviceToDevice,
                                    d->stream);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(d->stream);
            cudaFree(tmp);
            CKD(e);
            CKD(dalloc(&d->status_d, 1, tot));
            CKD(cudaMemset(d->status_d, 0, sizeof(int)));
            // scale bounds: ring rows not yet written hold zero
            CKD(dalloc(&d->row_max, (size_t)d->S, tot));
            CKD(cudaMemset(d->row_max, 0, sizeof(float) * d->S));
            std::vector<float2> hh((size_t)numDMs * N);
            CKD(cudaMemcpy(hh.data(), d->H, sizeof(float2) * hh.size(), cudaMemcpyDeviceToHost));
            std::vector<float> hm(numDMs, 0.f);
            std::vector<int> dmx(numDMs, 0);
            for (int t = 0; t < numDMs; ++t)
                for (unsigned long b = 0; b < N; ++b) {
                    const float2 v = hh[(size_t)t * N + b];
                    hm[t] = std::fmax(hm[t], std::fmax(std::fabs(v.x), std::fabs(v.y)));
                    dmx[t] = std::max(dmx[t], d->delays[(size_t)t * N + b]);
                }
            CKD(dalloc(&d->h_max, (size_t)numDMs, tot));
            CKD(dalloc(&d->delay_max_d, (size_t)numDMs, tot));
            CKD(cudaMemcpy(d->h_max, hm.data(), sizeof(float) * numDMs, cudaMemcpyHostToDevice));
            CKD(cudaMemcpy(d->delay_max_d, dmx.data(), sizeof(int) * numDMs, cudaMemcpyHostToDevice));
        }
        CKD(plan_grid(d));
    } else {
        if ((s = upload_table(&d->tw1f, 1 << d->log2n1, -1, tot, d->stream)) != MSOSM_OK ||
            (s = upload_table(&d->tw1i, 1 << d->log2n1, +1, tot, d->stream)) != MSOSM_OK ||
            (s = upload_table(&d->tw2f, 1 << d->log2n2, -1, tot, d->stream)) != MSOSM_OK ||
            (s = upload_table(&d->tw2i, 1 << d->log2n2, +1, tot, d->stream)) != MSOSM_OK) {
            release(d);
            return s;
        }
        CKD(dalloc(&d->lA, (size_t)count * N, tot));
        CKD(dalloc(&d->lB, (size_t)numDMs * count * N, tot));
        if ((s = design_filters_large(log2n, cp, scale, sign, d->H, d->stream)) != MSOSM_OK) {
            release(d);
            return s;
        }
    }
#undef CKD
    *out = d;
    return MSOSM_OK;
}

msosm_status msosm_dedisp_destroy(msosm_dedisp *d)
{
    release(d);
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_info(const msosm_dedisp *d, msosm_dedisp_info *info)
{
    if (check_handle(d) || !info)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    info->M = d->M;
    info->fftpoint = d->N;
    info->M_min = d->M_min;
    info->count = d->count;
    info->numDMs = d->D;
    info->ring_slots = d->S;
    info->max_delaycount = d->max_dc;
    info->flags = d->flags;
    info->calls = d->calls;
    info->device_bytes = d->device_bytes;
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_nd(const msosm_dedisp *d, unsigned long *Nd)
{
    if (check_handle(d) || !Nd)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    for (int i = 0; i < d->D; ++i)
        Nd[i] = d->Nd[i];
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_delaycount(const msosm_dedisp *d, int *dc)
{
    if (check_handle(d) || !dc)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    for (int i = 0; i < d->D; ++i)
        dc[i] = d->dc[i];
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_delay_points(const msosm_dedisp *d, int i, int *dp)
{
    if (check_handle(d) || !dp || i < 0 || i >= d->D)
        return fail(MSOSM_ERR_BAD_ARG, "bad trial index or null output");
    std::memcpy(dp, d->delays.data() + (size_t)i * d->N, sizeof(int) * d->N);
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_dedisp_params(const msosm_dedisp *d, int i, msosm_complex *H)
{
    if (check_handle(d) || !H || i < 0 || i >= d->D)
        return fail(MSOSM_ERR_BAD_ARG, "bad trial index or null output");
    CK(cudaStreamSynchronize(d->stream));
    std::vector<msosm_complex> tmp(d->N);
    CK(cudaMemcpy(tmp.data(), d->H + (size_t)i * d->N, sizeof(float2) * d->N, cudaMemcpyDeviceToHost));
    const float up = (float)d->N * (float)d->N;  // undo the 1/N^2 (a power of two: exact)
    const unsigned long N1 = 1ul << d->log2n1, N2 = 1ul << d->log2n2;
    for (unsigned long b = 0; b < d->N; ++b) {
        // four-step layout: bin b = k1 + N1*k2 sits at k1*N2 + k2
        const unsigned long p = d->large ? (b % N1) * N2 + b / N1 : (d->tc ? (unsigned long)tc::tc_pos((int)b, d->log2n) : b);
        H[b].x = tmp[p].x * up;
        H[b].y = tmp[p].y * up;
    }
    return MSOSM_OK;
}

msosm_status msosm_dedisp_set_stream(msosm_dedisp *d, void *stream)
{
    if (check_handle(d))
        return MSOSM_ERR_BAD_ARG;
    CK(cudaStreamSynchronize(d->stream));
    d->stream = stream ? (cudaStream_t)stream : d->own_stream;
    return MSOSM_OK;
}

msosm_status msosm_dedisp_set_tc_wait_limit(msosm_dedisp *d, long long ns)
{
    if (check_handle(d))
        return fail(MSOSM_ERR_BAD_ARG, "null handle");
    if (!d->tc)
        return fail(MSOSM_ERR_STATE, "handle does not run the tensor-core kernel");
    d->tc_wait_limit_ns = ns < 0 ? kTcWaitLimitDefaultNs : ns;
    return MSOSM_OK;
}

// fold bookkeeping shared by both layouts: plan this call's spans, upload
// them, flush a pending period that completes now, clear the partial rows
static msosm_status fold_prepare(msosm_dedisp *d, int sb, FoldArgs &fa)
{
    bool flush = false;
    d->planner->chunk((unsigned long)d->count * d->M, d->spans, flush);
    const int n = (int)d->spans.size();
    if (n > d->span_cap)
        return fail(MSOSM_ERR_STATE, "fold planner produced %d spans (capacity %d)", n, d->span_cap);
    // reuse of the pinned span staging: wait for its copy two calls ago
    CK(cudaEventSynchronize(d->ev_spans[sb]));
    long long *h = d->span_host + (size_t)sb * 4 * d->span_cap;
    int *hp = reinterpret_cast<int *>(h + 2 * d->span_cap);
    for (int i = 0; i < n; ++i) {
        h[i] = d->spans[i].a;
        h[d->span_cap + i] = d->spans[i].b;
        hp[i] = d->spans[i].phase0;
        hp[d->span_cap + i] = d->spans[i].dest;
    }
    // a kernel reads the staging: copies on this stream would wait behind the
    // next call's input copy on the copy engine, and the dedispersion kernel
    // with them
    CK(launch_span_upload(h, n, d->span_cap, d->span_a_d, d->span_b_d, d->span_p_d, d->span_dest_d, d->stream));
    d->launches += n > 0 ? 1 : 0;
    CK(cudaEventRecord(d->ev_spans[sb], d->stream));
    if (flush) {
        CK(launch_fold_flush(d->acc_main, d->acc_pend, (size_t)d->D * d->nbins, d->stream));
        d->launches += 1;
    }
    const size_t prow = (size_t)d->D * d->R * d->nbins;
    CK(cudaMemsetAsync(d->part_main, 0, sizeof(float) * prow, d->stream));
    CK(cudaMemsetAsync(d->part_pend, 0, sizeof(float) * prow, d->stream));
    fa.span_a = d->span_a_d;
    fa.span_b = d->span_b_d;
    fa.span_phase0 = d->span_p_d;
    fa.span_dest = d->span_dest_d;
    fa.nspans = n;
    fa.bpt = d->bpt;
    fa.nbins = d->nbins;
    fa.detect = d->detect;
    fa.part_main = d->part_main;
    fa.part_pend = d->part_pend;
    fa.smem_prof = prof_in_smem(d) ? 1 : 0;
    fa.span_cap = d->win_cap;
    fa.inv_bpt = 1.0f / (float)d->bpt;
    fa.g_shift = fold_g_shift(d->bpt, d->large ? 256 : (int)(d->N / 16));
    return MSOSM_OK;
}

// One call with the four-step layout: column + row forward passes into the
// ring, then per trial the gathering inverse row pass and the pruned inverse
// column pass; folding runs over the materialised intensities.
static msosm_status filter_block_large(msosm_dedisp *d, const void *src, InputKind kind,
                                       msosm_dedisp::CallEvents *ev, unsigned long long launches0)
{
    const int sb = (int)(d->calls & 1);
    const long long N = (long long)d->N;
    LargeColArgs ca{};
    ca.input = src;
    ca.hist_in = d->hist + (size_t)(d->calls & 1) * d->M;
    ca.hist_out = d->hist + (size_t)((d->calls + 1) & 1) * d->M;
    ca.out = d->lA;
    ca.N = N;
    ca.N2 = 1ll << d->log2n2;
    ca.log2n = d->log2n;
    ca.count = d->count;
    ca.tw1 = d->tw1f;
    if (ev)
        CK(cudaEventRecord(ev->e[0], d->stream));
    CK(launch_large_col_fwd(d->log2n1, kind, ca, d->count, d->stream));
    LargeRowArgs ra{};
    ra.in = d->lA;
    ra.ring = d->ring;
    ra.S = d->S;
    ra.k0 = (long long)d->calls * d->count;
    ra.count = d->count;
    ra.N = N;
    ra.log2n = d->log2n;
    ra.tw2 = d->tw2f;
    CK(launch_large_row(d->log2n2, 0, ra, 1 << d->log2n1, d->count, 1, d->stream));
    d->launches += 2;
    CK(cudaEventRecord(d->ev_consumed[sb], d->stream));
    if (ev)
        CK(cudaEventRecord(ev->e[1], d->stream));
    FoldArgs fa{};
    if (d->fold) {
        msosm_status s = fold_prepare(d, sb, fa);
        if (s != MSOSM_OK)
            return s;
    }
    if (ev)
        CK(cudaEventRecord(ev->e[2], d->stream));
    ra.out = d->lB;
    ra.H = d->H;
    ra.delays = d->delays_d;
    ra.tw2 = d->tw2i;
    CK(launch_large_row(d->log2n2, 1, ra, 1 << d->log2n1, d->count, d->D, d->stream));
    LargeColArgs ia{};
    ia.in = d->lB;
    ia.N = N;
    ia.N2 = 1ll << d->log2n2;
    ia.log2n = d->log2n;
    ia.count = d->count;
    ia.tw1 = d->tw1i;
    ia.series = d->series_buf;
    ia.intensity = d->fold ? d->lI : nullptr;
    ia.detect = d->detect;
    CK(launch_large_col_inv(d->log2n1, ia, d->count, d->D, d->stream));
    d->launches += 2;
    if (ev)
        CK(cudaEventRecord(ev->e[3], d->stream));
    if (d->fold) {
        CK(launch_fold_series(d->lI, (long long)d->count * d->M, d->R, fa, d->grid, d->D, d->stream));
        CK(launch_fold_reduce(d->part_main, d->part_pend, d->D, d->R, d->nbins, d->acc_main, d->acc_pend,
                              d->stream));
        d->launches += 2;
    }
    if (d->series)
        CK(cudaMemsetAsync(d->series_buf + (size_t)d->D * d->count * d->M, 0, sizeof(float2), d->stream));
    if (ev) {
        CK(cudaEventRecord(ev->e[6], d->stream));
        d->timed_launches += d->launches - launches0;
    }
    d->calls += 1;
    return MSOSM_OK;
}

// After the handle's stream has drained: a timed-out wait of the
// tensor-core kernel (the results of the calls since the last check are then
// invalid).  The status word is cleared once reported, so the handle goes
// on with the next call.
static msosm_status kernel_status(msosm_dedisp *d)
{
    if (!d->status_d)
        return MSOSM_OK;
    int st = 0;
    CK(cudaMemcpy(&st, d->status_d, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) {
        CK(cudaMemset(d->status_d, 0, sizeof(int)));
        return fail(MSOSM_ERR_TIMEOUT, "tensor-core kernel: a wait on the tensor core timed out");
    }
    return MSOSM_OK;
}

// The first part of a filter call: the input staged (host inputs through a
// device buffer on the copy stream), the forward transform into the ring,
// the fold's spans for this call; da receives the dedispersion kernel's
// arguments.  For the four-step layout the whole call runs here (*done).
static msosm_status call_begin(msosm_dedisp *d, const void *input, InputKind kind, msosm_dedisp::CallEvents *ev,
                               unsigned long long launches0, DedispArgs &da, bool &done)
{
    done = false;
    const size_t elem = kind == kInputU16 ? 4 : 8;
    const size_t bytes = (size_t)d->count * d->M * elem;
    const int sb = (int)(d->calls & 1);
    const void *src = input;
    if (!is_device_ptr(input)) {
        // stage through a device buffer on the copy stream; the host buffer
        // may be reused as soon as this call returns
        CK(cudaStreamWaitEvent(d->copy_stream, d->ev_consumed[sb], 0));
        if (ev) {
            CK(cudaEventRecord(ev->e[4], d->copy_stream));
            ev->h2d = true;
        }
        CK(cudaMemcpyAsync(d->staging[sb], input, bytes, cudaMemcpyHostToDevice, d->copy_stream));
        if (ev)
            CK(cudaEventRecord(ev->e[5], d->copy_stream));
        CK(cudaEventRecord(d->ev_copied[sb], d->copy_stream));
        CK(cudaEventSynchronize(d->ev_copied[sb]));
        CK(cudaStreamWaitEvent(d->stream, d->ev_copied[sb], 0));
        src = d->staging[sb];
    }
    if (d->large) {
        done = true;
        return filter_block_large(d, src, kind, ev, launches0);
    }
    FwdArgs fa{};
    fa.input = src;
    fa.hist_in = d->hist + (size_t)(d->calls & 1) * d->M;
    fa.hist_out = d->hist + (size_t)((d->calls + 1) & 1) * d->M;
    fa.ring = d->ring;
    fa.S = d->S;
    fa.k0 = (long long)d->calls * d->count;
    fa.count = d->count;
    fa.tw = d->tw_fwd;
    fa.tc_order = d->tc ? 1 : 0;
    fa.row_max = d->row_max;
    if (ev)
        CK(cudaEventRecord(ev->e[0], d->stream));
    CK(launch_forward(d->log2n, kind, fa, d->stream));
    d->launches += 1;
    CK(cudaEventRecord(d->ev_consumed[sb], d->stream));
    if (ev)
        CK(cudaEventRecord(ev->e[1], d->stream));

    da = DedispArgs{};
    da.ring = d->ring;
    da.S = d->S;
    da.max_delay = d->max_delay;
    da.k0 = fa.k0;
    da.count = d->count;
    da.D = d->D;
    da.R = d->R;
    da.H = d->H;
    da.delays = d->delays_d;
    da.tw = d->tw_inv;
    da.series = d->series_buf;
    da.fold.nspans = -1;
    da.status = d->status_d;
    da.wait_limit_ns = d->tc_wait_limit_ns;
    da.row_max = d->row_max;
    da.h_max = d->h_max;
    da.delay_max = d->delay_max_d;
    if (d->fold) {
        msosm_status st = fold_prepare(d, sb, da.fold);
        if (st != MSOSM_OK)
            return st;
    }
    return MSOSM_OK;
}

// The last part of a filter call, after the dedispersion kernel: the ordered
// reduction of the R partial profile rows, the series' trailing element.
static msosm_status call_end(msosm_dedisp *d, msosm_dedisp::CallEvents *ev, int R, unsigned long long launches0)
{
    if (d->fold) {
        CK(launch_fold_reduce(d->part_main, d->part_pend, d->D, R, d->nbins, d->acc_main, d->acc_pend, d->stream));
        d->launches += 1;
    }
    if (d->series)
        CK(cudaMemsetAsync(d->series_buf + (size_t)d->D * d->count * d->M, 0, sizeof(float2), d->stream));
    if (ev) {
        CK(cudaEventRecord(ev->e[6], d->stream));
        d->timed_launches += d->launches - launches0;
    }
    d->calls += 1;
    return MSOSM_OK;
}

static msosm_status filter_block(msosm_dedisp *d, const void *input, InputKind kind)
{
    if (check_handle(d) || !input)
        return fail(MSOSM_ERR_BAD_ARG, "null handle or input");
    msosm_dedisp::CallEvents *ev = nullptr;
    if (d->timing) {
        msosm_dedisp::CallEvents c{};
        for (cudaEvent_t &e : c.e)
            CK(cudaEventCreate(&e));
        c.h2d = false;
        d->timed.push_back(c);
        ev = &d->timed.back();
    }
    const unsigned long long launches0 = d->launches;
    DedispArgs da;
    bool done = false;
    msosm_status st = call_begin(d, input, kind, ev, launches0, da, done);
    if (st != MSOSM_OK || done)
        return st;
    // the partial-row clears and the flush above belong to the fold time;
    // the dedispersion kernel is timed alone
    if (ev)
        CK(cudaEventRecord(ev->e[2], d->stream));
    if (d->tc)
        CK(launch_tc_dedisp(d->log2n, d->tc_bf16, d->series, d->fold, da, d->grid, d->stream));
    else
        CK(launch_dedisp(d->log2n, d->pingpong, d->series, d->fold, da, d->grid, d->stream));
    d->launches += 1;
    if (ev)
        CK(cudaEventRecord(ev->e[3], d->stream));
    return call_end(d, ev, d->R, launches0);
}

// ---------------------------------------------------------------------------
// batches: one filter call of many handles, one launch per kernel group
// ---------------------------------------------------------------------------

struct msosm_batch {
    struct Group {
        std::vector<int> members;  // handle indices, largest work items first (at most kBatchMax)
        std::vector<int> R;        // block ranges per trial of each member in this batch
        int log2n = 0;
        bool bf16 = false, series = false, fold = false;
        size_t fold_smem = 0;
        int grid = 1;
        int items = 0;
        int *counter_d = nullptr;
        std::unique_ptr<BatchArgs> args;  // the launch's parameter: prefix and arguments
    };
    std::vector<msosm_dedisp *> h;
    std::vector<Group> groups;
    std::vector<int> alone;  // handles launched one by one
    cudaStream_t stream = nullptr;      // the stream everything runs on
    cudaStream_t own_stream = nullptr;  // the batch's own (the default)
    unsigned long long calls = 0;
};

static void batch_release(msosm_batch *b)
{
    if (!b)
        return;
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    for (auto &g : b->groups)
        cudaFree(g.counter_d);
    // the handles go back to their own streams
    for (msosm_dedisp *d : b->h)
        if (d->stream == b->stream)
            d->stream = d->own_stream;
    if (b->own_stream)
        cudaStreamDestroy(b->own_stream);
    delete b;
}

msosm_status msosm_batch_create(msosm_dedisp *const *handles, int n, msosm_batch **out)
{
    if (!out || !handles || n < 1)
        return fail(MSOSM_ERR_BAD_ARG, "msosm_batch_create: null argument or n < 1");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (check_handle(handles[i]))
            return fail(MSOSM_ERR_BAD_ARG, "msosm_batch_create: handle %d is null", i);
        for (int j = 0; j < i; ++j)
            if (handles[j] == handles[i])
                return fail(MSOSM_ERR_BAD_ARG, "msosm_batch_create: handle %d appears twice", i);
    }
    msosm_batch *b = new (std::nothrow) msosm_batch;
    if (!b)
        return fail(MSOSM_ERR_OOM, "host allocation");
    b->h.assign(handles, handles + n);
#define CKB(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            msosm_status s_ = cuda_fail(e_, #call);                                                      \
            batch_release(b);                                                                            \
            return s_;                                                                                   \
        }                                                                                                \
    } while (0)
    CKB(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
    b->stream = b->own_stream;
    int dev = 0, sms = 1;
    CKB(cudaGetDevice(&dev));
    CKB(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int i = 0; i < n; ++i) {
        msosm_dedisp *d = b->h[i];
        // every handle's earlier work is done before the batch's stream takes over
        CKB(cudaStreamSynchronize(d->stream));
        d->stream = b->stream;
        if (!d->tc || d->large) {
            b->alone.push_back(i);
            continue;
        }
        int gi = -1;
        for (size_t k = 0; k < b->groups.size(); ++k) {
            const auto &g = b->groups[k];
            if (g.log2n == d->log2n && g.bf16 == d->tc_bf16 && g.series == d->series && g.fold == d->fold &&
                (int)g.members.size() < kBatchMax)
                gi = (int)k;
        }
        if (gi < 0) {
            b->groups.emplace_back();
            gi = (int)b->groups.size() - 1;
            auto &g = b->groups.back();
            g.log2n = d->log2n;
            g.bf16 = d->tc_bf16;
            g.series = d->series;
            g.fold = d->fold;
        }
        b->groups[gi].members.push_back(i);
    }
    for (auto &g : b->groups) {
        // each member keeps its own cut of trials into block ranges and its
        // item order (range-major, so the CTAs working at one time read the
        // same ring rows, which stay in L2 for every trial), as in its own
        // calls; members are ordered largest first, so the last items of the
        // launch are small ones
        for (int i : g.members) {
            const msosm_dedisp *d = b->h[i];
            if (g.fold)
                g.fold_smem = std::max(g.fold_smem, fold_smem_bytes(d->nbins, d->win_cap, prof_in_smem(d),
                                                                    tc_threads(d->log2n)));
        }
        int per_sm = tc_blocks_per_sm(g.log2n, g.bf16, g.series, g.fold, g.fold_smem);
        if (per_sm < 1)
            per_sm = 1;
        const long long resident = (long long)per_sm * sms;
        std::vector<std::pair<long long, int>> order;
        for (int i : g.members) {
            const msosm_dedisp *d = b->h[i];
            const int bps = tc_blocks_per_step(d->log2n);
            order.push_back({(long long)d->D * ((d->count + bps - 1) / bps), i});
        }
        std::stable_sort(order.begin(), order.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
        g.members.clear();
        std::vector<int> prefix(1, 0);
        for (const auto &o : order) {
            const msosm_dedisp *d = b->h[o.second];
            g.members.push_back(o.second);
            g.R.push_back(d->R);
            prefix.push_back(prefix.back() + d->D * d->R);
        }
        g.items = prefix.back();
        g.grid = (int)std::min<long long>(g.items, resident);
        const size_t nm = g.members.size();
        CKB(cudaMalloc((void **)&g.counter_d, sizeof(int)));
        g.args.reset(new (std::nothrow) BatchArgs{});
        if (!g.args) {
            batch_release(b);
            return fail(MSOSM_ERR_OOM, "host allocation");
        }
        g.args->nobs = (int)nm;
        g.args->counter = g.counter_d;
        for (size_t j = 0; j <= nm; ++j)
            g.args->prefix[j] = prefix[j];
    }
#undef CKB
    *out = b;
    return MSOSM_OK;
}

msosm_status msosm_batch_destroy(msosm_batch *b)
{
    batch_release(b);
    return MSOSM_OK;
}

msosm_status msosm_batch_get_info(const msosm_batch *b, int *groups, int *launches_per_call, int *items)
{
    if (!b)
        return fail(MSOSM_ERR_BAD_ARG, "null batch");
    if (groups)
        *groups = (int)b->groups.size();
    if (launches_per_call)
        *launches_per_call = (int)(b->groups.size() + b->alone.size());
    if (items) {
        int t = 0;
        for (const auto &g : b->groups)
            t += g.items;
        *items = t;
    }
    return MSOSM_OK;
}

msosm_status msosm_batch_filter(msosm_batch *b, const void *const *inputs, int input_kind)
{
    if (!b || !inputs)
        return fail(MSOSM_ERR_BAD_ARG, "null batch or inputs");
    if (input_kind != MSOSM_INPUT_UINT16 && input_kind != MSOSM_INPUT_C64)
        return fail(MSOSM_ERR_BAD_ARG, "input_kind must be MSOSM_INPUT_UINT16 or MSOSM_INPUT_C64");
    const InputKind kind = input_kind == MSOSM_INPUT_UINT16 ? kInputU16 : kInputC64;
    for (size_t i = 0; i < b->h.size(); ++i)
        if (!inputs[i])
            return fail(MSOSM_ERR_BAD_ARG, "input %zu is null", i);
    // handles outside every group: their whole call, one after another
    for (int i : b->alone) {
        msosm_status st = filter_block(b->h[i], inputs[i], kind);
        if (st != MSOSM_OK)
            return st;
    }
    for (auto &g : b->groups) {
        const size_t nm = g.members.size();
        std::vector<unsigned long long> l0(nm);
        for (size_t j = 0; j < nm; ++j) {
            msosm_dedisp *d = b->h[g.members[j]];
            l0[j] = d->launches;
            bool done = false;
            msosm_status st = call_begin(d, inputs[g.members[j]], kind, nullptr, l0[j], g.args->args[j], done);
            if (st != MSOSM_OK)
                return st;
            g.args->args[j].R = g.R[j];
        }
        CK(cudaMemsetAsync(g.counter_d, 0, sizeof(int), b->stream));
        // the table travels as the launch's parameter (copied at the launch)
        CK(launch_tc_dedisp_batch(g.log2n, g.bf16, g.series, g.fold, *g.args, g.fold_smem, g.grid, b->stream));
        for (size_t j = 0; j < nm; ++j) {
            msosm_dedisp *d = b->h[g.members[j]];
            msosm_status st = call_end(d, nullptr, g.R[j], l0[j]);
            if (st != MSOSM_OK)
                return st;
        }
    }
    b->calls += 1;
    return MSOSM_OK;
}

msosm_status msosm_batch_set_stream(msosm_batch *b, void *stream)
{
    if (!b)
        return fail(MSOSM_ERR_BAD_ARG, "null batch");
    CK(cudaStreamSynchronize(b->stream));
    b->stream = stream ? (cudaStream_t)stream : b->own_stream;
    for (msosm_dedisp *d : b->h)
        d->stream = b->stream;
    return MSOSM_OK;
}

msosm_status msosm_batch_synchronize(msosm_batch *b)
{
    if (!b)
        return fail(MSOSM_ERR_BAD_ARG, "null batch");
    CK(cudaStreamSynchronize(b->stream));
    for (msosm_dedisp *d : b->h) {
        msosm_status st = kernel_status(d);
        if (st != MSOSM_OK)
            return st;
    }
    return MSOSM_OK;
}

msosm_status msosm_dedisp_filter_block_uint16(msosm_dedisp *d, const msosm_uint16_pair *input)
{
    return filter_block(d, input, kInputU16);
}

msosm_status msosm_dedisp_filter_block_c64(msosm_dedisp *d, const msosm_complex *input)
{
    return filter_block(d, input, kInputC64);
}

msosm_status msosm_dedisp_get_output_c64(msosm_dedisp *d, msosm_complex *out)
{
    if (check_handle(d) || !out)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    if (!d->series)
        return fail(MSOSM_ERR_STATE, "handle created with MSOSM_FLAG_NO_SERIES");
    const size_t n = (size_t)d->D * d->count * d->M + 1;
    CK(cudaMemcpyAsync(out, d->series_buf, sizeof(float2) * n, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return kernel_status(d);
}

msosm_status msosm_dedisp_get_output_uint16(msosm_dedisp *d, msosm_uint16_pair *out)
{
    if (check_handle(d) || !out)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    if (!d->series)
        return fail(MSOSM_ERR_STATE, "handle created with MSOSM_FLAG_NO_SERIES");
    const size_t n = (size_t)d->D * d->count * d->M + 1;
    if (!d->u16_out)
        CK(dalloc(&d->u16_out, n, d->device_bytes));
    CK(launch_encode_u16(d->series_buf, d->u16_out, n, d->stream));
    CK(cudaMemcpyAsync(out, d->u16_out, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return kernel_status(d);
}

msosm_status msosm_dedisp_output_device_ptr(msosm_dedisp *d, msosm_complex **ptr)
{
    if (check_handle(d) || !ptr)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    *ptr = reinterpret_cast<msosm_complex *>(d->series_buf);
    return d->series ? MSOSM_OK : fail(MSOSM_ERR_STATE, "handle created with MSOSM_FLAG_NO_SERIES");
}

msosm_status msosm_dedisp_fold_init(msosm_dedisp *d, float period, float fs, unsigned long time_bin,
                                    unsigned long discard_Nd, int detect)
{
    if (check_handle(d))
        return MSOSM_ERR_BAD_ARG;
    if (d->fold)
        return fail(MSOSM_ERR_STATE, "fold already configured");
    if (detect != MSOSM_DETECT_POWER && detect != MSOSM_DETECT_AMPLITUDE)
        return fail(MSOSM_ERR_BAD_ARG, "unknown detection %d", detect);
    if (!(period > 0) || !(fs > 0))
        return fail(MSOSM_ERR_BAD_ARG, "period and fs must be positive");
    FoldPlanner *p = new (std::nothrow) FoldPlanner(period, fs, discard_Nd, true);
    if (!p)
        return fail(MSOSM_ERR_OOM, "host allocation");
    const unsigned long ps = p->period_samples();
    if (ps == 0 || ps > (1ul << 30)) {
        delete p;
        return fail(MSOSM_ERR_BAD_ARG, "period*fs gives %lu samples", ps);
    }
    const unsigned long nb = time_bin == 0 ? ps : time_bin;
    if (nb > ps || nb > (1ul << 22)) {
        delete p;
        return fail(MSOSM_ERR_BAD_ARG, "time_bin %lu exceeds period_samples %lu or 2^22", nb, ps);
    }
    d->planner = p;
    d->ps = ps;
    d->nbins = (int)nb;
    d->bpt = nb == ps ? 1 : (int)(ps / nb);
    d->out_scale = nb == ps ? 1.0 : 1.0 / (double)d->bpt;
    d->detect = detect;
    d->span_cap = (int)((unsigned long)d->count * d->M / ps) + 8;
    // spans one block can touch: ceil(M/ps) + 2 periods
    d->win_cap = (int)(d->M / ps) + 4;
    if (d->win_cap < 64)
        d->win_cap = 64;
    d->fold = true;
    if (!d->large) {
        cudaError_t e = plan_grid(d);
        if (e != cudaSuccess) {
            d->fold = false;
            return cuda_fail(e, "plan_grid");
        }
    } else {
        // the series fold: ranges of 2048-sample blocks per trial, about four
        // thread blocks per SM over all trials
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const long long nblk = ((long long)d->count * d->M + fold_series_block() - 1) / fold_series_block();
        long long R = (4ll * (sms > 0 ? sms : 1) + d->D - 1) / d->D;
        R = R > nblk ? nblk : (R < 1 ? 1 : R);
        d->R = (int)R;
        d->grid = (int)R;
    }
    d->fold = false;
    size_t &tot = d->device_bytes;
    if (d->large)
        CK(dalloc(&d->lI, (size_t)d->D * d->count * d->M, tot));
    const size_t prow = (size_t)d->D * d->R * d->nbins;
    const size_t nacc = (size_t)d->D * d->nbins;
    CK(dalloc(&d->part_main, prow, tot));
    CK(dalloc(&d->part_pend, prow, tot));
    CK(dalloc(&d->acc_main, nacc, tot));
    CK(dalloc(&d->acc_pend, nacc, tot));
    CK(dalloc(&d->prof_out, nacc, tot));
    CK(dalloc(&d->span_a_d, (size_t)d->span_cap, tot));
    CK(dalloc(&d->span_b_d, (size_t)d->span_cap, tot));
    CK(dalloc(&d->span_p_d, (size_t)d->span_cap, tot));
    CK(dalloc(&d->span_dest_d, (size_t)d->span_cap, tot));
    CK(cudaMallocHost((void **)&d->span_host, sizeof(long long) * 2 * 4 * d->span_cap));
    CK(cudaMemsetAsync(d->acc_main, 0, sizeof(double) * nacc, d->stream));
    CK(cudaMemsetAsync(d->acc_pend, 0, sizeof(double) * nacc, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    d->fold = true;
    return MSOSM_OK;
}

// Frees what fold_init allocated and forgets the fold configuration.
static void fold_free(msosm_dedisp *d)
{
    void *bufs[] = {d->part_main, d->part_pend, d->acc_main, d->acc_pend, d->prof_out,
                    d->span_a_d, d->span_b_d, d->span_p_d, d->span_dest_d, d->lI};
    for (void *p : bufs)
        if (p)
            cudaFree(p);
    if (d->span_host)
        cudaFreeHost(d->span_host);
    const size_t prow = (size_t)d->D * d->R * d->nbins, nacc = (size_t)d->D * d->nbins;
    size_t freed = 2 * prow * sizeof(float) + 2 * nacc * sizeof(double) + nacc * sizeof(float) +
                   (size_t)d->span_cap * (2 * sizeof(long long) + 2 * sizeof(int));
    if (d->large)
        freed += (size_t)d->D * d->count * d->M * sizeof(float);
    d->device_bytes = d->device_bytes > freed ? d->device_bytes - freed : 0;
    d->part_main = d->part_pend = d->prof_out = d->lI = nullptr;
    d->acc_main = d->acc_pend = nullptr;
    d->span_a_d = d->span_b_d = nullptr;
    d->span_p_d = d->span_dest_d = nullptr;
    d->span_host = nullptr;
    delete d->planner;
    d->planner = nullptr;
    d->fold = false;
}

msosm_status msosm_dedisp_reset(msosm_dedisp *d)
{
    if (check_handle(d))
        return fail(MSOSM_ERR_BAD_ARG, "null handle");
    CK(cudaStreamSynchronize(d->stream));
    CK(cudaStreamSynchronize(d->copy_stream));
    // the kernels read no ring row of a block before the stream start, so a
    // new stream needs only the zero history of its first window
    CK(cudaMemset(d->hist, 0, sizeof(float2) * 2 * d->M));
    d->calls = 0;
    if (d->fold)
        fold_free(d);
    if (d->status_d)
        CK(cudaMemset(d->status_d, 0, sizeof(int)));
    if (!d->large) {
        // the grid the handle had before fold_init
        cudaError_t e = plan_grid(d);
        if (e != cudaSuccess)
            return cuda_fail(e, "plan_grid");
    }
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_profiles(msosm_dedisp *d, float *out)
{
    if (check_handle(d) || !out)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    if (!d->fold)
        return fail(MSOSM_ERR_STATE, "fold not configured (msosm_dedisp_fold_init)");
    const size_t n = (size_t)d->D * d->nbins;
    CK(launch_fold_readout(d->acc_main, n, d->out_scale, d->prof_out, d->stream));
    CK(cudaMemcpyAsync(out, d->prof_out, sizeof(float) * n, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return kernel_status(d);
}

msosm_status msosm_dedisp_folded_periods(const msosm_dedisp *d, unsigned long long *n)
{
    if (check_handle(d) || !n)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    *n = d->planner ? d->planner->completed_folded() : 0;
    return MSOSM_OK;
}

msosm_status msosm_dedisp_synchronize(msosm_dedisp *d)
{
    if (check_handle(d))
        return MSOSM_ERR_BAD_ARG;
    CK(cudaStreamSynchronize(d->stream));
    CK(cudaStreamSynchronize(d->copy_stream));
    return kernel_status(d);
}

msosm_status msosm_dedisp_enable_timing(msosm_dedisp *d, int on)
{
    if (check_handle(d))
        return MSOSM_ERR_BAD_ARG;
    CK(cudaStreamSynchronize(d->stream));
    for (auto &c : d->timed)
        for (cudaEvent_t e : c.e)
            cudaEventDestroy(e);
    d->timed.clear();
    d->timed_launches = 0;
    d->timing = on != 0;
    return MSOSM_OK;
}

msosm_status msosm_dedisp_get_timing(msosm_dedisp *d, msosm_timing *t)
{
    if (check_handle(d) || !t)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    CK(cudaStreamSynchronize(d->stream));
    CK(cudaStreamSynchronize(d->copy_stream));
    std::memset(t, 0, sizeof *t);
    for (auto &c : d->timed) {
        float a = 0, b = 0, f = 0, g = 0, h = 0;
        CK(cudaEventElapsedTime(&a, c.e[0], c.e[1]));
        CK(cudaEventElapsedTime(&b, c.e[2], c.e[3]));
        CK(cudaEventElapsedTime(&f, c.e[1], c.e[2]));
        CK(cudaEventElapsedTime(&g, c.e[3], c.e[6]));
        t->forward_ms += a;
        t->dedisp_ms += b;
        t->fold_ms += f + g;
        if (c.h2d) {
            CK(cudaEventElapsedTime(&h, c.e[4], c.e[5]));
            t->h2d_ms += h;
        }
    }
    t->calls = d->timed.size();
    t->kernel_launches = d->timed_launches;
    return MSOSM_OK;
}

// ---------------------------------------------------------------------------
// Fold_GPU
// ---------------------------------------------------------------------------

struct msosm_fold {
    unsigned long size = 0, ps = 0;
    int nbins = 0, bpt = 1, span_cap = 0, win_cap = 64, R = 1, grid = 1;
    double out_scale = 1.0;
    float period = 0.f, fs = 0.f;
    FoldPlanner *planner = nullptr;
    bool started = false;
    std::vector<FoldSpan> spans;
    cudaStream_t stream = nullptr;
    float *I = nullptr, *part_main = nullptr, *part_pend = nullptr, *prof_out = nullptr;
    double *acc_main = nullptr, *acc_pend = nullptr;
    long long *span_a = nullptr, *span_b = nullptr;
    int *span_p = nullptr, *span_dest = nullptr;
    long long *span_host = nullptr;
};

static void fold_release(msosm_fold *f)
{
    if (!f)
        return;
    if (f->stream)
        cudaStreamSynchronize(f->stream);
    void *bufs[] = {f->I, f->part_main, f->part_pend, f->prof_out, f->acc_main, f->acc_pend,
                    f->span_a, f->span_b, f->span_p, f->span_dest};
    for (void *p : bufs)
        if (p)
            cudaFree(p);
    if (f->span_host)
        cudaFreeHost(f->span_host);
    if (f->stream)
        cudaStreamDestroy(f->stream);
    delete f->planner;
    delete f;
}

msosm_status msosm_fold_create(float period, float fs, unsigned long size, unsigned long time_bin, msosm_fold **out)
{
    if (!out || !(period > 0) || !(fs > 0) || size == 0 || size >= (1ul << 31))
        return fail(MSOSM_ERR_BAD_ARG, "msosm_fold_create: period, fs must be positive, 0 < size < 2^31");
    *out = nullptr;
    if (msosm_device_count() == 0)
        return fail(MSOSM_ERR_NO_DEVICE, "no CUDA device");
    msosm_fold *f = new (std::nothrow) msosm_fold;
    if (!f)
        return fail(MSOSM_ERR_OOM, "host allocation");
    f->period = period;
    f->fs = fs;
    f->size = size;
    // period_samples as fold_gpu.cpp:5-7 computes it
    const float psf = period * fs;
    f->ps = (unsigned long)psf;
    if (f->ps == 0 || f->ps > (1ul << 30)) {
        fold_release(f);
        return fail(MSOSM_ERR_BAD_ARG, "period*fs gives %lu samples", f->ps);
    }
    const unsigned long nb = (time_bin == 0 || time_bin == (unsigned long)-1) ? f->ps : time_bin;
    if (nb > f->ps || nb > (1ul << 22)) {
        fold_release(f);
        return fail(MSOSM_ERR_BAD_ARG, "time_bin %lu exceeds period_samples %lu", time_bin, f->ps);
    }
    f->nbins = (int)nb;
    f->bpt = nb == f->ps ? 1 : (int)(f->ps / nb);
    f->out_scale = nb == f->ps ? 1.0 : 1.0 / (double)f->bpt;
    f->span_cap = (int)(size / f->ps) + 8;
    f->win_cap = (int)((unsigned long)fold_series_block() / f->ps) + 4;
    if (f->win_cap < 64)
        f->win_cap = 64;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = ((long long)size + fold_series_block() - 1) / fold_series_block();
    long long R = 4ll * (sms > 0 ? sms : 1);
    if (R > blocks)
        R = blocks;
    f->R = (int)(R < 1 ? 1 : R);
    f->grid = f->R;
    size_t tot = 0;
#define CKF(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            msosm_status s_ = cuda_fail(e_, #call);                                                    \
            fold_release(f);                                                                           \
            return s_;                                                                                 \
        }                                                                                              \
    } while (0)
    CKF(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
    CKF(dalloc(&f->I, size, tot));
    CKF(dalloc(&f->part_main, (size_t)f->R * f->nbins, tot));
    CKF(dalloc(&f->part_pend, (size_t)f->R * f->nbins, tot));
    CKF(dalloc(&f->acc_main, (size_t)f->nbins, tot));
    CKF(dalloc(&f->acc_pend, (size_t)f->nbins, tot));
    CKF(dalloc(&f->prof_out, (size_t)f->nbins, tot));
    CKF(dalloc(&f->span_a, (size_t)f->span_cap, tot));
    CKF(dalloc(&f->span_b, (size_t)f->span_cap, tot));
    CKF(dalloc(&f->span_p, (size_t)f->span_cap, tot));
    CKF(dalloc(&f->span_dest, (size_t)f->span_cap, tot));
    CKF(cudaMallocHost((void **)&f->span_host, sizeof(long long) * 4 * f->span_cap));
    CKF(cudaMemsetAsync(f->acc_main, 0, sizeof(double) * f->nbins, f->stream));
    CKF(cudaMemsetAsync(f->acc_pend, 0, sizeof(double) * f->nbins, f->stream));
    CKF(cudaMemsetAsync(f->I, 0, sizeof(float) * size, f->stream));
    CKF(cudaStreamSynchronize(f->stream));
#undef CKF
    f->planner = new (std::nothrow) FoldPlanner(period, fs, 0, true);
    if (!f->planner) {
        fold_release(f);
        return fail(MSOSM_ERR_OOM, "host allocation");
    }
    *out = f;
    return MSOSM_OK;
}

msosm_status msosm_fold_destroy(msosm_fold *f)
{
    fold_release(f);
    return MSOSM_OK;
}

msosm_status msosm_fold_discard_samples(msosm_fold *f, unsigned long Nd)
{
    if (!f)
        return fail(MSOSM_ERR_BAD_ARG, "null handle");
    if (f->started)
        return fail(MSOSM_ERR_STATE, "discard_samples after the first fold_data");
    FoldPlanner *p = new (std::nothrow) FoldPlanner(f->period, f->fs, Nd, true);
    if (!p)
        return fail(MSOSM_ERR_OOM, "host allocation");
    delete f->planner;
    f->planner = p;
    return MSOSM_OK;
}

msosm_status msosm_fold_calculate_intensity(msosm_fold *f, const msosm_complex *a, const msosm_complex *b)
{
    if (!f || !a)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    if (!is_device_ptr(a) || (b && !is_device_ptr(b)))
        return fail(MSOSM_ERR_BAD_ARG, "calculate_intensity takes device series (e.g. output_buffer_d)");
    // the producer of a and b is unknown: wait for all prior device work
    CK(cudaDeviceSynchronize());
    CK(launch_intensity(reinterpret_cast<const float2 *>(a), reinterpret_cast<const float2 *>(b), f->I, f->size,
                        f->stream));
    return MSOSM_OK;
}

msosm_status msosm_fold_calculate_intensity_dedisp(msosm_fold *f, msosm_dedisp *a, msosm_dedisp *b)
{
    if (!f || !a)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    msosm_dedisp *hs[2] = {a, b};
    for (msosm_dedisp *d : hs) {
        if (!d)
            continue;
        if (!d->series)
            return fail(MSOSM_ERR_STATE, "handle created with MSOSM_FLAG_NO_SERIES");
        if ((unsigned long)d->count * d->M != f->size || d->D != 1)
            return fail(MSOSM_ERR_BAD_ARG, "series of %d trial(s) x %lu samples, fold chunk is %lu samples", d->D,
                        (unsigned long)d->count * d->M, f->size);
    }
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaSuccess;
    for (msosm_dedisp *d : hs)
        if (d && e == cudaSuccess) {
            e = cudaEventRecord(ev, d->stream);
            if (e == cudaSuccess)
                e = cudaStreamWaitEvent(f->stream, ev, 0);
        }
    if (e == cudaSuccess)
        e = launch_intensity(a->series_buf, b ? b->series_buf : nullptr, f->I, f->size, f->stream);
    // the handles' next calls overwrite their series: order them after this read
    if (e == cudaSuccess)
        e = cudaEventRecord(ev, f->stream);
    for (msosm_dedisp *d : hs)
        if (d && e == cudaSuccess)
            e = cudaStreamWaitEvent(d->stream, ev, 0);
    cudaEventDestroy(ev);
    if (e != cudaSuccess)
        return cuda_fail(e, "calculate_intensity");
    return MSOSM_OK;
}

msosm_status msosm_fold_set_intensity(msosm_fold *f, const float *intensity)
{
    if (!f || !intensity)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    CK(cudaMemcpyAsync(f->I, intensity, sizeof(float) * f->size, cudaMemcpyDefault, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return MSOSM_OK;
}

msosm_status msosm_fold_get_intensity(msosm_fold *f, float *out)
{
    if (!f || !out)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    CK(cudaMemcpyAsync(out, f->I, sizeof(float) * f->size, cudaMemcpyDefault, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return MSOSM_OK;
}

msosm_status msosm_fold_data(msosm_fold *f)
{
    if (!f)
        return fail(MSOSM_ERR_BAD_ARG, "null handle");
    f->started = true;
    bool flush = false;
    f->planner->chunk(f->size, f->spans, flush);
    const int n = (int)f->spans.size();
    if (n > f->span_cap)
        return fail(MSOSM_ERR_STATE, "fold planner produced %d spans (capacity %d)", n, f->span_cap);
    long long *h = f->span_host;
    int *hp = reinterpret_cast<int *>(h + 2 * f->span_cap);
    for (int i = 0; i < n; ++i) {
        h[i] = f->spans[i].a;
        h[f->span_cap + i] = f->spans[i].b;
        hp[i] = f->spans[i].phase0;
        hp[f->span_cap + i] = f->spans[i].dest;
    }
    // read by a kernel, not copied: see fold_prepare
    CK(launch_span_upload(h, n, f->span_cap, f->span_a, f->span_b, f->span_p, f->span_dest, f->stream));
    if (flush)
        CK(launch_fold_flush(f->acc_main, f->acc_pend, (size_t)f->nbins, f->stream));
    CK(cudaMemsetAsync(f->part_main, 0, sizeof(float) * f->R * f->nbins, f->stream));
    CK(cudaMemsetAsync(f->part_pend, 0, sizeof(float) * f->R * f->nbins, f->stream));
    FoldArgs a;
    a.span_a = f->span_a;
    a.span_b = f->span_b;
    a.span_phase0 = f->span_p;
    a.span_dest = f->span_dest;
    a.nspans = n;
    a.bpt = f->bpt;
    a.nbins = f->nbins;
    a.detect = 0;
    a.part_main = f->part_main;
    a.part_pend = f->part_pend;
    a.smem_prof = f->nbins <= kMaxSmemBins ? 1 : 0;
    a.span_cap = f->win_cap;
    a.inv_bpt = 1.0f / (float)f->bpt;
    a.g_shift = fold_g_shift(f->bpt, 256);
    CK(launch_fold_series(f->I, (long long)f->size, f->R, a, f->grid, 1, f->stream));
    CK(launch_fold_reduce(f->part_main, f->part_pend, 1, f->R, f->nbins, f->acc_main, f->acc_pend, f->stream));
    // the pinned span staging is reused by the next call
    CK(cudaStreamSynchronize(f->stream));
    return MSOSM_OK;
}

msosm_status msosm_fold_data_bins(msosm_fold *f, float *out)
{
    if (!f || !out)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    CK(launch_fold_readout(f->acc_main, (size_t)f->nbins, f->out_scale, f->prof_out, f->stream));
    CK(cudaMemcpyAsync(out, f->prof_out, sizeof(float) * f->nbins, cudaMemcpyDeviceToHost, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return MSOSM_OK;
}

msosm_status msosm_fold_get_shape(const msosm_fold *f, unsigned long *period_samples, unsigned long *time_bin)
{
    if (!f || !period_samples || !time_bin)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    *period_samples = f->ps;
    *time_bin = (unsigned long)f->nbins;
    return MSOSM_OK;
}

// ---------------------------------------------------------------------------
// fold planner introspection
// ---------------------------------------------------------------------------

struct msosm_fold_planner {
    FoldPlanner p;
    std::vector<FoldSpan> spans;
    msosm_fold_planner(float period, float fs, unsigned long nd) : p(period, fs, nd, true) {}
};

msosm_status msosm_fold_planner_create(float period, float fs, unsigned long discard_Nd, msosm_fold_planner **out)
{
    if (!out || !(period > 0) || !(fs > 0))
        return fail(MSOSM_ERR_BAD_ARG, "bad arguments");
    *out = new (std::nothrow) msosm_fold_planner(period, fs, discard_Nd);
    if (!*out)
        return fail(MSOSM_ERR_OOM, "host allocation");
    if ((*out)->p.period_samples() == 0) {
        delete *out;
        *out = nullptr;
        return fail(MSOSM_ERR_BAD_ARG, "period*fs < 1 sample");
    }
    return MSOSM_OK;
}

msosm_status msosm_fold_planner_destroy(msosm_fold_planner *p)
{
    delete p;
    return MSOSM_OK;
}

msosm_status msosm_fold_planner_chunk(msosm_fold_planner *p, unsigned long size, int64_t *dest,
                                      unsigned long long *completed)
{
    if (!p || !dest)
        return fail(MSOSM_ERR_BAD_ARG, "null argument");
    bool flush = false;
    p->p.chunk(size, p->spans, flush);
    for (unsigned long i = 0; i < size; ++i)
        dest[i] = -1;
    for (const FoldSpan &s : p->spans) {
        if (s.dest == 0)
            continue;
        for (int64_t t = s.a; t < s.b; ++t)
            dest[t] = (s.period << 32) | (int64_t)(s.phase0 + (t - s.a));
    }
    if (completed)
        *completed = p->p.completed_folded();
    return MSOSM_OK;
}

msosm_status msosm_tc_gemm_check(int step, const uint16_t *a, float *d)
{
    if (step < 1 || step > 4 || !a || !d)
        return fail(MSOSM_ERR_BAD_ARG, "step must be 1 .. 4; a and d non-null");
    if (msosm_device_count() == 0)
        return fail(MSOSM_ERR_NO_DEVICE, "no CUDA device");
    const size_t na = (size_t)128 * (step >= 3 ? 256 : 128);
    const size_t nd = (size_t)128 * (step == 3 ? 256 : (step == 2 ? 64 : 128));
    uint16_t *ad = nullptr;
    float *dd = nullptr;
    int *st = nullptr;
    int status = 0;
    cudaError_t e = cudaMalloc((void **)&ad, sizeof(uint16_t) * na);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&dd, sizeof(float) * nd);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&st, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemset(st, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpy(ad, a, sizeof(uint16_t) * na, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch_tc_probe(step, ad, dd, st, nullptr);
    if (e == cudaSuccess)
        e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(d, dd, sizeof(float) * nd, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&status, st, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(ad);
    cudaFree(dd);
    cudaFree(st);
    if (e != cudaSuccess)
        return cuda_fail(e, "tensor-core GEMM check");
    if (status != 0)
        return fail(MSOSM_ERR_TIMEOUT, "tensor-core GEMM check: wait timed out");
    return MSOSM_OK;
}

}  // extern "C"
