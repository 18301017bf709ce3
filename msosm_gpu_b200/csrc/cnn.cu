// cnn.cu -- the DM-proposal network: a small 1-D CNN over coarse-DM folded
// profiles, trained and run with these kernels (msosm_cnn_* of msosm_b200.h).
//
// Input [B][Cin][L]: the folded profiles of Cin coarse DM trials, L phase
// bins.  `layers` circular ("same", wrapping in phase) convolutions of
// `channels` outputs and odd kernel K, each with ReLU; the mean over phase;
// two linear heads, a detection logit and a DM offset.  Weights are held in
// FP32 (the optimiser's copy) and used rounded to bf16; every product is
// accumulated in FP32.  Loss: the logistic loss of the logit, plus dm_weight
// times the mean over positive samples of the squared offset error.  Every
// reduction runs in a fixed order, so a step is deterministic.
//
// Parameter vector (one FP32 array): per layer the weights [C_out][C_in][K]
// and biases [C_out]; then the detection head's weights [C] and bias, then
// the offset head's weights [C] and bias.
#include "msosm_b200.h"

#include <cmath>
#include <cstdio>
#include <new>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "kernels.hpp"

using namespace msosm;

namespace {

constexpr int kCoBlock = 8;  // output (or input) channels a thread accumulates

// x[b] -> xs[c][j] = x[b][c][(j - p) mod L], j < L + 2p (circular halo)
__device__ __forceinline__ void load_halo(const float *__restrict__ src, int C, int L, int p, float *xs)
{
    const int W = L + 2 * p;
    for (int e = threadIdx.x; e < C * W; e += blockDim.x) {
        const int c = e / W, j = e - c * W;
        int s = j - p;
        s += s < 0 ? L : 0;
        s -= s >= L ? L : 0;
        xs[e] = src[(size_t)c * L + s];
    }
}

// y[b][co][t] = relu(bias[co] + sum_ci sum_k w[co][ci][k] x[b][ci][t + k - p]),
// co in this block's kCoBlock channels; one thread per t
__global__ void conv_fwd_kernel(const float *__restrict__ x, int Ci, int L, int K,
                                const __nv_bfloat16 *__restrict__ w, const float *__restrict__ bias, int Co,
                                float *__restrict__ y)
{
    extern __shared__ float smc[];
    const int b = blockIdx.x, co0 = blockIdx.y * kCoBlock, p = K / 2;
    float *xs = smc;
    float *ws = smc + Ci * (L + 2 * p);  // [kCoBlock][Ci][K]
    load_halo(x + (size_t)b * Ci * L, Ci, L, p, xs);
    for (int e = threadIdx.x; e < kCoBlock * Ci * K; e += blockDim.x)
        ws[e] = __bfloat162float(w[(size_t)co0 * Ci * K + e]);
    __syncthreads();
    const int t = threadIdx.x;
    if (t >= L)
        return;
    float acc[kCoBlock];
#pragma unroll
    for (int j = 0; j < kCoBlock; ++j)
        acc[j] = bias[co0 + j];
    for (int ci = 0; ci < Ci; ++ci) {
        const float *xr = xs + ci * (L + 2 * p) + t;
        for (int k = 0; k < K; ++k) {
            const float xv = xr[k];
#pragma unroll
            for (int j = 0; j < kCoBlock; ++j)
                acc[j] = fmaf(ws[(j * Ci + ci) * K + k], xv, acc[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < kCoBlock; ++j)
        y[((size_t)b * Co + co0 + j) * L + t] = fmaxf(acc[j], 0.f);
}

// dx[b][ci][s] = (a[b][ci][s] > 0) * sum_co sum_k w[co][ci][k] g[b][co][s + p - k],
// ci in this block's kCoBlock input channels; one thread per s
__global__ void conv_bwd_data_kernel(const float *__restrict__ g, int Co, int L, int K,
                                     const __nv_bfloat16 *__restrict__ w, int Ci, const float *__restrict__ a,
                                     float *__restrict__ dx)
{
    extern __shared__ float smc[];
    const int b = blockIdx.x, ci0 = blockIdx.y * kCoBlock, p = K / 2;
    float *gs = smc;
    float *ws = smc + Co * (L + 2 * p);  // [kCoBlock][Co][K]
    load_halo(g + (size_t)b * Co * L, Co, L, p, gs);
    for (int e = threadIdx.x; e < kCoBlock * Co * K; e += blockDim.x) {
        const int j = e / (Co * K), r = e - j * Co * K, co = r / K, k = r - co * K;
        ws[e] = __bfloat162float(w[((size_t)co * Ci + ci0 + j) * K + k]);
    }
    __syncthreads();
    const int s = threadIdx.x;
    if (s >= L)
        return;
    float acc[kCoBlock];
#pragma unroll
    for (int j = 0; j < kCoBlock; ++j)
        acc[j] = 0.f;
    for (int co = 0; co < Co; ++co) {
        // g[s + p - k] = gs[co][s + 2p - k]
        const float *gr = gs + co * (L + 2 * p) + s + 2 * p;
        for (int k = 0; k < K; ++k) {
            const float gv = gr[-k];
#pragma unroll
            for (int j = 0; j < kCoBlock; ++j)
                acc[j] = fmaf(ws[(j * Co + co) * K + k], gv, acc[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < kCoBlock; ++j) {
        const size_t i = ((size_t)b * Ci + ci0 + j) * L + s;
        dx[i] = a[i] > 0.f ? acc[j] : 0.f;
    }
}

// dw[co][ci][k] = sum_b sum_t g[b][co][t] a[b][ci][t + k - p]; with ci == 0
// also db[co] = sum_b sum_t g[b][co][t].  One block per (co, ci); each thread
// sums its phases over the batch, then a fixed tree over the threads.
__global__ void conv_bwd_weight_kernel(const float *__restrict__ g, int Co, const float *__restrict__ a, int Ci,
                                       int B, int L, int K, float *__restrict__ dw, float *__restrict__ db)
{
    extern __shared__ float red[];  // [K + 1][blockDim.x]
    const int co = blockIdx.x, ci = blockIdx.y, p = K / 2;
    float acc[16];
    for (int k = 0; k <= K; ++k)
        acc[k] = 0.f;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        for (int b = 0; b < B; ++b) {
            const float gv = g[((size_t)b * Co + co) * L + t];
            const float *ar = a + ((size_t)b * Ci + ci) * L;
            for (int k = 0; k < K; ++k) {
                int s = t + k - p;
                s += s < 0 ? L : 0;
                s -= s >= L ? L : 0;
                acc[k] = fmaf(gv, ar[s], acc[k]);
            }
            acc[K] += gv;
        }
    }
    for (int k = 0; k <= K; ++k)
        red[k * blockDim.x + threadIdx.x] = acc[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
            for (int k = 0; k <= K; ++k)
                red[k * blockDim.x + threadIdx.x] += red[k * blockDim.x + threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k)
            dw[((size_t)co * Ci + ci) * K + k] = red[k * blockDim.x];
        if (ci == 0)
            db[co] = red[K * blockDim.x];
    }
}

// h[b][c] = mean over t of a[b][c][t]: warp w of the block takes channels
// w, w + warps, ...
__global__ void pool_kernel(const float *__restrict__ a, int C, int L, float *__restrict__ h)
{
    const int b = blockIdx.x, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int c = threadIdx.x >> 5; c < C; c += warps) {
        const float *r = a + ((size_t)b * C + c) * L;
        float s = 0.f;
        for (int t = lane; t < L; t += 32)
            s += r[t];
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
            h[b * C + c] = s / (float)L;
    }
}

// threads of the heads kernel: one per sample and per channel, whole warps
inline int head_threads(int B, int C)
{
    const int n = B > C ? B : C;
    return ((n + 31) / 32) * 32;
}
// power-of-two block of the weight-gradient reduction, <= min(L, 256)
inline int wgrad_threads(int L)
{
    int t = 32;
    while (2 * t <= L && 2 * t <= 256)
        t *= 2;
    return t;
}

struct HeadArgs {
    const float *h;                                  // [B][C]
    const __nv_bfloat16 *wd, *wr;                    // [C]
    const float *bd, *br;                            // [1]
    const float *label, *target;                     // [B] (training only)
    float *logit, *offset;                           // [B]
    float *dh;                                       // [B][C] (training only)
    float *gwd, *gbd, *gwr, *gbr;                    // head gradients (training only)
    float *loss;                                     // [1]
    int B, C;
    float dm_weight;
};

// Both heads, and with labels the loss and its gradients: one block, one
// thread per sample (B <= blockDim.x); sums in a fixed order.
__global__ void heads_kernel(HeadArgs a)
{
    extern __shared__ float hs[];  // [3][blockDim.x]: dlogit, doff, loss terms
    float *dl = hs, *dof = hs + blockDim.x, *lt = hs + 2 * blockDim.x;
    const int b = threadIdx.x;
    const bool train = a.label != nullptr;
    float lg = 0.f, of = 0.f, y = 0.f, err = 0.f;
    bool pos = false;
    if (b < a.B) {
        lg = *a.bd;
        of = *a.br;
        for (int c = 0; c < a.C; ++c) {
            const float hv = a.h[b * a.C + c];
            lg = fmaf(hv, __bfloat162float(a.wd[c]), lg);
            of = fmaf(hv, __bfloat162float(a.wr[c]), of);
        }
        a.logit[b] = lg;
        a.offset[b] = of;
        if (train) {
            y = a.label[b];
            pos = y > 0.5f;
            err = of - a.target[b];
        }
    }
    if (!train)
        return;
    // number of positive samples
    dof[b] = (b < a.B && pos) ? 1.f : 0.f;
    __syncthreads();
    if (b == 0) {
        float n = 0.f;
        for (int i = 0; i < a.B; ++i)
            n += dof[i];
        lt[0] = fmaxf(n, 1.f);
    }
    __syncthreads();
    const float npos = lt[0];
    __syncthreads();
    if (b < a.B) {
        const float sg = 1.f / (1.f + expf(-lg));
        dl[b] = (sg - y) / (float)a.B;
        dof[b] = pos ? a.dm_weight * 2.f * err / npos : 0.f;
        const float lo = fmaxf(lg, 0.f) - lg * y + log1pf(expf(-fabsf(lg)));
        lt[b] = lo / (float)a.B + (pos ? a.dm_weight * err * err / npos : 0.f);
        for (int c = 0; c < a.C; ++c)
            a.dh[b * a.C + c] = dl[b] * __bfloat162float(a.wd[c]) + dof[b] * __bfloat162float(a.wr[c]);
    }
    __syncthreads();
    if (b < a.C) {
        float gd = 0.f, gr = 0.f;
        for (int i = 0; i < a.B; ++i) {
            gd = fmaf(dl[i], a.h[i * a.C + b], gd);
            gr = fmaf(dof[i], a.h[i * a.C + b], gr);
        }
        a.gwd[b] = gd;
        a.gwr[b] = gr;
    }
    if (b == 0) {
        float sd = 0.f, sr = 0.f, l = 0.f;
        for (int i = 0; i < a.B; ++i) {
            sd += dl[i];
            sr += dof[i];
            l += lt[i];
        }
        *a.gbd = sd;
        *a.gbr = sr;
        *a.loss = l;
    }
}

// g[b][c][t] = (a[b][c][t] > 0) dh[b][c] / L  (the mean's and ReLU's backward)
__global__ void pool_bwd_kernel(const float *__restrict__ dh, const float *__restrict__ a, int C, int L, long long n,
                                float *__restrict__ g)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const long long bc = i / L;
    g[i] = a[i] > 0.f ? dh[bc] / (float)L : 0.f;
}

// Adam on the FP32 parameters, then their bf16 copy
__global__ void adam_kernel(float *__restrict__ th, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, __nv_bfloat16 *__restrict__ q, long long n, float lr, float b1,
                            float b2, float c1, float c2, float eps)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float t = th[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    th[i] = t;
    q[i] = __float2bfloat16_rn(t);
}

__global__ void quantise_kernel(const float *__restrict__ th, __nv_bfloat16 *__restrict__ q, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        q[i] = __float2bfloat16_rn(th[i]);
}

inline unsigned nblocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

msosm_status cfail(msosm_status s, const std::string &m)
{
    set_error_message(m.c_str());
    return s;
}

msosm_status ccuda(cudaError_t e, const char *what)
{
    cudaGetLastError();
    return cfail(e == cudaErrorMemoryAllocation ? MSOSM_ERR_OOM : MSOSM_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

bool on_device(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace

struct msosm_cnn {
    msosm_cnn_config cfg{};
    long long n = 0;                 // parameters
    std::vector<long long> w_off, b_off;  // per layer; then the heads at hd..
    long long wd_off = 0, bd_off = 0, wr_off = 0, br_off = 0;
    float *th = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *q = nullptr;
    std::vector<float *> act;        // act[1..layers]: [max_batch][C][L]
    float *xin = nullptr, *lab = nullptr, *tgt = nullptr;  // staged host inputs
    float *g0 = nullptr, *g1 = nullptr;  // gradient ping-pong [max_batch][max(Cin, C)][L]
    float *h = nullptr, *dh = nullptr, *logit = nullptr, *off = nullptr, *loss = nullptr;
    cudaStream_t st = nullptr;
    long long steps = 0;
    size_t smem_max = 0;

    void release()
    {
        float *fs[] = {th, grad, m, v, xin, lab, tgt, g0, g1, h, dh, logit, off, loss};
        for (float *p : fs)
            if (p)
                cudaFree(p);
        for (float *p : act)
            if (p)
                cudaFree(p);
        if (q)
            cudaFree(q);
        if (st)
            cudaStreamDestroy(st);
    }
};

namespace {

cudaError_t conv_forward(msosm_cnn *c, const float *x, int B)
{
    const msosm_cnn_config &g = c->cfg;
    const float *in = x;
    int ci = g.in_channels;
    for (int l = 0; l < g.layers; ++l) {
        const size_t sm = sizeof(float) * ((size_t)ci * (g.length + g.kernel - 1) + (size_t)kCoBlock * ci * g.kernel);
        conv_fwd_kernel<<<dim3(B, g.channels / kCoBlock), g.length, sm, c->st>>>(
            in, ci, g.length, g.kernel, c->q + c->w_off[l], c->th + c->b_off[l], g.channels, c->act[l + 1]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return e;
        in = c->act[l + 1];
        ci = g.channels;
    }
    pool_kernel<<<B, 32 * (g.channels < 32 ? g.channels : 32), 0, c->st>>>(c->act[g.layers], g.channels, g.length,
                                                                           c->h);
    return cudaGetLastError();
}

HeadArgs head_args(msosm_cnn *c, int B)
{
    HeadArgs a{};
    a.h = c->h;
    a.wd = c->q + c->wd_off;
    a.wr = c->q + c->wr_off;
    a.bd = c->th + c->bd_off;
    a.br = c->th + c->br_off;
    a.logit = c->logit;
    a.offset = c->off;
    a.B = B;
    a.C = c->cfg.channels;
    a.dm_weight = c->cfg.dm_weight;
    return a;
}

// device copy of a [n] float input (host or device pointer)
const float *stage(msosm_cnn *c, const float *src, float *buf, size_t n, cudaError_t &e)
{
    if (on_device(src))
        return src;
    e = cudaMemcpyAsync(buf, src, sizeof(float) * n, cudaMemcpyHostToDevice, c->st);
    return buf;
}

msosm_status check_batch(const msosm_cnn *c, int B)
{
    if (!c)
        return cfail(MSOSM_ERR_BAD_ARG, "null network");
    if (B < 1 || B > c->cfg.max_batch)
        return cfail(MSOSM_ERR_BAD_ARG, "batch must be 1 .. max_batch");
    return MSOSM_OK;
}

}  // namespace

extern "C" {

msosm_status msosm_cnn_create(const msosm_cnn_config *cfg, unsigned long long seed, msosm_cnn **out)
{
    if (!cfg || !out)
        return cfail(MSOSM_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    const msosm_cnn_config &g = *cfg;
    if (g.in_channels < 1 || g.in_channels > 256 || g.length < 32 || g.length > 1024 || g.length % 32 != 0 ||
        g.channels < kCoBlock || g.channels > 256 || g.channels % kCoBlock != 0 || g.in_channels % kCoBlock != 0 ||
        g.kernel < 1 || g.kernel > 15 || g.kernel % 2 == 0 || g.kernel > g.length || g.layers < 1 ||
        g.layers > 16 || g.max_batch < 1 || g.max_batch > 1024 || !(g.dm_weight >= 0.f))
        return cfail(MSOSM_ERR_BAD_ARG,
                     "cnn: in_channels and channels multiples of 8 (<= 256), length a multiple of 32 in 32 .. 1024, "
                     "odd kernel <= 15, 1 .. 16 layers, max_batch 1 .. 1024, dm_weight >= 0");
    // shared memory of the widest convolution step
    const int cmax = g.in_channels > g.channels ? g.in_channels : g.channels;
    const size_t sm = sizeof(float) * ((size_t)cmax * (g.length + g.kernel - 1) + (size_t)kCoBlock * cmax * g.kernel);
    if (sm > 200 * 1024)
        return cfail(MSOSM_ERR_UNSUPPORTED, "cnn: channels x length too large for one block's shared memory");
    if (msosm_device_count() == 0)
        return cfail(MSOSM_ERR_NO_DEVICE, "no CUDA device");
    msosm_cnn *c = new (std::nothrow) msosm_cnn;
    if (!c)
        return cfail(MSOSM_ERR_OOM, "host allocation");
    c->cfg = g;
    c->smem_max = sm;
    long long o = 0;
    int ci = g.in_channels;
    for (int l = 0; l < g.layers; ++l) {
        c->w_off.push_back(o);
        o += (long long)g.channels * ci * g.kernel;
        c->b_off.push_back(o);
        o += g.channels;
        ci = g.channels;
    }
    c->wd_off = o;
    o += g.channels;
    c->bd_off = o;
    o += 1;
    c->wr_off = o;
    o += g.channels;
    c->br_off = o;
    o += 1;
    c->n = o;
    // He-uniform initial weights (fan-in), zero biases, from a seeded engine
    std::vector<float> init((size_t)o, 0.f);
    std::mt19937_64 rng(seed);
    ci = g.in_channels;
    for (int l = 0; l < g.layers; ++l) {
        const double lim = std::sqrt(6.0 / (double)(ci * g.kernel));
        std::uniform_real_distribution<double> u(-lim, lim);
        for (long long i = 0; i < (long long)g.channels * ci * g.kernel; ++i)
            init[(size_t)(c->w_off[l] + i)] = (float)u(rng);
        ci = g.channels;
    }
    {
        const double lim = std::sqrt(3.0 / (double)g.channels);
        std::uniform_real_distribution<double> u(-lim, lim);
        for (int i = 0; i < g.channels; ++i) {
            init[(size_t)(c->wd_off + i)] = (float)u(rng);
            init[(size_t)(c->wr_off + i)] = (float)u(rng);
        }
    }
    const size_t B = (size_t)g.max_batch, L = (size_t)g.length;
    const size_t gmax = B * (size_t)cmax * L;
    cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    auto al = [&](float **p, size_t count) {
        if (e == cudaSuccess)
            e = cudaMalloc((void **)p, sizeof(float) * count + 16);
    };
    al(&c->th, (size_t)o);
    al(&c->grad, (size_t)o);
    al(&c->m, (size_t)o);
    al(&c->v, (size_t)o);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&c->q, sizeof(__nv_bfloat16) * (size_t)o + 16);
    c->act.assign(g.layers + 1, nullptr);
    for (int l = 1; l <= g.layers; ++l)
        al(&c->act[l], B * g.channels * L);
    al(&c->xin, B * (size_t)g.in_channels * L);
    al(&c->lab, B);
    al(&c->tgt, B);
    al(&c->g0, gmax);
    al(&c->g1, gmax);
    al(&c->h, B * g.channels);
    al(&c->dh, B * g.channels);
    al(&c->logit, B);
    al(&c->off, B);
    al(&c->loss, 1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(conv_bwd_data_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) {
        msosm_status s = ccuda(e, "msosm_cnn_create");
        c->release();
        delete c;
        return s;
    }
    *out = c;
    msosm_status s = msosm_cnn_set_params(c, init.data());
    if (s != MSOSM_OK) {
        c->release();
        delete c;
        *out = nullptr;
    }
    return s;
}

msosm_status msosm_cnn_destroy(msosm_cnn *c)
{
    if (c) {
        if (c->st)
            cudaStreamSynchronize(c->st);
        c->release();
        delete c;
    }
    return MSOSM_OK;
}

msosm_status msosm_cnn_param_count(const msosm_cnn *c, size_t *count)
{
    if (!c || !count)
        return cfail(MSOSM_ERR_BAD_ARG, "null argument");
    *count = (size_t)c->n;
    return MSOSM_OK;
}

msosm_status msosm_cnn_get_params(msosm_cnn *c, float *params)
{
    if (!c || !params)
        return cfail(MSOSM_ERR_BAD_ARG, "null argument");
    cudaError_t e = cudaMemcpyAsync(params, c->th, sizeof(float) * c->n, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(c->st);
    return e == cudaSuccess ? MSOSM_OK : ccuda(e, "msosm_cnn_get_params");
}

msosm_status msosm_cnn_set_params(msosm_cnn *c, const float *params)
{
    if (!c || !params)
        return cfail(MSOSM_ERR_BAD_ARG, "null argument");
    cudaError_t e = cudaMemcpyAsync(c->th, params, sizeof(float) * c->n, cudaMemcpyDefault, c->st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(c->m, 0, sizeof(float) * c->n, c->st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(c->v, 0, sizeof(float) * c->n, c->st);
    if (e == cudaSuccess) {
        quantise_kernel<<<nblocks(c->n, 256), 256, 0, c->st>>>(c->th, c->q, c->n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(c->st);
    c->steps = 0;
    return e == cudaSuccess ? MSOSM_OK : ccuda(e, "msosm_cnn_set_params");
}

msosm_status msosm_cnn_forward(msosm_cnn *c, const float *x, int batch, float *logit, float *offset)
{
    msosm_status s = check_batch(c, batch);
    if (s != MSOSM_OK)
        return s;
    if (!x || !logit || !offset)
        return cfail(MSOSM_ERR_BAD_ARG, "null argument");
    cudaError_t e = cudaSuccess;
    const float *xd = stage(c, x, c->xin, (size_t)batch * c->cfg.in_channels * c->cfg.length, e);
    if (e == cudaSuccess)
        e = conv_forward(c, xd, batch);
    if (e == cudaSuccess) {
        HeadArgs a = head_args(c, batch);
        const int tb = head_threads(batch, c->cfg.channels);
        heads_kernel<<<1, tb, 3 * sizeof(float) * tb, c->st>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(logit, c->logit, sizeof(float) * batch, cudaMemcpyDefault, c->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(offset, c->off, sizeof(float) * batch, cudaMemcpyDefault, c->st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(c->st);
    return e == cudaSuccess ? MSOSM_OK : ccuda(e, "msosm_cnn_forward");
}

msosm_status msosm_cnn_gradient(msosm_cnn *c, const float *x, const float *label, const float *target, int batch,
                                float *loss, float *grad)
{
    msosm_status s = check_batch(c, batch);
    if (s != MSOSM_OK)
        return s;
    if (!x || !label || !target)
        return cfail(MSOSM_ERR_BAD_ARG, "null argument");
    const msosm_cnn_config &g = c->cfg;
    const int L = g.length, C = g.channels, K = g.kernel;
    cudaError_t e = cudaSuccess;
    const float *xd = stage(c, x, c->xin, (size_t)batch * g.in_channels * L, e);
    const float *ld = e == cudaSuccess ? stage(c, label, c->lab, batch, e) : nullptr;
    const float *td = e == cudaSuccess ? stage(c, target, c->tgt, batch, e) : nullptr;
    if (e == cudaSuccess)
        e = conv_forward(c, xd, batch);
    if (e == cudaSuccess) {
        HeadArgs a = head_args(c, batch);
        a.label = ld;
        a.target = td;
        a.dh = c->dh;
        a.gwd = c->grad + c->wd_off;
        a.gbd = c->grad + c->bd_off;
        a.gwr = c->grad + c->wr_off;
        a.gbr = c->grad + c->br_off;
        a.loss = c->loss;
        const int tb = head_threads(batch, C);
        heads_kernel<<<1, tb, 3 * sizeof(float) * tb, c->st>>>(a);
        e = cudaGetLastError();
    }
    float *gcur = c->g0, *gnext = c->g1;
    if (e == cudaSuccess) {
        const long long n = (long long)batch * C * L;
        pool_bwd_kernel<<<nblocks(n, 256), 256, 0, c->st>>>(c->dh, c->act[g.layers], C, L, n, gcur);
        e = cudaGetLastError();
    }
    for (int l = g.layers - 1; l >= 0 && e == cudaSuccess; --l) {
        const int ci = l == 0 ? g.in_channels : C;
        const float *a_in = l == 0 ? xd : c->act[l];
        const int tpb = wgrad_threads(L);
        conv_bwd_weight_kernel<<<dim3(C, ci), tpb, sizeof(float) * (K + 1) * tpb, c->st>>>(
            gcur, C, a_in, ci, batch, L, K, c->grad + c->w_off[l], c->grad + c->b_off[l]);
        e = cudaGetLastError();
        if (e == cudaSuccess && l > 0) {
            const size_t sm = sizeof(float) * ((size_t)C * (L + K - 1) + (size_t)kCoBlock * C * K);
            conv_bwd_data_kernel<<<dim3(batch, ci / kCoBlock), L, sm, c->st>>>(gcur, C, L, K, c->q + c->w_off[l],
                                                                              ci, c->act[l], gnext);
            e = cudaGetLastError();
            float *t = gcur;
            gcur = gnext;
            gnext = t;
        }
    }
    if (e == cudaSuccess && loss)
        e = cudaMemcpyAsync(loss, c->loss, sizeof(float), cudaMemcpyDefault, c->st);
    if (e == cudaSuccess && grad)
        e = cudaMemcpyAsync(grad, c->grad, sizeof(float) * c->n, cudaMemcpyDefault, c->st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(c->st);
    return e == cudaSuccess ? MSOSM_OK : ccuda(e, "msosm_cnn_gradient");
}

msosm_status msosm_cnn_adam_step(msosm_cnn *c, float lr)
{
    if (!c || !(lr > 0.f))
        return cfail(MSOSM_ERR_BAD_ARG, "null network or learning rate <= 0");
    c->steps += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - (float)std::pow((double)b1, (double)c->steps);
    const float c2 = 1.f - (float)std::pow((double)b2, (double)c->steps);
    adam_kernel<<<nblocks(c->n, 256), 256, 0, c->st>>>(c->th, c->grad, c->m, c->v, c->q, c->n, lr, b1, b2, c1, c2,
                                                       eps);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(c->st);
    return e == cudaSuccess ? MSOSM_OK : ccuda(e, "msosm_cnn_adam_step");
}

}  // extern "C"
