/*
 * orc.c -- CPU FP64 restatement of the msosm_gpu coherent-dedispersion path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Loaded by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg; never by the
 * product library.  See orc.h for the reference file:line of each function.
 *
 * Build with -ffp-contract=off and without -ffast-math: the float/double
 * promotion sequence of the reference decides integer results (Nd, M,
 * delaycount, delay_points, fold period boundaries) and is reproduced
 * operation by operation below.
 */
#include "orc.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* reference: `constexpr auto pi = M_PI;` (utils/include/globals.h:29) and
 * `kdm = 4.15 * 1e15;` stored in a float member (msosm_prepare.cpp:6). */
static const double REF_PI = M_PI;
static float ref_kdm(void) { return (float)(4.15 * 1e15); }

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* filter design / segmentation                                              */
/* ------------------------------------------------------------------------ */

unsigned long orc_nd(float bw, float dm, float f0)
{
    /* msosm_prepare.cpp:5-8:
     *   fs = bw;  kdm (float) * dm (float) is a float product;
     *   pow(f0,2) promotes to double; (f0 + bw) is a float sum;
     *   (1 / fs) is a float quotient. */
    float fs = bw;
    float kdm = ref_kdm();
    float kd = kdm * dm;
    float f1 = f0 + bw;
    double a = 1.0 / pow((double)f0, 2.0);
    double b = 1.0 / pow((double)f1, 2.0);
    float inv_fs = 1.0f / fs;
    double v = floor((double)kd * (a - b) / (double)inv_fs);
    if (!(v > 0.0))
        return 0;
    return (unsigned long)v;
}

unsigned long orc_msosm_min_order(unsigned long Nd)
{
    /* msosm_prepare.cpp:21-23 */
    if (Nd == 0)
        return 0;
    double order = 2 * sqrt((double)Nd);
    return (unsigned long)pow(2.0, ceil(log2(order)));
}

static int ref_next_power_of_2(int n)
{
    /* osm_prepare.cpp:86-99 */
    if (n <= 0)
        return 1;
    --n;
    n |= n >> 1;
    n |= n >> 2;
    n |= n >> 4;
    n |= n >> 8;
    n |= n >> 16;
    return n + 1;
}

unsigned long orc_osm_min_order(unsigned long Nd)
{
    /* osm_prepare.cpp:21-24: int order = next_power_of_2(Nd); M = 2 * order */
    int order = ref_next_power_of_2((int)Nd);
    return 2ul * (unsigned long)order;
}

int orc_delaycount(unsigned long Nd, unsigned long M)
{
    /* msosm_prepare.cpp:88: ceil(Nd / static_cast<float>(M)) -- float quotient */
    if (M == 0)
        return 0;
    float q = (float)Nd / (float)M;
    return (int)ceilf(q);
}

int orc_segmentation(float bw, float dm, float f0, unsigned long Nd,
                     unsigned long M, int *delay_points)
{
    const unsigned long N = 2 * M;
    int dc = orc_delaycount(Nd, M);
    for (unsigned long k = 0; k < N; k++)
        delay_points[k] = 0;
    if (dc <= 0)
        return dc < 0 ? 0 : dc;

    float fs = bw;
    float kdm = ref_kdm();
    float w0 = (float)(2 * REF_PI * f0);
    float *w = (float *)malloc(sizeof(float) * (size_t)(dc + 1));
    w[0] = -1;
    w[dc] = 1;
    int pos_index = 1;
    for (int j = 1; j < dc; j++) {
        /* msosm_prepare.cpp:102:
         * (sqrt(1/(1/pow(w0,2) - j*M/fs/(4*pi*pi*kdm*dm))) - w0 - pi*fs)/pi/fs
         * j*M is an unsigned long; dividing by the float fs is a float
         * quotient; the rest is double. */
        double inv_w02 = 1.0 / pow((double)w0, 2.0);
        float jm_fs = (float)((unsigned long)j * M) / fs;
        double c = 4 * REF_PI * REF_PI * (double)kdm * (double)dm;
        double t = (double)jm_fs / c;
        double s = sqrt(1.0 / (inv_w02 - t));
        double num = s - (double)w0 - REF_PI * (double)fs;
        w[j] = (float)(num / REF_PI / (double)fs);
        if (w[j] < 0)
            pos_index = j + 1;
    }
    int negcount = pos_index;
    int poscount = dc - pos_index + 1;
    unsigned long *segneg = (unsigned long *)malloc(sizeof(unsigned long) * (size_t)(negcount + 1));
    unsigned long *segpos = (unsigned long *)malloc(sizeof(unsigned long) * (size_t)(poscount + 1));
    /* :112-121: float arithmetic (w[j] + 2) * M and w[j] * M, floor of a float */
    for (int j = 0; j < negcount; j++)
        segneg[j] = (unsigned long)floorf((w[j] + 2.0f) * (float)M);
    segneg[negcount] = N;
    segpos[0] = 0;
    for (int j = 0; j < poscount; j++)
        segpos[j + 1] = (unsigned long)floorf(w[j + negcount] * (float)M);
    /* :122-129 delays; :133-147 fill (negative segments first, then positive) */
    for (int j = 0; j < negcount; j++)
        for (unsigned long k = segneg[j]; k < segneg[j + 1] && k < N; k++)
            delay_points[k] = j;
    for (int j = 0; j < poscount; j++)
        for (unsigned long k = segpos[j]; k < segpos[j + 1] && k < N; k++)
            delay_points[k] = (negcount - 1) + j;
    free(w);
    free(segneg);
    free(segpos);
    return dc;
}

static float chirp_w(float fs, unsigned long order, unsigned long i)
{
    /* msosm_prepare.cpp:42,52-53 (and :59-60):
     *   float step = 2*pi*fs/M;                 (double quotient -> float)
     *   w[i] = -pi*fs + step*i;                 (step*i is a float product)
     *   w[i] = w[i] + pi*fs;                    (double sum -> float) */
    float step = (float)(2 * REF_PI * (double)fs / (double)order);
    float si = step * (float)i;
    float wi = (float)(-REF_PI * (double)fs + (double)si);
    wi = (float)((double)wi + REF_PI * (double)fs);
    return wi;
}

static double chirp_phase_w(float wi, float kdm, float dm, float w0)
{
    /* msosm_prepare.cpp:54: 4*pi*pi*kdm*dm*w*w/(w + w0)/w0/w0, left to right,
     * (w + w0) being a float sum. */
    float den = wi + w0;
    double p = 4 * REF_PI;
    p = p * REF_PI;
    p = p * (double)kdm;
    p = p * (double)dm;
    p = p * (double)wi;
    p = p * (double)wi;
    p = p / (double)den;
    p = p / (double)w0;
    p = p / (double)w0;
    return p;
}

double orc_chirp_phase(float bw, float dm, float f0, unsigned long M, unsigned long i)
{
    float w0 = (float)(2 * REF_PI * f0);
    return chirp_phase_w(chirp_w(bw, M, i), ref_kdm(), dm, w0);
}

/* ------------------------------------------------------------------------ */
/* FFT                                                                       */
/* ------------------------------------------------------------------------ */

static pthread_mutex_t tw_lock = PTHREAD_MUTEX_INITIALIZER;
static double *tw_cache[48];

static const double *twiddles(int log2n)
{
    pthread_mutex_lock(&tw_lock);
    if (!tw_cache[log2n]) {
        unsigned long n = 1ul << log2n;
        double *t = (double *)malloc(sizeof(double) * 2 * (n / 2 + 1));
        for (unsigned long k = 0; k <= n / 2; k++) {
            double a = -2.0 * M_PI * (double)k / (double)n;
            t[2 * k] = cos(a);
            t[2 * k + 1] = sin(a);
        }
        tw_cache[log2n] = t;
    }
    const double *r = tw_cache[log2n];
    pthread_mutex_unlock(&tw_lock);
    return r;
}

void orc_fft(double *x, unsigned long n, int sign)
{
    if (n < 2)
        return;
    int log2n = 0;
    while ((1ul << log2n) < n)
        log2n++;
    /* bit reversal */
    for (unsigned long i = 1, j = 0; i < n; i++) {
        unsigned long bit = n >> 1;
        for (; j & bit; bit >>= 1)
            j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = x[2 * i], ti = x[2 * i + 1];
            x[2 * i] = x[2 * j];
            x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = tr;
            x[2 * j + 1] = ti;
        }
    }
    const double *tw = twiddles(log2n);
    for (unsigned long len = 2; len <= n; len <<= 1) {
        unsigned long half = len >> 1;
        unsigned long stride = n / len;
        for (unsigned long i = 0; i < n; i += len) {
            for (unsigned long k = 0; k < half; k++) {
                double wr = tw[2 * k * stride];
                double wi = tw[2 * k * stride + 1];
                if (sign > 0)
                    wi = -wi;
                double *a = x + 2 * (i + k);
                double *b = x + 2 * (i + k + half);
                double br = b[0] * wr - b[1] * wi;
                double bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br;
                b[1] = a[1] - bi;
                a[0] += br;
                a[1] += bi;
            }
        }
    }
}

void orc_dedisp_params(float bw, float dm, float f0, unsigned long M, int sign, double *H)
{
    const unsigned long N = 2 * M;
    float fs = bw;
    float kdm = ref_kdm();
    float w0 = (float)(2 * REF_PI * f0);
    double *h = (double *)calloc(2 * M, sizeof(double));
    for (unsigned long i = 0; i < M; i++) {
        float wi = chirp_w(fs, M, i);
        double ph = chirp_phase_w(wi, kdm, dm, w0);
        /* :50-63: offsets [0, M/2) go to h[M/2 + i], [M/2, M) to h[i - M/2] */
        unsigned long j = (i < M / 2) ? (M / 2 + i) : (i - M / 2);
        h[2 * j] = cos(ph);
        h[2 * j + 1] = (sign < 0) ? -sin(ph) : sin(ph);
    }
    /* :65-74: unnormalised backward M-point DFT; the /M result is discarded */
    orc_fft(h, M, +1);
    memset(H, 0, sizeof(double) * 2 * N);
    memcpy(H, h, sizeof(double) * 2 * M);
    /* :78-81: zero-pad to 2M and forward DFT */
    orc_fft(H, N, -1);
    free(h);
}

/* ------------------------------------------------------------------------ */
/* codecs                                                                    */
/* ------------------------------------------------------------------------ */

void orc_decode_uint16(const uint16_t *src, size_t n_pairs, double *dst)
{
    for (size_t i = 0; i < 2 * n_pairs; i++)
        dst[i] = src[i] == 0 ? 0.0 : (double)src[i] - 32768.0;
}

void orc_encode_uint16(const double *src, size_t n_pairs, uint16_t *dst)
{
    for (size_t i = 0; i < 2 * n_pairs; i++) {
        float v = (float)src[i];
        float u = v + 32768.0f * (v != 0.0f ? 1.0f : 0.0f);
        if (!(u > 0.0f))
            u = 0.0f;
        if (u > 65535.0f)
            u = 65535.0f;
        dst[i] = (uint16_t)u;
    }
}

/* ------------------------------------------------------------------------ */
/* streaming dedispersion                                                    */
/* ------------------------------------------------------------------------ */

struct orc_dedisp {
    int D, count, osm, S, idx, nthreads;
    unsigned long M, N;
    unsigned long *Nd;
    int *dc;
    int *delays;   /* D x N */
    double *H;     /* D x N complex */
    double *inbuf; /* (count+1) x M complex */
    double *X;     /* count x N complex */
    double *ring;  /* MS-OSM: D x S x N complex (reference: per-DM product ring) */
};

orc_dedisp *orc_dedisp_create(const float *bw, const float *dm, const float *f0,
                              int numDMs, unsigned long fftpoint, int count,
                              unsigned long input_size, int osm, int nthreads)
{
    if (numDMs < 1 || count < 0)
        return NULL;
    orc_dedisp *d = (orc_dedisp *)calloc(1, sizeof(orc_dedisp));
    d->D = numDMs;
    d->osm = osm;
    d->nthreads = nthreads;
    d->Nd = (unsigned long *)calloc((size_t)numDMs, sizeof(unsigned long));
    d->dc = (int *)calloc((size_t)numDMs, sizeof(int));
    /* msosm_prepare_dm_concurrent.cpp:31-49 (calculate_min_order), then
     * msosm_gpu_dm_concurrent.cpp:29-42 (fftpoint override, input_size) */
    unsigned long Mc = 0;
    for (int i = 0; i < numDMs; i++) {
        d->Nd[i] = orc_nd(bw[i], dm[i], f0[i]);
        unsigned long m = osm ? orc_osm_min_order(d->Nd[i]) : orc_msosm_min_order(d->Nd[i]);
        if (m > Mc)
            Mc = m;
    }
    unsigned long M = Mc;
    if (fftpoint != 0) {
        M = fftpoint / 2;
        if (M < Mc)
            M = Mc;
    }
    if (M < 1) {
        free(d->Nd);
        free(d->dc);
        free(d);
        return NULL;
    }
    if (input_size != 0)
        count = (int)(input_size / M);
    if (count < 1)
        count = 1;
    d->M = M;
    d->N = 2 * M;
    d->count = count;
    const unsigned long N = d->N;
    d->delays = (int *)calloc((size_t)numDMs * N, sizeof(int));
    d->H = (double *)malloc(sizeof(double) * 2 * N * (size_t)numDMs);
    int S = 0;
    for (int i = 0; i < numDMs; i++) {
        if (!osm)
            d->dc[i] = orc_segmentation(bw[i], dm[i], f0[i], d->Nd[i], M, d->delays + (size_t)i * N);
        orc_dedisp_params(bw[i], dm[i], f0[i], M, -1, d->H + (size_t)i * 2 * N);
        /* msosm_gpu_dm_concurrent.cpp:90-98 */
        int dbs = d->dc[i] + count - 1;
        if (dbs % count != 0)
            dbs += count - dbs % count;
        if (dbs > S)
            S = dbs;
    }
    if (S < count)
        S = count;
    d->S = S;
    d->inbuf = (double *)calloc(2 * (size_t)(count + 1) * M, sizeof(double));
    d->X = (double *)calloc(2 * (size_t)count * N, sizeof(double));
    if (!osm)
        d->ring = (double *)calloc(2 * (size_t)numDMs * (size_t)S * N, sizeof(double));
    return d;
}

void orc_dedisp_destroy(orc_dedisp *d)
{
    if (!d)
        return;
    free(d->Nd);
    free(d->dc);
    free(d->delays);
    free(d->H);
    free(d->inbuf);
    free(d->X);
    free(d->ring);
    free(d);
}

unsigned long orc_dedisp_M(const orc_dedisp *d) { return d->M; }
int orc_dedisp_count(const orc_dedisp *d) { return d->count; }
int orc_dedisp_ring_slots(const orc_dedisp *d) { return d->S; }
int orc_dedisp_delaycount(const orc_dedisp *d, int i) { return d->dc[i]; }
unsigned long orc_dedisp_Nd(const orc_dedisp *d, int i) { return d->Nd[i]; }

void orc_dedisp_filter(orc_dedisp *d, const double *in, double *out)
{
    const unsigned long M = d->M, N = d->N;
    const int count = d->count, D = d->D, S = d->S;
    const double invN = 1.0 / (double)N;
    int nt = d->nthreads > 0 ? d->nthreads : orc_get_threads();
    (void)nt;
    /* :123-127 history copy + decode into inbuf[M ...] */
    memmove(d->inbuf, d->inbuf + 2 * (size_t)count * M, sizeof(double) * 2 * M);
    memcpy(d->inbuf + 2 * M, in, sizeof(double) * 2 * (size_t)count * M);
    /* :129 forward FFTs of count windows, hop M */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int c = 0; c < count; c++) {
        double *x = d->X + 2 * (size_t)c * N;
        memcpy(x, d->inbuf + 2 * (size_t)c * M, sizeof(double) * 2 * N);
        orc_fft(x, N, -1);
    }
#pragma omp parallel for num_threads(nt) schedule(dynamic)
    for (int i = 0; i < D; i++) {
        const double *H = d->H + (size_t)i * 2 * N;
        double *y = (double *)malloc(sizeof(double) * 2 * N);
        for (int c = 0; c < count; c++) {
            const double *x = d->X + 2 * (size_t)c * N;
            if (d->osm) {
                /* gpu_kernel.cu:56-66: (a/N) * H */
                for (unsigned long n = 0; n < N; n++) {
                    double ar = x[2 * n] * invN, ai = x[2 * n + 1] * invN;
                    y[2 * n] = ar * H[2 * n] - ai * H[2 * n + 1];
                    y[2 * n + 1] = ar * H[2 * n + 1] + ai * H[2 * n];
                }
            } else {
                /* gpu_kernel.cu:174-196: product to slot (index + c + delay) % S */
                const int *dl = d->delays + (size_t)i * N;
                double *ring = d->ring + (size_t)i * 2 * (size_t)S * N;
                for (unsigned long n = 0; n < N; n++) {
                    int j = (d->idx + c + dl[n]) % S;
                    double *dst = ring + 2 * ((size_t)j * N + n);
                    double ar = x[2 * n], ai = x[2 * n + 1];
                    dst[0] = (ar * H[2 * n] - ai * H[2 * n + 1]) * invN;
                    dst[1] = (ar * H[2 * n + 1] + ai * H[2 * n]) * invN;
                }
            }
            if (d->osm) {
                orc_fft(y, N, +1);
                double *o = out + 2 * ((size_t)i * count * M + (size_t)c * M);
                for (unsigned long m = 0; m < M; m++) {
                    o[2 * m] = y[2 * (M + m)] * invN;
                    o[2 * m + 1] = y[2 * (M + m) + 1] * invN;
                }
            }
        }
        if (!d->osm) {
            /* :140 inverse FFT of slots index .. index+count-1; :149-150 discard */
            double *ring = d->ring + (size_t)i * 2 * (size_t)S * N;
            for (int c = 0; c < count; c++) {
                memcpy(y, ring + 2 * (size_t)(d->idx + c) * N, sizeof(double) * 2 * N);
                orc_fft(y, N, +1);
                double *o = out + 2 * ((size_t)i * count * M + (size_t)c * M);
                for (unsigned long m = 0; m < M; m++) {
                    o[2 * m] = y[2 * (M + m)] * invN;
                    o[2 * m + 1] = y[2 * (M + m) + 1] * invN;
                }
            }
        }
        free(y);
    }
    if (!d->osm) {
        /* :142-146 */
        d->idx += count;
        if (d->idx >= S)
            d->idx -= S;
    }
}

/* ------------------------------------------------------------------------ */
/* detection + folding                                                       */
/* ------------------------------------------------------------------------ */

void orc_intensity(const double *a, const double *b, size_t n, double *out)
{
    for (size_t i = 0; i < n; i++) {
        double p = a[2 * i] * a[2 * i] + a[2 * i + 1] * a[2 * i + 1];
        if (b)
            p += b[2 * i] * b[2 * i] + b[2 * i + 1] * b[2 * i + 1];
        out[i] = sqrt(p);
    }
}

struct orc_fold {
    unsigned long size, ps, time_bin, current_index;
    float psf, diff, current_diff;
    int ready, discard_count, current_discard, accf;
    double *raw, *tmp;
    float *rawf, *tmpf;
};

orc_fold *orc_fold_create(float period, float fs, unsigned long size,
                          unsigned long time_bin, int accumulate_float)
{
    /* fold_gpu.cpp:3-27 */
    orc_fold *f = (orc_fold *)calloc(1, sizeof(orc_fold));
    f->size = size;
    f->psf = period * fs;
    f->ps = (unsigned long)f->psf;
    f->diff = f->psf - (float)f->ps;
    f->time_bin = (time_bin == (unsigned long)-1) ? f->ps : time_bin;
    f->accf = accumulate_float;
    f->raw = (double *)calloc(f->ps ? f->ps : 1, sizeof(double));
    f->tmp = (double *)calloc(f->ps ? f->ps : 1, sizeof(double));
    f->rawf = (float *)calloc(f->ps ? f->ps : 1, sizeof(float));
    f->tmpf = (float *)calloc(f->ps ? f->ps : 1, sizeof(float));
    return f;
}

void orc_fold_destroy(orc_fold *f)
{
    if (!f)
        return;
    free(f->raw);
    free(f->tmp);
    free(f->rawf);
    free(f->tmpf);
    free(f);
}

void orc_fold_discard_samples(orc_fold *f, unsigned long Nd)
{
    /* fold_gpu.cpp:29-33: ceil(Nd / period_samples_float), a float quotient */
    f->discard_count = (int)ceilf((float)Nd / f->psf);
    f->current_discard = 0;
}

unsigned long orc_fold_period_samples(const orc_fold *f) { return f->ps; }
unsigned long orc_fold_time_bin(const orc_fold *f) { return f->time_bin; }

static void fold_tmp(orc_fold *f, unsigned long at, double v)
{
    if (f->accf)
        f->tmpf[at] = (float)v;
    else
        f->tmp[at] = v;
}

static void fold_raw_add(orc_fold *f, unsigned long at, double v)
{
    if (f->accf)
        f->rawf[at] += (float)v;
    else
        f->raw[at] += v;
}

static void fold_count_period(orc_fold *f)
{
    if (!f->ready) {
        f->current_discard += 1;
        if (f->current_discard == f->discard_count) {
            f->ready = 1;
            f->current_discard = 0;
        }
    }
}

void orc_fold_data(orc_fold *f, const double *I)
{
    /* fold_gpu.cpp:48-173.  current_size is unsigned in the reference and a
     * skip at the very end of a chunk makes it wrap to -1; the first branch
     * (:98-109) then defers the skip to the next call without counting the
     * period towards the discard; the while loop (:124-152) would read past
     * the chunk instead.  Here both defer the skip; the while loop counts the
     * period first, as its code does before the wrap is reached. */
    const unsigned long ps = f->ps;
    unsigned long cs = f->size, ci = 0;
    if (ps == 0)
        return;
    if (f->current_diff > 1.0f) {
        f->current_diff -= 1.0f;
        ci += 1;
        cs -= 1;
        if (cs == 0)
            return;
    }
    if (f->current_index != 0) {
        if (cs < ps - f->current_index) {
            if (f->ready)
                for (unsigned long i = 0; i < cs; i++)
                    fold_tmp(f, f->current_index + i, I[ci + i]);
            f->current_index += cs;
            return;
        }
        if (f->ready) {
            for (unsigned long i = 0; i < ps - f->current_index; i++)
                fold_tmp(f, f->current_index + i, I[ci + i]);
            for (unsigned long i = 0; i < ps; i++) {
                if (f->accf)
                    f->rawf[i] += f->tmpf[i];
                else
                    f->raw[i] += f->tmp[i];
            }
        }
        cs -= ps - f->current_index;
        ci += ps - f->current_index;
        f->current_index = 0;
        f->current_diff += f->diff;
        if (f->current_diff > 1.0f) {
            f->current_diff -= 1.0f;
            ci += 1;
            if (cs == 0) {
                f->current_diff += 1.0f;
                return;
            }
            cs -= 1;
        }
        fold_count_period(f);
    }
    while (cs >= ps) {
        if (f->ready)
            for (unsigned long i = 0; i < ps; i++)
                fold_raw_add(f, i, I[ci + i]);
        cs -= ps;
        ci += ps;
        f->current_diff += f->diff;
        int wrap = 0;
        if (f->current_diff > 1.0f) {
            f->current_diff -= 1.0f;
            ci += 1;
            if (cs == 0)
                wrap = 1;
            else
                cs -= 1;
        }
        fold_count_period(f);
        if (wrap) {
            f->current_diff += 1.0f;
            return;
        }
    }
    if (cs > 0) {
        if (f->ready)
            for (unsigned long i = 0; i < cs; i++)
                fold_tmp(f, i, I[ci + i]);
        f->current_index = cs;
    }
}

void orc_fold_data_bins(orc_fold *f, double *out)
{
    /* fold_gpu.cpp:175-194 */
    if (f->time_bin == f->ps) {
        for (unsigned long i = 0; i < f->ps; i++)
            out[i] = f->accf ? (double)f->rawf[i] : f->raw[i];
        return;
    }
    int bpt = (int)(f->ps / f->time_bin);
    for (unsigned long i = 0; i < f->time_bin; i++) {
        if (f->accf) {
            float s = 0.0f;
            for (int j = 0; j < bpt; j++)
                s += f->rawf[i * (unsigned long)bpt + (unsigned long)j];
            out[i] = (double)(s / (float)bpt);
        } else {
            double s = 0.0;
            for (int j = 0; j < bpt; j++)
                s += f->raw[i * (unsigned long)bpt + (unsigned long)j];
            out[i] = s / (double)bpt;
        }
    }
}

size_t orc_fold_period_starts(float period, float fs, unsigned long total,
                              int64_t *start, size_t cap)
{
    /* the global view of fold_gpu.cpp:48-173 for one unbroken stream: period
     * p covers [start[p], start[p] + period_samples); after each period the
     * float drift accumulates and a sample is skipped when it exceeds 1. */
    float psf = period * fs;
    unsigned long ps = (unsigned long)psf;
    float diff = psf - (float)ps;
    float cd = 0.0f;
    size_t n = 0;
    int64_t s = 0;
    if (ps == 0 || cap == 0)
        return 0;
    while (n < cap) {
        start[n++] = s;
        if ((unsigned long)s + ps > total)
            break;
        s += (int64_t)ps;
        cd += diff;
        if (cd > 1.0f) {
            cd -= 1.0f;
            s += 1;
        }
    }
    return n;
}

/* ------------------------------------------------------------------------ */
/* simulated pulsar                                                          */
/* ------------------------------------------------------------------------ */

unsigned long orc_simulate_two_spike(float bw, float dm, float f0, float period,
                                     unsigned long repeat, double *out,
                                     unsigned long cap)
{
    /* simulated_complex_signal.cpp:12-24 (parameters) and :40-175 */
    float fs = bw;
    unsigned long Np = (unsigned long)(period * fs);
    unsigned long Nd = orc_nd(bw, dm, f0);
    if (Np < 4 || repeat * Np > cap)
        return 0;
    unsigned long range = (unsigned long)ceilf((float)Nd / (float)Np);
    if (range == 0)
        range = 1;
    unsigned long order = (unsigned long)pow(2.0, ceil(log2((double)(range * Np))));
    unsigned long fftpoint = 2 * order;
    float kdm = ref_kdm();
    float w0 = (float)(2 * REF_PI * f0);
    double *H1 = (double *)calloc(2 * order, sizeof(double));
    double *H = (double *)calloc(2 * fftpoint, sizeof(double));
    double *sfd = (double *)malloc(sizeof(double) * 2 * fftpoint);
    double *one = (double *)calloc(2 * Np, sizeof(double));
    for (unsigned long i = 0; i < order; i++) {
        float wi = chirp_w(fs, order, i);
        double ph = chirp_phase_w(wi, kdm, dm, w0);
        unsigned long j = (i < order / 2) ? (order / 2 + i) : (i - order / 2);
        H1[2 * j] = cos(ph);
        H1[2 * j + 1] = sin(ph);
    }
    /* :253-261 backward, normalised by order; :263-268 placed in the upper
     * half of a zero buffer of 2*order and transformed forward */
    orc_fft(H1, order, +1);
    for (unsigned long i = 0; i < 2 * order; i++)
        H1[i] /= (double)order;
    memcpy(H + 2 * order, H1, sizeof(double) * 2 * order);
    orc_fft(H, fftpoint, -1);
    memset(out, 0, sizeof(double) * 2 * Np);
    unsigned long pulse = Np / 2;
    for (unsigned long i = 0; i < range; i++) {
        memset(sfd, 0, sizeof(double) * 2 * fftpoint);
        sfd[2 * (i * Np + pulse)] = 1.0;
        sfd[2 * (i * Np + pulse + 2)] = 1.0;
        orc_fft(sfd, fftpoint, -1);
        for (unsigned long j = 0; j < fftpoint; j++) {
            double re = sfd[2 * j] * H[2 * j] - sfd[2 * j + 1] * H[2 * j + 1];
            double im = sfd[2 * j] * H[2 * j + 1] + sfd[2 * j + 1] * H[2 * j];
            sfd[2 * j] = re;
            sfd[2 * j + 1] = im;
        }
        orc_fft(sfd, fftpoint, +1);
        for (unsigned long j = 0; j < Np; j++) {
            out[2 * j] += sfd[2 * j] / (double)fftpoint;
            out[2 * j + 1] += sfd[2 * j + 1] / (double)fftpoint;
        }
    }
    for (unsigned long r = 1; r < repeat; r++)
        memcpy(out + 2 * r * Np, out, sizeof(double) * 2 * Np);
    free(H1);
    free(H);
    free(sfd);
    free(one);
    return Np;
}
