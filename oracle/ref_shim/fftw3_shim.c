/* FFTW3f API stand-in for compiling the reference (test infrastructure).
 * Power-of-two sizes only, which is all the reference plans. */
#include "fftw3.h"
#include <stdlib.h>
#include <string.h>
#include "../orc.h"

struct fftwf_plan_s {
    int n, sign;
    fftwf_complex *in, *out;
};

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags)
{
    (void)flags;
    fftwf_plan p = (fftwf_plan)malloc(sizeof(*p));
    p->n = n;
    p->sign = sign;
    p->in = in;
    p->out = out;
    return p;
}

void fftwf_execute(const fftwf_plan p)
{
    double *x = (double *)malloc(sizeof(double) * 2 * (size_t)p->n);
    for (int i = 0; i < p->n; i++) {
        x[2 * i] = p->in[i][0];
        x[2 * i + 1] = p->in[i][1];
    }
    orc_fft(x, (unsigned long)p->n, p->sign < 0 ? -1 : +1);
    for (int i = 0; i < p->n; i++) {
        p->out[i][0] = (float)x[2 * i];
        p->out[i][1] = (float)x[2 * i + 1];
    }
    free(x);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
void *fftwf_malloc(size_t n) { return malloc(n); }
void fftwf_free(void *p) { free(p); }
