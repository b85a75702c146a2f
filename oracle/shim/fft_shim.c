/*
 * FFTW-API shim (test infrastructure only): lets the reference's FFT actors
 * (param_code/code_fft_1core/src/CPU/fft_run.c:23-83) link without FFTW.
 * Plans only record their arguments; execution calls the oracle's
 * double-precision DFT (../fft_ref.c), so the float build's FFT is rounded
 * once from a double result.  This is the only stand-in in the compiled
 * reference; every other symbol comes from the reference sources.
 */
#include <stdlib.h>

#include "fftw3.h"
#include "../fft_ref.h"

struct shim_plan_s {
    int n0, n1, sign, is_double;
    void *in, *out;
};

static struct shim_plan_s *make_plan(int n0, int n1, void *in, void *out, int sign, int is_double)
{
    struct shim_plan_s *p = (struct shim_plan_s *)malloc(sizeof(*p));
    p->n0 = n0;
    p->n1 = n1;
    p->sign = sign;
    p->is_double = is_double;
    p->in = in;
    p->out = out;
    return p;
}

static void run_plan(const struct shim_plan_s *p)
{
    if (p->is_double)
        oracle_fft2d_c128(p->n0, p->n1, (const double *)p->in, (double *)p->out, p->sign);
    else
        oracle_fft2d_c64(p->n0, p->n1, (const float *)p->in, (float *)p->out, p->sign);
}

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags)
{
    (void)flags;
    return make_plan(n0, n1, in, out, sign, 0);
}
void fftwf_execute(const fftwf_plan p) { run_plan(p); }
void fftwf_destroy_plan(fftwf_plan p) { free(p); }

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
    (void)flags;
    return make_plan(n0, n1, in, out, sign, 1);
}
void fftw_execute(const fftw_plan p) { run_plan(p); }
void fftw_destroy_plan(fftw_plan p) { free(p); }
