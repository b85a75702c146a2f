/*
 * FFTW-3 API subset used by the reference's FFT actors
 * (param_code/code_fft_1core/src/CPU/fft_run.c:37-39, 45-47, 67-69, 75-77).
 *
 * Test infrastructure only: FFTW is not installed on this machine, so the
 * reference's actor sources are linked against fft_shim.c, which implements
 * these five entry points with this project's own double-precision FFT
 * (fft_ref.c).  Nothing in the product links this file.
 *
 * Semantics kept from FFTW's documented interface:
 *   FFTW_FORWARD  = -1 : X[k] = sum_n x[n] e^{-2 pi i k n / N}
 *   FFTW_BACKWARD = +1 : X[k] = sum_n x[n] e^{+2 pi i k n / N}   (unnormalised)
 *   plan_dft_2d(n0, n1, ...) transforms a row-major n0 x n1 array.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef float fftwf_complex[2];
typedef double fftw_complex[2];

typedef struct shim_plan_s *fftwf_plan;
typedef struct shim_plan_s *fftw_plan;

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
