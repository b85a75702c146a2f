/* ORACLE (test infrastructure): double-precision 2-D DFT, FFTW sign convention. */
#ifndef ORACLE_FFT_REF_H
#define ORACLE_FFT_REF_H
#ifdef __cplusplus
extern "C" {
#endif
/* Row-major n0 x n1 complex arrays (interleaved re, im).  in may equal out.
 * sign = -1 forward, +1 backward; unnormalised both ways. */
void oracle_fft2d_c128(int n0, int n1, const double *in, double *out, int sign);
/* Same transform for complex64 buffers; computed in double, rounded once. */
void oracle_fft2d_c64(int n0, int n1, const float *in, float *out, int sign);
#ifdef __cplusplus
}
#endif
#endif
