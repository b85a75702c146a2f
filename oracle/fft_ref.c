/*
 * ORACLE (test infrastructure, never linked into the product).
 *
 * Double-precision 2-D complex DFT with FFTW's sign convention and no
 * normalisation, used (a) behind the FFTW-API shim so the reference's FFT
 * actors (param_code/code_fft_1core/src/CPU/fft_run.c:23-83) can be compiled
 * and run here, and (b) by the oracle restatement (sdp_oracle.c).
 *
 * The reference's FFT lives in FFTW 3 (third party, absent from the reference
 * tree; version pinned only as fftw-3.3.8 in
 * param_code/code_fft_1core/CMakeLists.txt:195).  What is restated here is the
 * mathematical transform FFTW documents:
 *     X[k0,k1] = sum_{n0,n1} x[n0,n1] exp(sign * 2 pi i (k0 n0 / N0 + k1 n1 / N1)).
 * Power-of-two lengths use an iterative radix-2 Cooley-Tukey transform with
 * twiddles from cos/sin in double; other lengths use the O(N^2) definition.
 * It is checked against numpy.fft (pocketfft) in tests/test_oracle_fft.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft_ref.h"

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place 1-D transform of n complex values stored as interleaved doubles. */
static void fft1d_pow2(double *x, int n, int sign)
{
    /* bit reversal */
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = x[2 * i], ti = x[2 * i + 1];
            x[2 * i] = x[2 * j];
            x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = tr;
            x[2 * j + 1] = ti;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1;
        for (int k = 0; k < half; ++k) {
            double ang = (double)sign * 2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (int s = 0; s < n; s += len) {
                double *a = x + 2 * (s + k);
                double *b = x + 2 * (s + k + half);
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

static void dft1d_naive(double *x, int n, int sign, double *tmp)
{
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) {
            /* reduce k*j mod n exactly before forming the angle */
            long long kj = ((long long)k * (long long)j) % n;
            double ang = (double)sign * 2.0 * M_PI * (double)kj / (double)n;
            double c = cos(ang), s = sin(ang);
            sr += x[2 * j] * c - x[2 * j + 1] * s;
            si += x[2 * j] * s + x[2 * j + 1] * c;
        }
        tmp[2 * k] = sr;
        tmp[2 * k + 1] = si;
    }
    memcpy(x, tmp, sizeof(double) * 2 * (size_t)n);
}

static void fft1d(double *x, int n, int sign, double *tmp)
{
    if (is_pow2(n))
        fft1d_pow2(x, n, sign);
    else
        dft1d_naive(x, n, sign, tmp);
}

void oracle_fft2d_c128(int n0, int n1, const double *in, double *out, int sign)
{
    size_t total = (size_t)n0 * (size_t)n1;
    double *work = (double *)malloc(sizeof(double) * 2 * total);
    int nmax = n0 > n1 ? n0 : n1;
    double *line = (double *)malloc(sizeof(double) * 2 * (size_t)nmax);
    double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)nmax);
    memcpy(work, in, sizeof(double) * 2 * total);

    /* rows (contiguous, length n1) */
    for (int r = 0; r < n0; ++r)
        fft1d(work + 2 * (size_t)r * n1, n1, sign, tmp);
    /* columns (stride n1, length n0) */
    for (int c = 0; c < n1; ++c) {
        for (int r = 0; r < n0; ++r) {
            line[2 * r] = work[2 * ((size_t)r * n1 + c)];
            line[2 * r + 1] = work[2 * ((size_t)r * n1 + c) + 1];
        }
        fft1d(line, n0, sign, tmp);
        for (int r = 0; r < n0; ++r) {
            work[2 * ((size_t)r * n1 + c)] = line[2 * r];
            work[2 * ((size_t)r * n1 + c) + 1] = line[2 * r + 1];
        }
    }
    memcpy(out, work, sizeof(double) * 2 * total);
    free(tmp);
    free(line);
    free(work);
}

void oracle_fft2d_c64(int n0, int n1, const float *in, float *out, int sign)
{
    size_t total = (size_t)n0 * (size_t)n1;
    double *buf = (double *)malloc(sizeof(double) * 2 * total);
    for (size_t i = 0; i < 2 * total; ++i) buf[i] = (double)in[i];
    oracle_fft2d_c128(n0, n1, buf, buf, sign);
    for (size_t i = 0; i < 2 * total; ++i) out[i] = (float)buf[i];
    free(buf);
}
