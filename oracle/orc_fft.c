/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle (see orc_fft.h).
 *
 * Recursive decimation-in-time Cooley-Tukey FFT for any length: the length is
 * split by its smallest prime factor p, the p sub-sequences are transformed
 * recursively and combined with an O(p^2) DFT butterfly.  Twiddles are read
 * from one table of exp(sign*2*pi*i*t/n) for the top-level n, built with
 * exact values on the axes, so sub-transforms index it with a stride.
 * Accuracy is checked against numpy.fft in tests/test_oracle.py.
 */
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static orc_cplx twiddle(long t, long n, int sign)
{
    orc_cplx w;
    t %= n;
    if (t == 0) { w.re = 1.0; w.im = 0.0; return w; }
    if (4 * t == n) { w.re = 0.0; w.im = (double)sign; return w; }
    if (2 * t == n) { w.re = -1.0; w.im = 0.0; return w; }
    if (4 * t == 3 * n) { w.re = 0.0; w.im = -(double)sign; return w; }
    double a = 2.0 * M_PI * (double)t / (double)n;
    w.re = cos(a);
    w.im = sign * sin(a);
    return w;
}

static int smallest_factor(int n)
{
    if (n % 2 == 0) return 2;
    for (int p = 3; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

static inline orc_cplx cmul(orc_cplx a, orc_cplx b)
{
    orc_cplx c;
    c.re = a.re * b.re - a.im * b.im;
    c.im = a.re * b.im + a.im * b.re;
    return c;
}

/* out[k] = sum_j in[j*is] * W^(j*k*ws), k < n;  W = table for length ntop. */
static void fft_rec(int n, const orc_cplx *in, long is, orc_cplx *out,
                    const orc_cplx *W, long ntop, long ws, orc_cplx *scratch)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = smallest_factor(n);
    int m = n / p;
    for (int r = 0; r < p; r++)
        fft_rec(m, in + (long)r * is, is * p, out + (long)r * m, W, ntop, ws * p, scratch);
    /* butterflies: X[q*m+s] = sum_r (Y_r[s] * w_n^(r*s)) * w_p^(r*q) */
    orc_cplx *y = scratch;
    for (int s = 0; s < m; s++) {
        for (int r = 0; r < p; r++) {
            orc_cplx v = out[(long)r * m + s];
            long t = ((long)r * s * ws) % ntop;
            y[r] = (t == 0) ? v : cmul(v, W[t]);
        }
        if (p == 2) {
            out[s].re = y[0].re + y[1].re;
            out[s].im = y[0].im + y[1].im;
            out[m + s].re = y[0].re - y[1].re;
            out[m + s].im = y[0].im - y[1].im;
        } else {
            for (int q = 0; q < p; q++) {
                orc_cplx acc = y[0];
                for (int r = 1; r < p; r++) {
                    long t = ((long)r * q * m * ws) % ntop;
                    orc_cplx v = (t == 0) ? y[r] : cmul(y[r], W[t]);
                    acc.re += v.re;
                    acc.im += v.im;
                }
                out[(long)q * m + s] = acc;
            }
        }
    }
}

void orc_fft1d(int n, orc_cplx *data, long stride, int sign)
{
    if (n <= 1) return;
    orc_cplx *W = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
    orc_cplx *in = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
    orc_cplx *out = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
    orc_cplx *scr = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
    for (int t = 0; t < n; t++) W[t] = twiddle(t, n, sign);
    for (int j = 0; j < n; j++) in[j] = data[(long)j * stride];
    fft_rec(n, in, 1, out, W, n, 1, scr);
    for (int j = 0; j < n; j++) data[(long)j * stride] = out[j];
    free(W); free(in); free(out); free(scr);
}

/* Same as orc_fft1d but for many lines sharing one twiddle table. */
static void fft_lines(int n, orc_cplx *base, long stride, long nlines,
                      const long *line_off, int sign)
{
    if (n <= 1) return;
    orc_cplx *W = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
    for (int t = 0; t < n; t++) W[t] = twiddle(t, n, sign);
    /* lines are independent: with OpenMP each thread transforms its own lines
     * with private buffers (identical arithmetic per line) */
#pragma omp parallel
    {
        orc_cplx *in = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
        orc_cplx *out = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
        orc_cplx *scr = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
#pragma omp for schedule(static)
        for (long L = 0; L < nlines; L++) {
            orc_cplx *d = base + line_off[L];
            for (int j = 0; j < n; j++) in[j] = d[(long)j * stride];
            fft_rec(n, in, 1, out, W, n, 1, scr);
            for (int j = 0; j < n; j++) d[(long)j * stride] = out[j];
        }
        free(in); free(out); free(scr);
    }
    free(W);
}

void orc_fft3d(const int n[3], orc_cplx *data, int sign)
{
    const long n0 = n[0], n1 = n[1], n2 = n[2];
    long maxl = n0 * n1;
    if (n1 * n2 > maxl) maxl = n1 * n2;
    if (n0 * n2 > maxl) maxl = n0 * n2;
    long *off = (long *)malloc(sizeof(long) * maxl);
    long c;
    /* axis 0 (stride 1) */
    c = 0;
    for (long k = 0; k < n2; k++)
        for (long j = 0; j < n1; j++) off[c++] = n0 * (j + n1 * k);
    fft_lines((int)n0, data, 1, c, off, sign);
    /* axis 1 (stride n0) */
    c = 0;
    for (long k = 0; k < n2; k++)
        for (long i = 0; i < n0; i++) off[c++] = i + n0 * n1 * k;
    fft_lines((int)n1, data, n0, c, off, sign);
    /* axis 2 (stride n0*n1) */
    c = 0;
    for (long j = 0; j < n1; j++)
        for (long i = 0; i < n0; i++) off[c++] = i + n0 * j;
    fft_lines((int)n2, data, n0 * n1, c, off, sign);
    free(off);
}
