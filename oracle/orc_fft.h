/*
 * TEST INFRASTRUCTURE ONLY -- part of the CPU oracle. Never linked into the
 * product library, never timed as the product.
 *
 * Double-precision complex FFT (mixed radix, any length; radices 2 and 3
 * cover every grid this project runs: 2^a * 3^b).  It stands in for the
 * FFTW c2c transforms that heFFTe performs in the reference
 * (src/poisson/poisson.cpp:225,250: fft->forward / fft->backward, unscaled).
 * Sign convention as FFTW: forward uses exp(-2*pi*i*j*k/n), backward
 * exp(+2*pi*i*j*k/n); neither direction scales.
 */
#ifndef ORC_FFT_H
#define ORC_FFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } orc_cplx;

/* In-place 1-D transform of n points spaced `stride` apart. sign = -1 forward, +1 backward. */
void orc_fft1d(int n, orc_cplx *data, long stride, int sign);

/* In-place 3-D transform of an n0 x n1 x n2 array with index i + n0*(j + n1*k)
 * (first index fastest, heFFTe's default box ordering). */
void orc_fft3d(const int n[3], orc_cplx *data, int sign);

#ifdef __cplusplus
}
#endif
#endif
