// Register-resident DFT building blocks of the spectral Poisson solve
// (nova_pois_i.cu, nova_fft2d.cu): complex products, and R-point DFTs (R = 4,
// 8, 16) in natural order with twiddles W_R^m read from a table of W_N^m
// (N a multiple of R) at compile-time indices.
#pragma once

#include <cuda_runtime.h>

namespace nova {

__device__ __forceinline__ double2 cmul(double2 a, double2 w)
{
    return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}

__device__ __forceinline__ double2 conj2(double2 w) { return make_double2(w.x, -w.y); }

// 1/a for a >= 1e-16 (normal in FP32 for every mesh the Poisson scales meet):
// the correctly rounded FP32 reciprocal refined by two Newton-Raphson steps
// y <- y + y (1 - a y) in FP64 (relative error about 2^-23 -> 2^-46 -> below
// an ulp of FP64, up to the rounding of the last step)
__device__ __forceinline__ double recip(double a)
{
    double y = (double)__frcp_rn((float)a);
    y = fma(y, fma(-a, y, 1.0), y);
    return fma(y, fma(-a, y, 1.0), y);
}

__host__ __device__ constexpr int bitrev(int x, int bits)
{
    int r = 0;
    for (int b = 0; b < bits; b++) r |= ((x >> b) & 1) << (bits - 1 - b);
    return r;
}

// in-place R-point DFT of v in natural order: v[k] = sum_n v[n] W_R^(+-n k)
// (- forward, + inverse); W_R^m = tw[m * (N / R)] (tw: the W_N table in
// shared memory, read at compile-time indices, i.e. broadcast).
// R = 8: radix-2 decimation in time.
template <int R, int N, bool INV> __device__ __forceinline__ void dft_radix2(double2 (&v)[R], const double2 *tw)
{
    constexpr int bits = R == 8 ? 3 : 4;
#pragma unroll
    for (int x = 0; x < R; x++) {
        const int y = bitrev(x, bits);
        if (y > x) {
            const double2 t = v[x];
            v[x] = v[y];
            v[y] = t;
        }
    }
#pragma unroll
    for (int len = 2; len <= R; len *= 2) {
        const int half = len / 2;
#pragma unroll
        for (int b = 0; b < R; b += len) {
#pragma unroll
            for (int j = 0; j < half; j++) {
                const double2 a = v[b + j];
                double2 c = v[b + j + half];
                if (j != 0) {
                    const double2 w = tw[j * (R / len) * (N / R)];
                    c = cmul(c, INV ? conj2(w) : w);
                }
                v[b + j] = make_double2(a.x + c.x, a.y + c.y);
                v[b + j + half] = make_double2(a.x - c.x, a.y - c.y);
            }
        }
    }
}

// 4-point DFT in place; W_4 = -i forward, +i inverse (no multiplications)
template <bool INV> __device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3)
{
    const double2 t0 = make_double2(a0.x + a2.x, a0.y + a2.y), t1 = make_double2(a0.x - a2.x, a0.y - a2.y);
    const double2 t2 = make_double2(a1.x + a3.x, a1.y + a3.y), d = make_double2(a1.x - a3.x, a1.y - a3.y);
    const double2 t3 = INV ? make_double2(-d.y, d.x) : make_double2(d.y, -d.x);
    a0 = make_double2(t0.x + t2.x, t0.y + t2.y);
    a2 = make_double2(t0.x - t2.x, t0.y - t2.y);
    a1 = make_double2(t1.x + t3.x, t1.y + t3.y);
    a3 = make_double2(t1.x - t3.x, t1.y - t3.y);
}

// R = 16 as 4 x 4 (n = 4 n1 + n2, k = k1 + 4 k2): 4-point DFTs over n1, the
// twiddles W_16^(n2 k1) (W_16^4 = -+i free), 4-point DFTs over n2, then the
// 4 x 4 index transpose, which is a renaming of registers
template <int N, bool INV> __device__ __forceinline__ void dft16(double2 (&v)[16], const double2 *tw)
{
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4<INV>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
#pragma unroll
    for (int n2 = 1; n2 < 4; n2++)
#pragma unroll
        for (int k1 = 1; k1 < 4; k1++) {
            double2 &x = v[4 * k1 + n2];
            if (n2 * k1 == 4)
                x = INV ? make_double2(-x.y, x.x) : make_double2(x.y, -x.x);
            else
                x = cmul(x, INV ? conj2(tw[n2 * k1 * (N / 16)]) : tw[n2 * k1 * (N / 16)]);
        }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4<INV>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    double2 o[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) o[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = o[k];
}

template <int R, int N, bool INV> __device__ __forceinline__ void dft(double2 (&v)[R], const double2 *tw)
{
    static_assert(R == 8 || R == 16, "R-point DFTs of 8 or 16 points");
    if constexpr (R == 16)
        dft16<N, INV>(v, tw);
    else
        dft_radix2<R, N, INV>(v, tw);
}

}  // namespace nova
