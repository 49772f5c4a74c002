// The y direction of the wall Poisson solve in DCT mode (walls on the y nodes
// j = 0 and j = N, Neumann-0 pressure; DCT-I along y, FFTs along x and z):
// src/poisson/poisson.cpp:183-199, 268-335 build it with FFTW's REDFT00
// (`fftw_cos1`, poisson.cpp:97-101) on the N + 1 y nodes.
//
// cuFFT transforms the (i, k) planes of every stored y row (a batched 2-D D2Z
// over the N + 1 rows, no extension), and k_pois_dct does the rest in one pass
// over the half spectrum [i][j][kz] (j = 0..N): per (i, kz) column the DCT-I
// along j, the scale -1/k'^2/(N0 2N N2) (k'^2 = kx'^2 + ky'^2 + kz'^2, the y
// modified wavenumbers of period 2 L_y), and the DCT-I back.  With
//   X_m = x_0 + (-1)^m x_N + 2 sum_{n=1}^{N-1} x_n cos(pi n m / N)
// (the 2N-point DFT of the even extension) the solve is p = X(s X(rhs)), the
// even-extension solve's values up to rounding.
//
// DCT-I of N + 1 points from one N-point complex FFT (N = 256 = 16 x 16, the
// register DFTs of nova_fft.cuh).  For complex f (the real-linear transform
// applies to the real and imaginary parts at once):
//   w_0 = (f_0 + f_N) / 2,  w_n = (f_n + f_{N-n}) / 2 - sin(pi n / N)(f_n - f_{N-n}),
//   W = DFT_N(w)  (e^{-2 pi i n k / N}),
//   X_{2k}   = W_k + W_{N-k}                           (k = 0..N/2, W_N = W_0),
//   X_1      = (f_0 - f_N) + 2 sum_{n=1}^{N-1} f_n cos(pi n / N),
//   X_{2k+1} = X_{2k-1} + i (W_k - W_{N-k})            (k = 1..N/2-1).
// (Split f_n into its part symmetric and antisymmetric under n -> N - n: the
// DFT of the first is the real cosine sum, of the second times sin(pi n/N)
// the sine sum, and cos(a + b) - cos(a - b) = -2 sin a sin b links the odd
// outputs.)  The odd outputs are a prefix sum along k.
#include "nova_fft.cuh"
#include "nova_internal.cuh"
#include "nova_ops.cuh"
#include "nova_tma.cuh"

#include <algorithm>

namespace nova {

namespace {

constexpr int kN = 256;            // y intervals: N + 1 stored rows
constexpr int kR = 16;             // 256 = 16 x 16
constexpr int kCol = 8;            // columns per block (4 blocks per SM)
constexpr int kDThreads = kCol * kR;  // thread (col = tid % 8, t = tid / 8)
constexpr int kRows = kN + 1;
// shared memory: the column tile [257][8], W_256, W_512^n (n < 256), ky'^2 (257), scan scratch [16][8]
constexpr size_t kDSmem = sizeof(double2) * ((size_t)kRows * kCol + kN + kN + (size_t)kR * kCol) + sizeof(double) * kRows;

__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// global -> shared copies that hold no registers while in flight
// (cp.async; 16 bytes through L2 only, or 8 bytes)
__device__ __forceinline__ void cp16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// X = DCT-I(f) of column c: on entry S[n * 8 + c] = f_n (n = 0..N) for every
// column, all threads synchronised; on return x[q] = X_{16 t + q} and, for
// t = 15, xN = X_N.  S (and red) are overwritten; the caller synchronises
// before writing S again.
__device__ __forceinline__ void dct1(double2 *S, double2 *red, int c, int t, const double2 *tw, const double2 *t512,
                                     double2 (&x)[kR], double2 &xN)
{
    // pre-twiddle of this thread's inputs n = t + 16 n1, and its share of X_1's sum
    const double2 f0 = S[c], fN = S[kN * kCol + c];
    double2 v[kR];
    double2 cs = make_double2(0.0, 0.0);
#pragma unroll
    for (int n1 = 0; n1 < kR; n1++) {
        const int n = t + kR * n1;
        const double2 fn = S[n * kCol + c];
        if (n == 0) {
            v[n1] = make_double2(0.5 * (f0.x + fN.x), 0.5 * (f0.y + fN.y));
        } else {
            const double2 fm = S[(kN - n) * kCol + c];
            const double cn = t512[n].x, sn = -t512[n].y;  // cos, sin (pi n / N)
            const double2 d = sub(fn, fm);
            v[n1] = make_double2(fma(-sn, d.x, 0.5 * (fn.x + fm.x)), fma(-sn, d.y, 0.5 * (fn.y + fm.y)));
            cs = make_double2(fma(cn, fn.x, cs.x), fma(cn, fn.y, cs.y));
        }
    }
    red[t * kCol + c] = cs;
    __syncthreads();  // every read of f done (S is scratch from here), partial sums in red
    double2 x1 = make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < kR; u++) x1 = add(x1, red[u * kCol + c]);
    x1 = make_double2(fma(2.0, x1.x, f0.x - fN.x), fma(2.0, x1.y, f0.y - fN.y));

    // W = DFT_256(w): step 1 (thread = n2 = t) over n1, twiddle W^(t k1)
    dft<kR, kN, false>(v, tw);
#pragma unroll
    for (int k1 = 0; k1 < kR; k1++) S[(k1 * kR + t) * kCol + c] = k1 == 0 ? v[0] : cmul(v[k1], tw[(t * k1) % kN]);
    __syncthreads();
    // step 2 (thread = k1 = t) over n2 -> W_{t + 16 k2}
#pragma unroll
    for (int n2 = 0; n2 < kR; n2++) v[n2] = S[(t * kR + n2) * kCol + c];
    __syncthreads();
    dft<kR, kN, false>(v, tw);
#pragma unroll
    for (int k2 = 0; k2 < kR; k2++) S[(t + kR * k2) * kCol + c] = v[k2];
    __syncthreads();

    // post: thread t owns k = 8 t .. 8 t + 7, i.e. outputs m = 16 t .. 16 t + 15
    double2 run = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < kR / 2; q++) {
        const int k = (kR / 2) * t + q;
        const double2 wk = S[k * kCol + c], wm = S[((kN - k) % kN) * kCol + c];
        x[2 * q] = add(wk, wm);
        if (k > 0) run = add(run, make_double2(wm.y - wk.y, wk.x - wm.x));  // i (W_k - W_{N-k})
        x[2 * q + 1] = run;
    }
    xN = S[(kN / 2) * kCol + c];
    xN = add(xN, xN);
    red[t * kCol + c] = run;  // this thread's block sum (red's earlier reads precede the last barrier)
    __syncthreads();
    double2 excl = x1;
    for (int u = 0; u < t; u++) excl = add(excl, red[u * kCol + c]);
#pragma unroll
    for (int q = 0; q < kR / 2; q++) x[2 * q + 1] = add(excl, x[2 * q + 1]);
}

// Task t < nmain: columns (i, kz0 + c), i = t / nch, kz0 = 8 (t % nch); task
// t >= nmain: columns (8 (t - nmain) + c, nzh - 1), the last kz of 8
// consecutive i.  spec[(i (N + 1) + j) nzh + kz], j = 0..N.
__global__ void __launch_bounds__(kDThreads, 4)
    k_pois_dct(int nzh, int nch, int nmain, double2 *__restrict__ spec, const double2 *__restrict__ twg,
               const double2 *__restrict__ t512g, const double *__restrict__ kx2, const double *__restrict__ ky2e,
               const double *__restrict__ kz2, double invN3)
{
    extern __shared__ __align__(16) unsigned char smdct[];
    double2 *S = reinterpret_cast<double2 *>(smdct);  // [257][8]
    double2 *tw = S + kRows * kCol;                   // W_256^m
    double2 *t512 = tw + kN;                          // W_512^n = (cos, -sin)(pi n / N)
    double2 *red = t512 + kN;                         // [16][8]
    double *ky2 = reinterpret_cast<double *>(red + kR * kCol);
    const int tid = threadIdx.x, c = tid % kCol, t = tid / kCol;

    const int task = blockIdx.x;
    int i0, kz0, di, dkz;  // column c: i = i0 + di c, kz = kz0 + dkz c
    if (task < nmain) {
        i0 = task / nch, kz0 = kCol * (task % nch), di = 0, dkz = 1;
    } else {
        i0 = kCol * (task - nmain), kz0 = nzh - 1, di = 1, dkz = 0;
    }
    const long long rowst = nzh;                      // j stride
    const long long ist = (long long)kRows * nzh;     // i stride
    auto addr = [&](int col, int j) -> long long { return (i0 + di * col) * ist + j * rowst + kz0 + dkz * col; };
    // every global load of the block in flight at once, straight into shared
    // memory: the column tile (element e = j * 8 + col, thread tid takes
    // e = tid + 128 u) and the tables
    constexpr int kLd = (kRows * kCol + kDThreads - 1) / kDThreads;
    constexpr int kTb = kN / kDThreads;
#pragma unroll
    for (int u = 0; u < kLd; u++) {
        const int e = tid + kDThreads * u;
        if (u < kLd - 1 || e < kRows * kCol) cp16(S + e, spec + addr(e % kCol, e / kCol));
    }
#pragma unroll
    for (int u = 0; u < kTb; u++) {
        cp16(tw + tid + kDThreads * u, twg + tid + kDThreads * u);
        cp16(t512 + tid + kDThreads * u, t512g + tid + kDThreads * u);
    }
#pragma unroll
    for (int u = 0; u <= kTb; u++)
        if (tid + kDThreads * u < kRows) cp8(ky2 + tid + kDThreads * u, ky2e + tid + kDThreads * u);
    const double kxx = kx2[i0 + di * c], kzz = kz2[kz0 + dkz * c];
    cp_wait_all();
    __syncthreads();

    double2 x[kR], xN;
    dct1(S, red, c, t, tw, t512, x, xN);
    // scale -1 / k'^2 / (N0 2N N2), 0 where k'^2 < 1e-16 (k_scale's sum order;
    // one reciprocal per element instead of two divisions)
    auto scale = [&](double2 v, int m) -> double2 {
        const double k2 = (kxx + ky2[m]) + kzz;
        const double f = k2 < 1.0e-16 ? 0.0 : -invN3 * recip(k2);
        return make_double2(v.x * f, v.y * f);
    };
    __syncthreads();  // every read of S inside dct1 done
#pragma unroll
    for (int q = 0; q < kR; q++) S[(kR * t + q) * kCol + c] = scale(x[q], kR * t + q);
    if (t == kR - 1) S[kN * kCol + c] = scale(xN, kN);
    __syncthreads();
    dct1(S, red, c, t, tw, t512, x, xN);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kR; q++) S[(kR * t + q) * kCol + c] = x[q];
    if (t == kR - 1) S[kN * kCol + c] = xN;
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kLd; u++) {
        const int e = tid + kDThreads * u;
        if (u < kLd - 1 || e < kRows * kCol) spec[addr(e % kCol, e / kCol)] = S[e];
    }
}

}  // namespace

bool pois_dct_fits(const Geo &g, int ny)
{
    const int nzh = g.N2 / 2 + 1;
    return g.wallY && ny == kN && g.N1 == kRows && (nzh - 1) % kCol == 0 && g.N0 % kCol == 0;
}

void launch_pois_dct(const Geo &g, void *spec, const double *tw256, const double *t512, const double *kx2,
                     const double *ky2e, const double *kz2, double invN3, cudaStream_t st)
{
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_pois_dct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDSmem);
        attr = true;
    }
    const int nzh = g.N2 / 2 + 1, nch = (nzh - 1) / kCol;
    const int nmain = g.N0 * nch, ntask = nmain + g.N0 / kCol;
    k_pois_dct<<<ntask, kDThreads, kDSmem, st>>>(nzh, nch, nmain, (double2 *)spec, (const double2 *)tw256,
                                                 (const double2 *)t512, kx2, ky2e, kz2, invN3);
}

}  // namespace nova
