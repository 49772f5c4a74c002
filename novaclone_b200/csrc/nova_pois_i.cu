// The i direction of the periodic spectral Poisson solve, fused with the
// spectral scale (src/poisson/poisson.cpp:223-265):
//
//   rhs^ = FFT_i FFT_j FFT_k rhs,  rhs^ = -rhs^ / k'^2 / (N0 N1 N2)  (0 where k'^2 < 1e-16),
//   p = IFFT_k IFFT_j IFFT_i rhs^
//
// cuFFT runs the (j, k) planes as batched 2-D transforms (D2Z before, Z2D
// after); this kernel does FFT_i, the scale and IFFT_i of every (j, kz)
// column of the half spectrum [i][j][kz] in one pass over HBM, where a 3-D
// cuFFT plan needs an i pass on either side and the scale a pass of its own.
//
// Length N0 = R * R, two-step decomposition with n = R n1 + n2, k = k1 + R k2:
//   X[k1 + R k2] = sum_n2 W_R^(n2 k2) W_N^(n2 k1) sum_n1 x[R n1 + n2] W_R^(n1 k1)
// and the inverse with the roles of the two indices exchanged.  A block owns
// kCols consecutive kz columns of one j; thread (col, t) loads its R values
// x[R n1 + t] straight from HBM, runs R-point DFTs in registers, and one
// shared-memory transpose joins the two steps.  The twiddles W_N^m are a
// host-computed table; the scale is k_scale's up to the rounding of one
// reciprocal (within an ulp or two of its two divisions).
#include "nova_fft.cuh"
#include "nova_internal.cuh"
#include "nova_ops.cuh"

namespace nova {

namespace {

constexpr int kCols = 16;  // kz columns per block: 16 x 16 B = 256 contiguous bytes per i row

// 1/a for a >= 1e-16 (normal in FP32 for every mesh this solver meets):
// the correctly rounded FP32 reciprocal refined by two Newton-Raphson steps
// y <- y + y (1 - a y) in FP64 (relative error about 2^-23 -> 2^-46 -> below
// an ulp of FP64, up to the rounding of the last step)
__device__ __forceinline__ double recip(double a)
{
    double y = (double)__frcp_rn((float)a);
    y = fma(y, fma(-a, y, 1.0), y);
    return fma(y, fma(-a, y, 1.0), y);
}

template <int R>
__global__ void __launch_bounds__(kCols *R, R == 16 ? 2 : 4)
    k_pois_i(int ny, int nzh, double2 *__restrict__ spec, const double2 *__restrict__ twN,
             const double *__restrict__ kx2, const double *__restrict__ ky2, const double *__restrict__ kz2,
             double invN3)
{
    constexpr int N = R * R;
    extern __shared__ __align__(16) unsigned char smraw[];
    double2 *tw = reinterpret_cast<double2 *>(smraw);  // W_N^m, m = 0..N-1
    double2 *S = tw + N;                               // transpose buffer [R][R][kCols]
    const int tid = threadIdx.x;
    const int col = tid % kCols, t = tid / kCols;
    const int j = blockIdx.y;
    const int kz = blockIdx.x * kCols + col;
    const bool valid = kz < nzh;
    for (int m = tid; m < N; m += kCols * R) tw[m] = twN[m];
    // element (i, j, kz) of the half spectrum; this thread's rows are i = t + R m
    const long long rowstride = (long long)ny * nzh;
    double2 *col_t = spec + (long long)t * rowstride + (long long)j * nzh + (valid ? kz : 0);
    const long long step = R * rowstride;

    double2 v[R];
#pragma unroll
    for (int n1 = 0; n1 < R; n1++) v[n1] = valid ? col_t[n1 * step] : make_double2(0.0, 0.0);
    __syncthreads();  // the twiddle table

    // forward, step 1 (thread = n2 = t): DFT over n1, twiddle W_N^(t k1)
    dft<R, N, false>(v, tw);
#pragma unroll
    for (int k1 = 0; k1 < R; k1++) S[(k1 * R + t) * kCols + col] = k1 == 0 ? v[0] : cmul(v[k1], tw[(t * k1) % N]);
    __syncthreads();
    // forward, step 2 (thread = k1 = t): DFT over n2 -> X[t + R k2]
#pragma unroll
    for (int n2 = 0; n2 < R; n2++) v[n2] = S[(t * R + n2) * kCols + col];
    __syncthreads();  // S is rewritten below
    dft<R, N, false>(v, tw);

    // scale: -1 / k'^2 / (N0 N1 N2), 0 where k'^2 < 1e-16 (k'^2 summed in
    // k_scale's order; one reciprocal per element instead of two divisions)
    const double kyz = ky2[j], kzz = valid ? kz2[kz] : 0.0;
#pragma unroll
    for (int k2 = 0; k2 < R; k2++) {
        const double k2v = (kx2[t + R * k2] + kyz) + kzz;
        const double f = k2v < 1.0e-16 ? 0.0 : -invN3 * recip(k2v);
        v[k2] = make_double2(v[k2].x * f, v[k2].y * f);
    }

    // inverse, step 1 (thread = k1 = t): DFT over k2, twiddle W_N^-(n1 t)
    dft<R, N, true>(v, tw);
#pragma unroll
    for (int n1 = 0; n1 < R; n1++)
        S[(n1 * R + t) * kCols + col] = n1 == 0 ? v[0] : cmul(v[n1], conj2(tw[(t * n1) % N]));
    __syncthreads();
    // inverse, step 2 (thread = n1 = t): DFT over k1 -> x[t + R n2]
#pragma unroll
    for (int k1 = 0; k1 < R; k1++) v[k1] = S[(t * R + k1) * kCols + col];
    dft<R, N, true>(v, tw);
    if (valid) {
#pragma unroll
        for (int n2 = 0; n2 < R; n2++) col_t[n2 * step] = v[n2];
    }
}

template <int R>
void launch_r(const Geo &g, int ny, void *spec, const double *twN, const double *kx2, const double *ky2,
              const double *kz2, double invN3, cudaStream_t st)
{
    constexpr int N = R * R;
    constexpr size_t smem = sizeof(double2) * ((size_t)N + (size_t)R * R * kCols);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_pois_i<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int nzh = g.N2 / 2 + 1;
    const dim3 grid((nzh + kCols - 1) / kCols, ny);
    k_pois_i<R><<<grid, kCols * R, smem, st>>>(ny, nzh, (double2 *)spec, (const double2 *)twN, kx2, ky2, kz2,
                                               invN3);
}

}  // namespace

bool pois_i_fits(const Geo &g) { return !g.wallY && (g.N0 == 64 || g.N0 == 256); }

void launch_pois_i(const Geo &g, int ny, void *spec, const double *twN, const double *kx2, const double *ky2,
                   const double *kz2, double invN3, cudaStream_t st)
{
    if (g.N0 == 256)
        launch_r<16>(g, ny, spec, twN, kx2, ky2, kz2, invN3, st);
    else
        launch_r<8>(g, ny, spec, twN, kx2, ky2, kz2, invN3, st);
}

}  // namespace nova
