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
//
// N0 = 256 with N2 % 16 == 0 and N1 % 8 == 0 runs k_pois_tma instead: the
// same arithmetic on tiles of 8 columns, fed by bulk tensor loads into a
// double-buffered shared-memory tile (the next tile lands while the block
// transforms the current one), in a persistent grid.  k_pois_i loads, computes
// and stores in turn, so with two blocks per SM the memory pipe idles while
// both compute (96 us at 256^3 against a 41 us byte floor).
#include "nova_fft.cuh"
#include "nova_internal.cuh"
#include "nova_ops.cuh"
#include "nova_tma.cuh"

#include <algorithm>
#include <cstring>

namespace nova {

namespace {

constexpr int kCols = 16;  // kz columns per block: 16 x 16 B = 256 contiguous bytes per i row

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

// ---- N0 = 256 on a TMA-fed, double-buffered tile ----
constexpr int kTR = 16, kTN = kTR * kTR;  // 256 = 16 x 16
constexpr int kTC = 8;                    // columns per tile
constexpr int kTThreads = kTC * kTR;      // thread (col, t): col = tid % 8, t = tid / 8
constexpr uint32_t kTileBytes = kTN * kTC * sizeof(double2);  // 32 KB
constexpr size_t kTSmem =
    2 * (size_t)kTileBytes + kTN * sizeof(double2) + kTN * sizeof(double) + 2 * sizeof(unsigned long long);

// the half spectrum as FP64 [i][j][2 nzh]: `col` boxes 16 x 1 x 256 (8 kz of
// one j, every i), `rem` boxes 2 x 8 x 256 (the last kz of 8 consecutive j);
// both land as [i][8 columns] complex
struct PoisMaps {
    CUtensorMap col, rem;
};

// Tasks t < nmain: j = t / nch, kz = 8 (t % nch) + col (nch = (nzh - 1) / 8);
// tasks t >= nmain: j = 8 (t - nmain) + col, kz = nzh - 1.  Block b takes
// tasks b, b + gridDim.x, ...; the load of the next one is issued when the
// current one starts.  Arithmetic, order and twiddles are k_pois_i<16>'s.
__global__ void __launch_bounds__(kTThreads, 3)
    k_pois_tma(int ny, int nzh, double2 *__restrict__ spec, const double2 *__restrict__ twN,
               const double *__restrict__ kx2, const double *__restrict__ ky2, const double *__restrict__ kz2,
               double invN3, const __grid_constant__ PoisMaps maps, int nmain, int ntask, int *err)
{
    extern __shared__ __align__(128) unsigned char smtile[];
    double2 *tiles = reinterpret_cast<double2 *>(smtile);  // [2][kTN][kTC]
    double2 *tw = tiles + 2 * kTN * kTC;                   // W_256^m
    double *kx2s = reinterpret_cast<double *>(tw + kTN);   // kx'^2 (the scale's i wavenumbers)
    const uint32_t bar0 = smem_addr(kx2s + kTN);           // one mbarrier per tile
    const int tid = threadIdx.x, col = tid % kTC, t = tid / kTC;
    const int nch = (nzh - 1) / kTC;
    for (int m = tid; m < kTN; m += kTThreads) {
        tw[m] = twN[m];
        kx2s[m] = kx2[m];
    }
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init_fence();
    }
    __syncthreads();
    auto issue = [&](int task, int b) {  // thread 0
        const uint32_t dst = smem_addr(tiles + b * kTN * kTC), bar = bar0 + 8u * b;
        mbar_expect_tx(bar, kTileBytes);
        if (task < nmain)
            tma_load_3d(dst, &maps.col, bar, 2 * kTC * (task % nch), task / nch, 0);
        else
            tma_load_3d(dst, &maps.rem, bar, 2 * (nzh - 1), kTC * (task - nmain), 0);
    };
    const long long rowstride = (long long)ny * nzh;
    int task = blockIdx.x;
    if (tid == 0 && task < ntask) issue(task, 0);
    for (int n = 0; task < ntask; n++, task += gridDim.x) {
        const int b = n & 1;
        const bool more = task + (int)gridDim.x < ntask;
        if (tid == 0 && more) issue(task + gridDim.x, b ^ 1);  // that tile was released at the end of step n - 1
        if (!__syncthreads_and(mbar_wait(bar0 + 8u * b, (n >> 1) & 1, err))) {
            // timed out: the loads still in flight land before the block leaves
            if (tid == 0) {
                mbar_wait(bar0 + 8u * b, (n >> 1) & 1, err, true);
                if (more) mbar_wait(bar0 + 8u * (b ^ 1), ((n + 1) >> 1) & 1, err, true);
            }
            return;
        }
        double2 *S = tiles + b * kTN * kTC;
        int jc, kzc;
        if (task < nmain) {
            jc = task / nch;
            kzc = kTC * (task % nch) + col;
        } else {
            jc = kTC * (task - nmain) + col;
            kzc = nzh - 1;
        }
        const double kyz = ky2[jc], kzz = kz2[kzc];  // issued early: used after the forward DFT
        double2 v[kTR];
#pragma unroll
        for (int n1 = 0; n1 < kTR; n1++) v[n1] = S[(t + kTR * n1) * kTC + col];
        __syncthreads();  // the tile is rewritten below
        // forward, step 1 (thread = n2 = t): DFT over n1, twiddle W_N^(t k1)
        dft<kTR, kTN, false>(v, tw);
#pragma unroll
        for (int k1 = 0; k1 < kTR; k1++) S[(k1 * kTR + t) * kTC + col] = k1 == 0 ? v[0] : cmul(v[k1], tw[(t * k1) % kTN]);
        __syncthreads();
        // forward, step 2 (thread = k1 = t): DFT over n2 -> X[t + R k2]
#pragma unroll
        for (int n2 = 0; n2 < kTR; n2++) v[n2] = S[(t * kTR + n2) * kTC + col];
        __syncthreads();
        dft<kTR, kTN, false>(v, tw);
#pragma unroll
        for (int k2 = 0; k2 < kTR; k2++) {
            const double k2v = (kx2s[t + kTR * k2] + kyz) + kzz;
            const double f = k2v < 1.0e-16 ? 0.0 : -invN3 * recip(k2v);
            v[k2] = make_double2(v[k2].x * f, v[k2].y * f);
        }
        // inverse, step 1 (thread = k1 = t): DFT over k2, twiddle W_N^-(n1 t)
        dft<kTR, kTN, true>(v, tw);
#pragma unroll
        for (int n1 = 0; n1 < kTR; n1++)
            S[(n1 * kTR + t) * kTC + col] = n1 == 0 ? v[0] : cmul(v[n1], conj2(tw[(t * n1) % kTN]));
        __syncthreads();
        // inverse, step 2 (thread = n1 = t): DFT over k1 -> x[t + R n2]
#pragma unroll
        for (int k1 = 0; k1 < kTR; k1++) v[k1] = S[(t * kTR + k1) * kTC + col];
        dft<kTR, kTN, true>(v, tw);
        double2 *dst = spec + (long long)t * rowstride + (long long)jc * nzh + kzc;
#pragma unroll
        for (int n2 = 0; n2 < kTR; n2++) dst[(long long)n2 * kTR * rowstride] = v[n2];
        // the transposes wrote the tile through the generic proxy; order those
        // writes before the bulk copy (async proxy) that refills it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();  // the tile is free for the load of step n + 2
    }
}

bool encode_spec(CUtensorMap *m, const void *spec, int n0, int ny, int nzh, unsigned bx, unsigned by)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = tma_encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)2 * nzh, (cuuint64_t)ny, (cuuint64_t)n0};
    const cuuint64_t strides[2] = {(cuuint64_t)2 * nzh * sizeof(double), (cuuint64_t)2 * nzh * ny * sizeof(double)};
    const cuuint32_t box[3] = {bx, by, (cuuint32_t)n0}, estr[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(spec), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool pois_tma_fits(const Geo &g, int ny)
{
    const int nzh = g.N2 / 2 + 1;
    return g.N0 == kTN && (nzh - 1) % kTC == 0 && ny % kTC == 0;
}

bool launch_pois_tma(const Geo &g, int ny, void *spec, const double *twN, const double *kx2, const double *ky2,
                     const double *kz2, double invN3, int *err, cudaStream_t st)
{
    const int nzh = g.N2 / 2 + 1;
    PoisMaps maps;
    std::memset(&maps, 0, sizeof maps);
    if (!encode_spec(&maps.col, spec, g.N0, ny, nzh, 2 * kTC, 1) || !encode_spec(&maps.rem, spec, g.N0, ny, nzh, 2, kTC))
        return false;
    static int nsm = 0;
    static bool attr = false;
    if (!attr) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_pois_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTSmem);
        attr = true;
    }
    const int nmain = ny * ((nzh - 1) / kTC), ntask = nmain + ny / kTC;
    const int grid = std::min(ntask, 3 * std::max(nsm, 1));
    k_pois_tma<<<grid, kTThreads, kTSmem, st>>>(ny, nzh, (double2 *)spec, (const double2 *)twN, kx2, ky2, kz2, invN3,
                                                maps, nmain, ntask, err);
    return true;
}

}  // namespace

bool pois_i_fits(const Geo &g) { return !g.wallY && (g.N0 == 64 || g.N0 == 256); }

void launch_pois_i(const Geo &g, int ny, void *spec, const double *twN, const double *kx2, const double *ky2,
                   const double *kz2, double invN3, int *err, cudaStream_t st)
{
    if (g.N0 == 256) {
        if (err && pois_tma_fits(g, ny) && launch_pois_tma(g, ny, spec, twN, kx2, ky2, kz2, invN3, err, st)) return;
        launch_r<16>(g, ny, spec, twN, kx2, ky2, kz2, invN3, st);
    } else {
        launch_r<8>(g, ny, spec, twN, kx2, ky2, kz2, invN3, st);
    }
}

}  // namespace nova
