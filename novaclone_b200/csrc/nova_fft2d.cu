// The (j, k) planes of the periodic spectral Poisson solve in one pass each
// way (src/poisson/poisson.cpp:225, 250: forward transform of the packed
// right-hand side, backward transform of the scaled spectrum).
//
// Forward: x[i][j][k] real (N1 = N2 = 256) -> X[i][j][kz], kz = 0..128, the
// half spectrum of the 2-D DFT over (j, k), unnormalised, in the layout of a
// batched cuFFT D2Z (k_pois_i runs the i direction on it).  Inverse: the
// unnormalised 2-D C2R back to x (the imaginary parts of the kz = 0 and 128
// columns' Hermitian partners are those of a real field; the solve produces
// them, and the rows' own DC and Nyquist imaginary parts are discarded as a
// C2R does).
//
// One cluster of 8 CTAs per i plane; CTA r owns rows j = 32 r .. 32 r + 31.
// Forward: phase 1 loads its 32 rows (64 KB, contiguous) into shared memory
// and runs the real-to-complex transform along k per row: a 128-point complex
// FFT of z[n] = x[2n] + i x[2n+1] (8 x 16 split, register DFTs, the index
// transposes through shared memory), then the split into the 129 outputs,
// pairwise in place (X[k] = E + W^k O, X[128-k] = conj(E - W^k O)).  After a
// cluster barrier, phase 2 takes 16 kz columns (17 for the last CTA) and runs
// the 256-point DFT along j (16 x 16 split), reading the column's rows from
// the eight CTAs' shared memory (distributed shared memory) and writing the
// finished column to HBM.  A second cluster barrier keeps every CTA's rows
// alive until the others have read them.  Inverse: the same steps backwards,
// the column results stored into the row owners' shared memory.
//
// HBM traffic is one read and one write of the plane (512 KB real, 528 KB
// complex), where the batched 2-D cuFFT makes two passes.  At 256^3 the pair
// still runs slower than cuFFT's (about 335 and 310 us against about 118 us
// a direction): with 133 KB of shared memory and 168 registers a CTA, one
// 8-warp CTA sits on an SM and the distributed-shared-memory reads and the
// phase barriers are not hidden (8 % of DRAM bandwidth).  So the solver keeps
// cuFFT and runs these kernels only under NOVA_FFT=cluster.
#include "nova_fft.cuh"
#include "nova_internal.cuh"
#include "nova_ops.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace nova {

namespace {

constexpr int kN = 256;            // N1 = N2
constexpr int kCL = 8;             // CTAs per cluster (rows split)
constexpr int kRows = kN / kCL;    // 32 rows per CTA
constexpr int kM = kN / 2;         // the complex length of a row, 128
constexpr int kNzh = kM + 1;       // 129 half-spectrum columns
constexpr int kSRow = kNzh;        // shared row stride (complex)
constexpr int kFThreads = 256;
constexpr int kChunk = 16;         // columns per phase-2 chunk
// shared memory: W_256 table | rows [32][129] | column scratch [16][256]
constexpr size_t kSmem = sizeof(double2) * ((size_t)kN + (size_t)kRows * kSRow + (size_t)kChunk * kN);

// kz columns of CTA r: 16 r .. 16 r + 15, the last CTA also 128
__device__ __forceinline__ int col_begin(int r) { return kChunk * r; }
__device__ __forceinline__ int col_count(int r) { return r == kCL - 1 ? kChunk + 1 : kChunk; }

__global__ void __cluster_dims__(kCL, 1, 1) __launch_bounds__(kFThreads, 1)
    k_fft2_fwd(const double *__restrict__ x, double2 *__restrict__ X, const double2 *__restrict__ twg)
{
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int i = blockIdx.y;
    const int t = threadIdx.x;
    extern __shared__ __align__(16) double2 smf[];
    double2 *tw = smf;               // W_256^m
    double2 *S = tw + kN;            // [row][kz]
    double2 *T = S + kRows * kSRow;  // [col][k1][n2]
    tw[t] = twg[t];

    // phase 1: the 32 rows, z[n] = (x[2n], x[2n+1]), contiguous in HBM
    const double2 *src = reinterpret_cast<const double2 *>(x + (size_t)i * kN * kN + (size_t)kRows * r * kN);
#pragma unroll 4
    for (int q = 0; q < kRows * kM / kFThreads; q++) {
        const int e = t + kFThreads * q;
        S[(e >> 7) * kSRow + (e & 127)] = src[e];
    }
    __syncthreads();
    // 128 = 8 x 16: n = n2 + 16 n1, k = k1 + 8 k2.  DFT-8 over n1, twiddle W_128^(n2 k1)
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int task = t + kFThreads * h, row = task >> 4, n2 = task & 15;
        double2 v[8];
        double2 *s = S + row * kSRow + n2;
#pragma unroll
        for (int n1 = 0; n1 < 8; n1++) v[n1] = s[16 * n1];
        dft<8, kN, false>(v, tw);
#pragma unroll
        for (int k1 = 0; k1 < 8; k1++) s[16 * k1] = k1 == 0 ? v[0] : cmul(v[k1], tw[2 * n2 * k1]);
    }
    __syncthreads();
    {  // DFT-16 over n2 -> Z[k1 + 8 k2]
        const int row = t >> 3, k1 = t & 7;
        double2 v[16];
        double2 *s = S + row * kSRow;
#pragma unroll
        for (int n2 = 0; n2 < 16; n2++) v[n2] = s[16 * k1 + n2];
        dft<16, kN, false>(v, tw);
        __syncthreads();
#pragma unroll
        for (int k2 = 0; k2 < 16; k2++) s[k1 + 8 * k2] = v[k2];
    }
    __syncthreads();
    // the real-to-complex split, pairs (k, 128 - k) in place; X[128] in column 128
    for (int task = t; task < kRows * 65; task += kFThreads) {
        const int row = task / 65, k = task % 65;
        double2 *s = S + row * kSRow;
        if (k == 0) {
            const double2 z = s[0];
            s[0] = make_double2(z.x + z.y, 0.0);
            s[kM] = make_double2(z.x - z.y, 0.0);
        } else if (k == kM / 2) {
            s[k] = conj2(s[k]);
        } else {
            const double2 a = s[k], b = s[kM - k];
            const double2 E = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
            const double2 O = make_double2(0.5 * (a.y + b.y), -0.5 * (a.x - b.x));  // (a - conj b) / 2i
            const double2 WO = cmul(O, tw[k]);
            s[k] = make_double2(E.x + WO.x, E.y + WO.y);
            s[kM - k] = make_double2(E.x - WO.x, -(E.y - WO.y));
        }
    }
    cl.sync();

    // phase 2: 256-point DFTs along j of this CTA's columns, 256 = 16 x 16:
    // j = n2 + 16 n1 (row j lives in CTA j / 32), frequency k1 + 16 k2
    const double2 *rem[kCL];
#pragma unroll
    for (int o = 0; o < kCL; o++) rem[o] = cl.map_shared_rank(S, o);
    const int c0 = col_begin(r), nct = col_count(r);
    double2 *dst = X + (size_t)i * kN * kNzh;
    for (int cs = 0; cs < nct; cs += kChunk) {
        const int nc = min(kChunk, nct - cs);
        for (int task = t; task < nc * 16; task += kFThreads) {
            const int col = task % nc, n2 = task / nc, kz = c0 + cs + col;
            double2 v[16];
#pragma unroll
            for (int n1 = 0; n1 < 16; n1++) {
                const int j = n2 + 16 * n1;
                v[n1] = rem[j >> 5][(j & 31) * kSRow + kz];
            }
            dft<16, kN, false>(v, tw);
            double2 *tc = T + col * kN + n2;
#pragma unroll
            for (int k1 = 0; k1 < 16; k1++) tc[16 * k1] = k1 == 0 ? v[0] : cmul(v[k1], tw[n2 * k1]);
        }
        __syncthreads();
        for (int task = t; task < nc * 16; task += kFThreads) {
            const int col = task % nc, k1 = task / nc, kz = c0 + cs + col;
            double2 v[16];
            const double2 *tc = T + col * kN + 16 * k1;
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) v[n2] = tc[n2];
            dft<16, kN, false>(v, tw);
#pragma unroll
            for (int k2 = 0; k2 < 16; k2++) dst[(size_t)(k1 + 16 * k2) * kNzh + kz] = v[k2];
        }
        __syncthreads();
    }
    cl.sync();  // the other CTAs have read these rows
}

__global__ void __cluster_dims__(kCL, 1, 1) __launch_bounds__(kFThreads, 1)
    k_fft2_inv(const double2 *__restrict__ X, double *__restrict__ x, const double2 *__restrict__ twg)
{
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int i = blockIdx.y;
    const int t = threadIdx.x;
    extern __shared__ __align__(16) double2 smf[];
    double2 *tw = smf;
    double2 *S = tw + kN;
    double2 *T = S + kRows * kSRow;
    tw[t] = twg[t];
    __syncthreads();

    // phase 1: inverse 256-point DFTs along j of this CTA's columns,
    // x[n2 + 16 n1] = sum_k1 W_256^-(n2 k1) W_16^-(n1 k1) sum_k2 X[k1 + 16 k2] W_16^-(n2 k2);
    // each result goes to the row owner's shared memory
    double2 *rem[kCL];
#pragma unroll
    for (int o = 0; o < kCL; o++) rem[o] = cl.map_shared_rank(S, o);
    const int c0 = col_begin(r), nct = col_count(r);
    const double2 *srcp = X + (size_t)i * kN * kNzh;
    cl.sync();  // every CTA's shared memory is live before the remote stores
    for (int cs = 0; cs < nct; cs += kChunk) {
        const int nc = min(kChunk, nct - cs);
        for (int task = t; task < nc * 16; task += kFThreads) {
            const int col = task % nc, k1 = task / nc, kz = c0 + cs + col;
            double2 v[16];
#pragma unroll
            for (int k2 = 0; k2 < 16; k2++) v[k2] = srcp[(size_t)(k1 + 16 * k2) * kNzh + kz];
            dft<16, kN, true>(v, tw);
            double2 *tc = T + col * kN + k1;
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) tc[16 * n2] = n2 == 0 ? v[0] : cmul(v[n2], conj2(tw[n2 * k1]));
        }
        __syncthreads();
        for (int task = t; task < nc * 16; task += kFThreads) {
            const int col = task % nc, n2 = task / nc, kz = c0 + cs + col;
            double2 v[16];
            const double2 *tc = T + col * kN + 16 * n2;
#pragma unroll
            for (int k1 = 0; k1 < 16; k1++) v[k1] = tc[k1];
            dft<16, kN, true>(v, tw);
#pragma unroll
            for (int n1 = 0; n1 < 16; n1++) {
                const int j = n2 + 16 * n1;
                rem[j >> 5][(j & 31) * kSRow + kz] = v[n1];
            }
        }
        __syncthreads();
    }
    cl.sync();  // the rows are complete

    // phase 2: complex-to-real along k per row.  Z[k] = (a + conj b) + i W^-k (a - conj b)
    // and Z[128-k] = (b + conj a) - i W^k (b - conj a), a = X[k], b = X[128-k]
    for (int task = t; task < kRows * 65; task += kFThreads) {
        const int row = task / 65, k = task % 65;
        double2 *s = S + row * kSRow;
        if (k == 0) {
            const double a = s[0].x, b = s[kM].x;  // the imaginary parts of DC and Nyquist are dropped
            s[0] = make_double2(a + b, a - b);
        } else if (k == kM / 2) {
            s[k] = make_double2(2.0 * s[k].x, -2.0 * s[k].y);
        } else {
            const double2 a = s[k], b = s[kM - k];
            const double2 P = make_double2(a.x + b.x, a.y - b.y);   // a + conj b
            const double2 D = make_double2(a.x - b.x, a.y + b.y);   // a - conj b
            const double2 Wd = cmul(D, conj2(tw[k]));             // W^-k (a - conj b)
            s[k] = make_double2(P.x - Wd.y, P.y + Wd.x);          // P + i Wd
            // b + conj a = conj P, b - conj a = -conj D, W^k (-conj D) = -conj(W^-k D) = -conj Wd
            s[kM - k] = make_double2(P.x + Wd.y, -P.y + Wd.x);    // conj P + i conj Wd
        }
    }
    __syncthreads();
    // inverse 128-point FFT: Z index k1 + 8 k2, output n2 + 16 n1
    {  // inverse DFT-16 over k2 -> n2, twiddle W_128^-(n2 k1)
        const int row = t >> 3, k1 = t & 7;
        double2 v[16];
        double2 *s = S + row * kSRow;
#pragma unroll
        for (int k2 = 0; k2 < 16; k2++) v[k2] = s[k1 + 8 * k2];
        dft<16, kN, true>(v, tw);
        __syncthreads();
#pragma unroll
        for (int n2 = 0; n2 < 16; n2++) s[16 * k1 + n2] = n2 == 0 ? v[0] : cmul(v[n2], conj2(tw[2 * n2 * k1]));
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; h++) {  // inverse DFT-8 over k1 -> n1: z[n2 + 16 n1]
        const int task = t + kFThreads * h, row = task >> 4, n2 = task & 15;
        double2 v[8];
        double2 *s = S + row * kSRow + n2;
#pragma unroll
        for (int k1 = 0; k1 < 8; k1++) v[k1] = s[16 * k1];
        dft<8, kN, true>(v, tw);
#pragma unroll
        for (int n1 = 0; n1 < 8; n1++) s[16 * n1] = v[n1];
    }
    __syncthreads();
    double2 *dst = reinterpret_cast<double2 *>(x + (size_t)i * kN * kN + (size_t)kRows * r * kN);
#pragma unroll 4
    for (int q = 0; q < kRows * kM / kFThreads; q++) {
        const int e = t + kFThreads * q;
        dst[e] = S[(e >> 7) * kSRow + (e & 127)];
    }
}

// the kernels' shared-memory attribute, and whether a cluster of eight such
// CTAs can be resident on this device (else the caller keeps cuFFT)
bool cluster_ok()
{
    static int ok = -1;
    if (ok >= 0) return ok == 1;
    ok = 0;
    if (cudaFuncSetAttribute(k_fft2_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_fft2_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem) != cudaSuccess)
        return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kCL, 1, 1);
    cfg.blockDim = dim3(kFThreads, 1, 1);
    cfg.dynamicSmemBytes = kSmem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kCL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n1 = 0, n2 = 0;
    if (cudaOccupancyMaxActiveClusters(&n1, k_fft2_fwd, &cfg) != cudaSuccess ||
        cudaOccupancyMaxActiveClusters(&n2, k_fft2_inv, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    ok = (n1 > 0 && n2 > 0) ? 1 : 0;
    return ok == 1;
}

}  // namespace

bool fft2_fits(const Geo &g) { return !g.wallY && g.N1 == kN && g.N2 == kN && cluster_ok(); }

void launch_fft2_fwd(const Geo &g, const double *x, void *spec, const double *tw256, cudaStream_t st)
{
    k_fft2_fwd<<<dim3(kCL, g.N0), kFThreads, kSmem, st>>>(x, (double2 *)spec, (const double2 *)tw256);
}

void launch_fft2_inv(const Geo &g, const void *spec, double *x, const double *tw256, cudaStream_t st)
{
    k_fft2_inv<<<dim3(kCL, g.N0), kFThreads, kSmem, st>>>((const double2 *)spec, x, (const double2 *)tw256);
}

}  // namespace nova
