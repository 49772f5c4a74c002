// Internal declarations shared by the CUDA translation units of libnova_b200.
//
// Device layout: every field is component-major over the unique nodes,
// [c][i][j][k] with k (z) fastest -- the reference Field<T> index order
// k + j*nk + i*nk*nj (src/Field/Field.h:82-85) without ghosts and without the
// duplicated periodic node.  Periodic ghosts are synthesised in the kernels by
// index wrapping (src/BC/periodicBC.hxx:1-66 becomes address arithmetic).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace nova {

constexpr int kTK = 32;   // tile extent along k (one warp, coalesced)
constexpr int kTJ = 8;    // tile extent along j
constexpr int kThreads = kTK * kTJ;

// N1 is the number of stored y nodes: N[1] when y is periodic, N[1] + 1 when
// y is bounded by walls (both wall nodes stored, as in the reference's
// interior range [m/2, n - m/2)).
struct Geo {
    int N0, N1, N2;
    long long N12, N3;
    int wallY;
};

// Ghosts beyond the y walls of the halo'd components, evaluated with the
// reference's own expressions (src/BC/neumannBC.hxx, src/BC/dirichletBC.hxx)
// for the l-th ghost and its mirror node f:
//   Neumann:   f - 2 l val dy     (both faces, as the reference writes it)
//   Dirichlet: 2 l val - f
// side 0 = south face (j = 0), side 1 = north face (j = N1 - 1).
template <typename T> struct Walls {
    int on;
    int dir[2][9];  // 1 = Dirichlet, 0 = Neumann
    T val[2][9];
    T dy;
};

// rounded like the reference's host code: every product and difference
// rounded separately (no fused multiply-add)
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ T wall_ghost(const Walls<T> &w, int side, int c, int l, T f)
{
    // selects instead of a runtime index keep the parameters in the constant bank
    const int dir = side == 0 ? w.dir[0][c] : w.dir[1][c];
    const T val = side == 0 ? w.val[0][c] : w.val[1][c];
    const T tv = rn_mul((T)2.0 * (T)l, val);
    return dir ? rn_sub(tv, f) : rn_sub(f, rn_mul(tv, w.dy));
}

// First/second-derivative weights of src/settings/settings.cpp:25-31 for half
// width H, per direction d: a[d][l] = c_l / (2 (l+1) delta_d) (grad.cpp:46),
// b[d][l] = c_l / ((l+1) delta_d)^2 (laplacian.hxx:153), b2[d] = 2 sum_l b[d][l].
template <typename T> struct Coef {
    T a[3][4];
    T b[3][4];
    T b2[3];
};

// Per-launch weights of the fused advection-diffusion sum of the Navier-Stokes
// stage (nova_stage_math.cuh): ha = a/2 per direction, vb = visc * b for x and
// y (the z weights are scaled per node by the metric).
template <typename T> struct StageCoef {
    T ha[3][4];
    T vb[2][4];
};

template <typename T> inline StageCoef<T> stage_coef(const Coef<T> &co, T visc)
{
    StageCoef<T> s{};
    for (int d = 0; d < 3; d++)
        for (int l = 0; l < 4; l++) {
            s.ha[d][l] = co.a[d][l] * T(0.5);
            if (d < 2) s.vb[d][l] = visc * co.b[d][l];
        }
    return s;
}

__host__ __device__ inline int wrapi(int x, int n)
{
    int r = x % n;
    return r < 0 ? r + n : r;
}

// ------------------------------------------------------------------ stencil math --
// `v(c, s)` returns component c at offset s (-H..H) along the current direction.

template <typename T, int H, class V>
__device__ __forceinline__ T d1(const V &v, int c, const T *a)
{
    T r = a[0] * (v(c, 1) - v(c, -1));
#pragma unroll
    for (int l = 1; l < H; l++) r = fma(a[l], v(c, l + 1) - v(c, -l - 1), r);
    return r;
}

// derivative of the product v_c1 * v_c2
template <typename T, int H, class V>
__device__ __forceinline__ T d1p(const V &v, int c1, int c2, const T *a)
{
    T r = a[0] * (v(c1, 1) * v(c2, 1) - v(c1, -1) * v(c2, -1));
#pragma unroll
    for (int l = 1; l < H; l++) r = fma(a[l], v(c1, l + 1) * v(c2, l + 1) - v(c1, -l - 1) * v(c2, -l - 1), r);
    return r;
}

template <typename T, int H, class V>
__device__ __forceinline__ T d2(const V &v, int c, const T *b, T b2)
{
    T r = b[0] * (v(c, 1) + v(c, -1));
#pragma unroll
    for (int l = 1; l < H; l++) r = fma(b[l], v(c, l + 1) + v(c, -l - 1), r);
    return fma(-b2, v(c, 0), r);
}

// A_d(V,F)_c = sum_l a_l [ F_c(+l) (V_d(+l) + V_d(0)) - F_c(-l) (V_d(-l) + V_d(0)) ]
//            = D_d(V_d F_c) + V_d(0) D_d F_c;  cf = component of F, cv = V_d, v0 = V_d(0)
template <typename T, int H, class V>
__device__ __forceinline__ T adv1(const V &v, int cf, int cv, T v0, const T *a)
{
    T r = a[0] * (v(cf, 1) * (v(cv, 1) + v0) - v(cf, -1) * (v(cv, -1) + v0));
#pragma unroll
    for (int l = 1; l < H; l++)
        r = fma(a[l], v(cf, l + 1) * (v(cv, l + 1) + v0) - v(cf, -l - 1) * (v(cv, -l - 1) + v0), r);
    return r;
}

// sum_l b_l (f(+l) + f(-l)); the centre term of the Laplacian is added once for all directions
template <typename T, int H, class V>
__device__ __forceinline__ T lsum(const V &v, int c, const T *b)
{
    T r = b[0] * (v(c, 1) + v(c, -1));
#pragma unroll
    for (int l = 1; l < H; l++) r = fma(b[l], v(c, l + 1) + v(c, -l - 1), r);
    return r;
}

// ------------------------------------------------------------- launch helpers --
struct StageArgs64 {
    const double *Y;   // halo'd stage state (3 comps)
    const double *X;   // second halo'd field (MHD), else nullptr
    const double *U0;  // RK base (stages 1, 2, 5)
    double *A;         // RK accumulator
    double *Ynext;     // next stage state, or U* after the last stage (stage 5: U*)
    double w;          // stage 5: the stage's weight
};

struct StageArgs32 {
    const float *Y;      // halo'd stage state (3 comps, FP32)
    const float *X;      // second halo'd field hi part (MHD)
    const float *U0hi;   // base hi
    const float *U0lo;   // base lo (last stage / literal / stage 5)
    float *A;            // FP32 increment accumulator
    float *Ynext;        // next stage state (FP32)
    float *outhi, *outlo;  // U* (last stage / literal / stage 5)
    float w;             // stage 5: the stage's weight
    double *out64;       // U* in FP64 instead of (outhi, outlo) (stages 3, 4, 5) when non-null
};

enum Physics { PHYS_NS = 0, PHYS_MHD_U = 1, PHYS_MHD_B = 2 };

// reverse RK4 stage of the discrete adjoint (nova_adjoint.cu)
// block-wide sum / max (blockDim.x a multiple of 32, sh >= 32 entries); the
// result is valid in thread 0
template <typename T>
__device__ __forceinline__ T block_reduce_sum(T v, T *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) r += sh[q];
    return r;
}

template <typename T>
__device__ __forceinline__ T block_reduce_max(T v, T *sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) r = fmax(r, sh[q]);
    return r;
}

struct AdjArgs {
    const double *Y;    // forward stage state Y_s (3 comps, halo'd)
    const double *G;    // adjoint stage direction g_s (halo'd); mu itself at s = 4
    const double *mu;   // projected adjoint of U*
    const double *Lam;  // running sum of xi (s < 4)
    double *Gout;       // g_{s-1}, or dJ/dU at s = 1
    double *LamOut;     // updated running sum (s > 1)
};
// err: the pipeline error word; with it, meshes that fit the TMA adjoint
// (nova_adj_tma.cu: periodic, N2 % 32 == 0, N1 a multiple of 8 and >= 16) run it
cudaError_t launch_adj_stage64(int s, const Geo &g, const Coef<double> &co, const double *ia, double dt, double nu,
                               const AdjArgs &a, cudaStream_t st, int *err = nullptr);
bool adj_tma_fits(const Geo &g);
// kind: 0, 1, 2 = the MHD pieces of launch_adj_mhd (acc: the adjoint they add
// into), 3 = the Navier-Stokes stage
cudaError_t launch_adj_tma64(int kind, int s, const Geo &g, const Coef<double> &co, const double *ia, double dt,
                             double nu, const AdjArgs &a, double *acc, int *err, cudaStream_t st);
// FP32-split adjoint stage: FP32 stage states, directions and running sum;
// mu (and dJ/dU, written to `lam` at s = 1) in FP64
struct AdjArgs32 {
    const float *Y;
    const float *G;      // g_s (s < 4)
    const double *mu;    // projected adjoint of U*
    const float *Lam;
    float *Gout;         // g_{s-1} (s > 1)
    float *LamOut;
    double *lam;         // dJ/dU (s = 1)
};
void launch_adj_stage32(int s, const Geo &g, const Coef<float> &co, const float *ia, float dt, float nu,
                        const AdjArgs32 &a, cudaStream_t st);
// FP32 MHD coupling transposes (tiled): kind 0, 1, 2 as launch_adj_mhd; acc FP64
void launch_adj_mhd32(int kind, int s, const Geo &g, const Coef<float> &co, const float *ia, float dt, float visc,
                      const AdjArgs32 &a, double *acc, cudaStream_t st);
// MHD adjoint stage pieces (nova_adjoint.cu, nova_adj_tma.cu): kind 0 = dF_U/dB
// (lambda_B += ...), 1 = dF_B/dU (lambda_U += ...), 2 = dF_B/dB with the
// reverse RK4 recursion; a.Y = the field in the transpose (B^n, Z_S or
// U^{n+1}), a.G = g_S; at s = 4 the direction is mu/6 and a.mu and a.G are mu
cudaError_t launch_adj_mhd(int kind, int s, const Geo &g, const Coef<double> &co, const double *ia, double dt,
                           double visc, const AdjArgs &a, double *acc, cudaStream_t st, int *err = nullptr);
void launch_scale_copy(long long n, double a, const double *x, double *y, cudaStream_t st);  // y = a x
void launch_axpy(long long n, double a, const double *x, double *y, cudaStream_t st);        // y += a x
// *out = scale * sum_t x[t] y[t] (nb blocks of partials in part)
void launch_dot(long long n, const double *x, const double *y, double scale, double *part, int nb, double *out,
                cudaStream_t st);

// Which kernel runs the Navier-Stokes stage: STAGE_AUTO = the TMA pipeline
// (nova_stage_tma.cu) where the mesh fits it (stage_tma_fits: N2 % 32 == 0,
// N1 at least twice the tile height 16 (FP64) or 8 (FP32), and with periodic y
// a multiple of it; FP32 walls in y take ragged last tiles), else the
// register-queue march (nova_stage.cu); STAGE_MARCH / STAGE_TMA force one
// (STAGE_TMA on a mesh that does not fit is an error).  err: device word
// raised by a pipeline wait that timed out.
enum StageImpl { STAGE_AUTO = 0, STAGE_MARCH = 1, STAGE_TMA = 2 };
struct StageExec {
    int impl;
    int *err;
};
bool stage_tma_fits(const Geo &g, bool fp64);
// tensor map of a 3-component FP64 field [c][i][j][k] (nova_stage_tma.cu):
// rows > 0: box kTK(k) x 3(c) x rows(j) x 1(i), landing [row][c][k];
// rows = 0: the 4-wide k-halo box 4(k) x 8(j) x 3(c) x 1(i), landing [c][j][k]
bool tma_encode_field(CUtensorMap *m, const double *base, const Geo &g, unsigned rows);
// The per-block diagnostics partials, kDiagParts doubles per block: sums over
// the unique nodes of 1/2|U|^2, 1/2|B|^2, |ex::curl(U)|, |ex::curl(B)| and the
// central 1/2|curl U|^2, 1/2|curl B|^2; maxima of |div U| and |div B| over
// every stored node, of |ex::curl(B)| and |U| over the unique nodes, and of
// U_x (from 0, signed) over every stored node (tools::CFL's cfl_x).
enum DiagPart {
    DP_EK = 0, DP_EM, DP_OMEGA, DP_JAV, DP_ENSU, DP_ENSB,  // sums
    DP_DIVU, DP_DIVB, DP_JMAX, DP_UMAX, DP_UX, DP_SPARE,  // maxima
    kDiagParts
};
// What the history row needs besides the partials (k_diag_final): the row's
// step and time, 1/(number of unique nodes), the viscosities of epsilon, and
// dt and the mesh spacing with the state itself for tools::CFL (the last node
// of its loop, (N0, N1, N2) of the reference's interior, is the stored node
// `last`).
struct DiagFinal {
    double invN3, step, time;
    double nu, eta, dt, dx, dy, dz;
    const double *U64;
    const float *Uhi, *Ulo;
    long long N3, last;
};
// diagnostics of a stage's input state taken by the stage itself (FP64 TMA
// stage 0 or literal stage 4, uniform periodic mesh): per-block partials into
// part (room for cap blocks), then the history row (k_diag_final)
struct StageDiag {
    double *part;
    int cap;
    double *row;
    int *flag;
    DiagFinal fin;
};
cudaError_t launch_stage_tma64(int stage, bool stretch, const Geo &g, const Walls<double> &wl, const Coef<double> &co,
                               const double *ia, const double *corr2, double dt, double visc, const StageArgs64 &a,
                               int *err, cudaStream_t st, const StageDiag *dg = nullptr, bool *dg_done = nullptr);
// MHD stage kernels on the TMA pipeline (nova_stage_mhd_tma.cu): periodic y,
// N2 % 32 == 0, N1 a multiple of the tile height 8 (FP64) or 16 (FP32) and at
// least twice it; a.X is the frozen field
bool mhd_tma_fits(const Geo &g, bool fp64);
cudaError_t launch_mhd_tma64(int phys, int stage, bool stretch, const Geo &g, const Coef<double> &co, const double *ia,
                             const double *corr2, double dt, double visc, const StageArgs64 &a, int *err,
                             cudaStream_t st);
cudaError_t launch_mhd_tma32(int phys, int stage, bool stretch, const Geo &g, const Coef<float> &co, const float *ia,
                             const float *corr2, float dt, float visc, const StageArgs32 &a, int *err,
                             cudaStream_t st);
cudaError_t launch_stage_tma32(int stage, bool stretch, const Geo &g, const Walls<float> &wl, const Coef<float> &co,
                               const float *ia, const float *corr2, float dt, float visc, const StageArgs32 &a,
                               int *err, cudaStream_t st);

// stage: 0..3 classical RK4 stages, 4 = literal reference loop (one RHS, 4-term sum),
// 5 = the shear-layer loop's stage U* = U0 + w dU (app/shearLayer/UEqn.H:28-29)
// stretch: apply the stretched-z Laplacian term (Mesh "hypz:"); on uniform
// meshes d2zdxi2 is round-off (|.| < 1e-9) and the term is skipped
// Returns cudaErrorNotSupported when STAGE_TMA is forced on a mesh it does not
// fit, cudaErrorInvalidValue when a tensor map cannot be encoded.
cudaError_t launch_stage64(int phys, int stage, bool stretch, const Geo &g, const Walls<double> &wl,
                           const Coef<double> &co, const double *ia, const double *corr2, double dt, double visc,
                           const StageArgs64 &a, cudaStream_t st, const StageExec &ex, const StageDiag *dg = nullptr,
                           bool *dg_done = nullptr);
cudaError_t launch_stage32(int phys, int stage, bool stretch, const Geo &g, const Walls<float> &wl,
                           const Coef<float> &co, const float *ia, const float *corr2, float dt, float visc,
                           const StageArgs32 &a, cudaStream_t st, const StageExec &ex);

}  // namespace nova
