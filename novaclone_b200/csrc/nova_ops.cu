// Projection, diagnostics, drop-in ex:: operators and layout conversion.
//
// Projection (app/TG_Piosson/RKLoop.H:30-38, app/OT_Poisson/BEqn.H:91-95):
//   rhs = div(U*) / dt                       k_div_tiled   (src/ex/div/div.hxx:22-81)
//   rhs^ = D2Z(rhs)                          cuFFT         (src/poisson/poisson.cpp:225)
//   rhs^ = -rhs^ / k'^2 / (N0 N1 N2)         k_scale       (poisson.cpp:230-249, 259)
//   p = Z2D(rhs^)                            cuFFT         (poisson.cpp:250)
//   U = U* - dt * grad(p)                    k_correct_tiled (src/ex/grad/grad.cpp:25-62)
// k'^2 is built from 1-D tables of squared modified wavenumbers
// (poisson::wavenumbersFFT_, poisson.cpp:337-396) summed in the reference's order.
#include "nova_gpu.h"
#include "nova_internal.cuh"
#include "nova_diag.cuh"
#include "nova_ops.cuh"
#include "nova_tile.cuh"

#include <cuComplex.h>


namespace nova {

namespace {

struct Ld64 {
    const double *p;
    long long n3;
    Walls<double> wl;  // y-wall ghosts of this field (wl.on = 0: periodic)
    __device__ double operator()(int c, long long o) const { return p[(long long)c * n3 + o]; }
};
struct LdSplit {
    const float *hi, *lo;
    long long n3;
    Walls<double> wl;
    __device__ double operator()(int c, long long o) const
    {
        return (double)hi[(long long)c * n3 + o] + (double)lo[(long long)c * n3 + o];
    }
};

// value of component c of f at (i,j,k) shifted by s along direction d:
// periodic axes wrap, y walls mirror with the field's ghost formulas
template <typename P>
__device__ __forceinline__ double at(const P &f, const Geo &g, int c, int i, int j, int k, int d, int s)
{
    if (d == 0) {
        i = wrapi(i + s, g.N0);
    } else if (d == 2) {
        k = wrapi(k + s, g.N2);
    } else {
        const int jj = j + s;
        if (f.wl.on && (jj < 0 || jj >= g.N1)) {
            const int side = jj < 0 ? 0 : 1;
            const int l = side == 0 ? -jj : jj - (g.N1 - 1);
            const int jm = side == 0 ? l : (g.N1 - 1) - l;
            return wall_ghost(f.wl, side, c, l, f(c, (long long)i * g.N12 + (long long)jm * g.N2 + k));
        }
        j = f.wl.on ? jj : wrapi(jj, g.N1);
    }
    return f(c, (long long)i * g.N12 + (long long)j * g.N2 + k);
}

__device__ __forceinline__ void pt_index(const Geo &g, long long t, int &i, int &j, int &k)
{
    k = (int)(t % g.N2);
    long long r = t / g.N2;
    j = (int)(r % g.N1);
    i = (int)(r / g.N1);
}

// first derivative along d of component c with weights a (already metric-scaled)
template <int H, typename P>
__device__ __forceinline__ double dd1(const P &f, const Geo &g, int c, int i, int j, int k, int d, const double *a)
{
    double r = 0.0;
#pragma unroll
    for (int l = 0; l < H; l++) r = fma(a[l], at(f, g, c, i, j, k, d, l + 1) - at(f, g, c, i, j, k, d, -l - 1), r);
    return r;
}

__global__ void k_scale(Geo g, int ny, cuDoubleComplex *__restrict__ spec, const double *__restrict__ kx2,
                        const double *__restrict__ ky2, const double *__restrict__ kz2, double invN3)
{
    const int nzh = g.N2 / 2 + 1;
    const long long tot = (long long)g.N0 * ny * nzh;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= tot) return;
    const int kz = (int)(t % nzh);
    const long long r = t / nzh;
    const int j = (int)(r % ny);
    const int i = (int)(r / ny);
    const double k2 = (kx2[i] + ky2[j]) + kz2[kz];
    cuDoubleComplex v = spec[t];
    if (k2 < 1.0e-16) {
        v = make_cuDoubleComplex(0.0, 0.0);
    } else {
        v = make_cuDoubleComplex((-v.x / k2) * invN3, (-v.y / k2) * invN3);
    }
    spec[t] = v;
}

// rhs = div(U*)/divisor and U = U* - s*grad(p): the 2.5-D march of nova_tile.cuh
// (register queue along i, shared plane for j/k), one read of each input.
template <int H, class LD, bool WALLS>
__global__ void __launch_bounds__(kThreads) k_div_tiled(Geo g, Coef<double> co, const double *__restrict__ ia, LD U,
                                                        double divisor, double *__restrict__ rhs, int ichunk)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, H, 3> *>(smraw);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[kw];
    tile_march<double, H, 3, WALLS>(g, U.wl, sm, U, ib, ie, [&](long long idx, auto &, const auto &vx, const auto &vy,
                                                          const auto &vz) {
        const double d = d1<double, H>(vx, 0, co.a[0]) + d1<double, H>(vy, 1, co.a[1]) + d1<double, H>(vz, 2, az);
        rhs[idx] = d / divisor;
    });
}

template <int H, bool SPLIT, bool WALLS>
__global__ void __launch_bounds__(kThreads) k_correct_tiled(Geo g, Walls<double> pw, Coef<double> co,
                                                            const double *__restrict__ ia, const double *__restrict__ p,
                                                            double s, const double *Us64, double *U64,
                                                            const float *Ushi, const float *Uslo, float *hi, float *lo,
                                                            int ichunk)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, H, 1> *>(smraw);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[kw];
    auto ld = [&](int, long long o) { return p[o]; };
    tile_march<double, H, 1, WALLS>(g, pw, sm, ld, ib, ie, [&](long long idx, auto &, const auto &vx, const auto &vy,
                                                          const auto &vz) {
        double us[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long o = c * g.N3 + idx;
            us[c] = (SPLIT && !Us64) ? (double)Ushi[o] + (double)Uslo[o] : Us64[o];
        }
        const double gr[3] = {d1<double, H>(vx, 0, co.a[0]), d1<double, H>(vy, 0, co.a[1]), d1<double, H>(vz, 0, az)};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long o = c * g.N3 + idx;
            const double x = us[c] - gr[c] * s;
            if constexpr (SPLIT) {
                const float h = (float)x;
                hi[o] = h;
                lo[o] = (float)(x - (double)h);
            } else {
                U64[o] = x;
            }
        }
    });
}

// Wall Poisson by the even extension in y (a DCT-I of the N1+1 node-based
// rows): ext has 2*ny rows, ext[j] = rhs[j] for j <= ny and ext[2 ny - j] =
// rhs[j] for 0 < j < ny.  The mirror image of a field with Neumann-0 ghosts
// is exactly this even extension, so the periodic solve on the doubled
// domain inverts D.G with the wall ghosts the stencils use.
__global__ void k_even_extend(Geo g, int ny, const double *__restrict__ rhs, double *__restrict__ ext)
{
    const long long tot = (long long)g.N0 * 2 * ny * g.N2;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= tot) return;
    const int k = (int)(t % g.N2);
    const long long r = t / g.N2;
    const int jj = (int)(r % (2 * ny));
    const int i = (int)(r / (2 * ny));
    const int j = jj <= ny ? jj : 2 * ny - jj;
    ext[t] = rhs[(long long)i * g.N12 + (long long)j * g.N2 + k];
}

__global__ void k_restrict_rows(Geo g, int ny, const double *__restrict__ ext, double *__restrict__ p)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    const int k = (int)(t % g.N2);
    const long long r = t / g.N2;
    const int j = (int)(r % g.N1);
    const int i = (int)(r / g.N1);
    p[t] = ext[((long long)i * 2 * ny + j) * g.N2 + k];
}

// ------------------------------------------------------------- diagnostics --
constexpr int kRedThreads = 256;


// The history row's per-block partials (DiagPart, kDiagParts per block).
// Means and |U|, |curl B| maxima cover the unique nodes as app/OT_Poisson/OT.cpp:136-155
// does (the stored north-wall row is the reference's last node and is skipped);
// the divergence maxima and U_x cover every stored node (tools::maximum,
// src/Tools/Tools.h:19-36; tools::CFL, src/Tools/Tools.cpp:15-25).
template <int H, int NC, class LD, bool WALLS>
__global__ void __launch_bounds__(kThreads, NC == 3 ? 2 : 1) k_diag_tiled(Geo g, Walls<double> wl, Coef<double> co,
                                                         const double *__restrict__ ia, LD U, LD B, int ichunk,
                                                         double *__restrict__ part)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, H, NC> *>(smraw);
    __shared__ double red[kDiagParts][kThreads / 32];
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[kw];
    const int rows_e = g.N1 - g.wallY;
    DiagAcc acc;
    auto ld = [&](int c, long long o) -> double { return c < 3 ? U(c, o) : B(c - 3, o); };
    tile_march<double, H, NC, WALLS>(g, wl, sm, ld, ib, ie, [&](long long idx, auto &q, const auto &vx, const auto &vy,
                                                          const auto &vz) {
        const int j = (int)((idx % g.N12) / g.N2);
        const bool ce = j < rows_e;
        const double u[3] = {q[H][0], q[H][1], q[H][2]};
        const double du = d1<double, H>(vx, 0, co.a[0]) + d1<double, H>(vy, 1, co.a[1]) + d1<double, H>(vz, 2, az);
        double q1, hs;
        curl_terms<H>(vx, vy, vz, 0, co.a[0], co.a[1], az, 1.0, q1, hs);
        acc.add_u(u, du, q1, hs, ce);
        if constexpr (NC == 6) {
            const double b[3] = {q[H][3], q[H][4], q[H][5]};
            const double db = d1<double, H>(vx, 3, co.a[0]) + d1<double, H>(vy, 4, co.a[1]) + d1<double, H>(vz, 5, az);
            curl_terms<H>(vx, vy, vz, 3, co.a[0], co.a[1], az, 1.0, q1, hs);
            acc.add_b(b, db, q1, hs, ce);
        }
    });
    const int tid = threadIdx.y * kTK + threadIdx.x, lane = tid & 31, w = tid >> 5;
    acc.warp_reduce();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < kDiagParts; q++) red[q][w] = acc.v[q];
    __syncthreads();
    if (tid < kDiagParts) {
        double a = 0.0;
        for (int x = 0; x < kThreads / 32; x++) a = tid >= DP_DIVU ? fmax(a, red[tid][x]) : a + red[tid][x];
        const long long blk = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        part[blk * kDiagParts + tid] = a;
    }
}

// std::max(a, b) of the reference: b only when a < b
__device__ __forceinline__ double ref_max(double a, double b) { return a < b ? b : a; }

__global__ void k_diag_final(const double *__restrict__ part, int nblk, DiagFinal fin, double *__restrict__ row,
                             int *__restrict__ flag)
{
    __shared__ double sh[32];
    double tot[kDiagParts];
#pragma unroll
    for (int q = 0; q < kDiagParts; q++) {
        double a = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x)
            a = q >= DP_DIVU ? fmax(a, part[(long long)b * kDiagParts + q]) : a + part[(long long)b * kDiagParts + q];
        tot[q] = q >= DP_DIVU ? block_reduce_max(a, sh) : block_reduce_sum(a, sh);
    }
    if (threadIdx.x == 0) {
        const double n = fin.invN3;
        const double om = tot[DP_OMEGA] * n, jav = tot[DP_JAV] * n;
        // tools::CFL: cfl_x = max over the nodes of U_x dt / dx (from 0); cfl_y,
        // cfl_z = std::max(cfl_x, U dt / d) at the loop's last node
        auto last = [&](int c) -> double {
            const long long o = (long long)c * fin.N3 + fin.last;
            return fin.U64 ? fin.U64[o] : (double)fin.Uhi[o] + (double)fin.Ulo[o];
        };
        const double cx = tot[DP_UX] * fin.dt / fin.dx;
        row[0] = fin.step;
        row[1] = fin.time;
        row[2] = tot[DP_EK] * n;
        row[3] = tot[DP_EM] * n;
        row[4] = tot[DP_DIVU];
        row[5] = tot[DP_DIVB];
        row[6] = om;
        row[7] = jav;
        row[8] = tot[DP_JMAX];
        row[9] = -fin.nu * (om * om) - fin.eta * (jav * jav);
        row[10] = tot[DP_UMAX];
        row[11] = cx;
        row[12] = ref_max(cx, last(1) * fin.dt / fin.dy);
        row[13] = ref_max(cx, last(2) * fin.dt / fin.dz);
        row[14] = tot[DP_ENSU] * n;
        row[15] = tot[DP_ENSB] * n;
        bool bad = false;
        for (int q = 0; q < kDiagParts; q++) bad = bad || !isfinite(tot[q]);
        if (bad) atomicExch(flag, 1);
    }
}

template <class LD>
__global__ void k_maxabs_part(long long n, LD f, double *__restrict__ part)
{
    __shared__ double sh[32];
    double m = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(f(0, t)));
    m = block_reduce_max(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

__global__ void k_max_final(const double *__restrict__ part, int n, double *__restrict__ out)
{
    __shared__ double sh[32];
    double m = 0.0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) m = fmax(m, part[q]);
    m = block_reduce_max(m, sh);
    if (threadIdx.x == 0) *out = m;
}

// one partial per fixed chunk of kMaxabsChunk nodes (no grid-stride loop, so the
// number of partials is the size the static scratch has to hold)
__global__ void __launch_bounds__(256) k_maxabs_chunks(long long n, const double *__restrict__ s,
                                                       double *__restrict__ part)
{
    __shared__ double sh[32];
    const long long b = (long long)blockIdx.x * kMaxabsChunk;
    const long long e = min(b + (long long)kMaxabsChunk, n);
    double m = 0.0;
    for (long long t = b + threadIdx.x; t < e; t += blockDim.x) m = fmax(m, fabs(s[t]));
    m = block_reduce_max(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

// --------------------------------------------------------------- operators --
// Simple one-thread-per-node kernels for the drop-in ex:: entry points.

template <int H>
__global__ void k_op_grad_s(Geo g, Walls<double> wa, Coef<double> co, const double *__restrict__ ia, const double *__restrict__ s,
                            double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 S{s, g.N3, wa};
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[k];
    out[t] = dd1<H>(S, g, 0, i, j, k, 0, co.a[0]);
    out[g.N3 + t] = dd1<H>(S, g, 0, i, j, k, 1, co.a[1]);
    out[2 * g.N3 + t] = dd1<H>(S, g, 0, i, j, k, 2, az);
}

// ex::grad(Field<vector>) keeps the reference's stencil c_l/(l+1)/delta*(f(+l) - f(-1-l)) (grad.cpp:82-94)
template <int H>
__global__ void k_op_grad_v(Geo g, Walls<double> wa, Coef<double> co, const double *__restrict__ ia, const double *__restrict__ U,
                            double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 F{U, g.N3, wa};
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double r = 0.0;
#pragma unroll
            for (int l = 0; l < H; l++) {
                double w = 2.0 * co.a[d][l];  // c_l/(l+1)/delta
                if (d == 2) w *= ia[k];
                r = fma(w, at(F, g, c, i, j, k, d, l) - at(F, g, c, i, j, k, d, -1 - l), r);
            }
            out[(long long)(3 * c + d) * g.N3 + t] = r;
        }
}

// ex::curl = antisymmetric part of ex::grad(vector) (src/ex/curl/curl.cpp:44-50)
template <int H>
__global__ void k_op_curl(Geo g, Walls<double> wa, Coef<double> co, const double *__restrict__ ia, const double *__restrict__ U,
                          double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 F{U, g.N3, wa};
    auto gv = [&](int c, int d) {
        double r = 0.0;
#pragma unroll
        for (int l = 0; l < H; l++) {
            double w = 2.0 * co.a[d][l];
            if (d == 2) w *= ia[k];
            r = fma(w, at(F, g, c, i, j, k, d, l) - at(F, g, c, i, j, k, d, -1 - l), r);
        }
        return r;
    };
    out[t] = gv(2, 1) - gv(1, 2);
    out[g.N3 + t] = gv(0, 2) - gv(2, 0);
    out[2 * g.N3 + t] = gv(1, 0) - gv(0, 1);
}

template <int H>
__global__ void k_op_div_v(Geo g, Walls<double> wa, Coef<double> co, const double *__restrict__ ia, const double *__restrict__ U,
                           double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 F{U, g.N3, wa};
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[k];
    out[t] = dd1<H>(F, g, 0, i, j, k, 0, co.a[0]) + dd1<H>(F, g, 1, i, j, k, 1, co.a[1])
             + dd1<H>(F, g, 2, i, j, k, 2, az);
}

// skew div(U, f), f with nc components (src/ex/div/div.hxx:84-172)
template <int H>
__global__ void k_op_div_vf(Geo g, Walls<double> wa, Walls<double> wb, Coef<double> co, const double *__restrict__ ia, const double *__restrict__ U,
                            const double *__restrict__ f, int nc, double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 V{U, g.N3, wa}, F{f, g.N3, wb};
    double a[3][H];
#pragma unroll
    for (int l = 0; l < H; l++) {
        a[0][l] = co.a[0][l];
        a[1][l] = co.a[1][l];
        a[2][l] = co.a[2][l] * ia[k];
    }
    double divU = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) divU += dd1<H>(V, g, d, i, j, k, d, a[d]);
    for (int c = 0; c < nc; c++) {
        const double f0 = F(c, t);
        double acc = f0 * divU;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double dq = 0.0;
#pragma unroll
            for (int l = 0; l < H; l++)
                dq = fma(a[d][l],
                         at(V, g, d, i, j, k, d, l + 1) * at(F, g, c, i, j, k, d, l + 1)
                             - at(V, g, d, i, j, k, d, -l - 1) * at(F, g, c, i, j, k, d, -l - 1),
                         dq);
            acc += dq + V(d, t) * dd1<H>(F, g, c, i, j, k, d, a[d]);
        }
        out[(long long)c * g.N3 + t] = 0.5 * acc;
    }
}

// laplacian(nu, f) with the stretched-z term (src/ex/laplacian/laplacian.hxx:130-191)
template <int H>
__global__ void k_op_lap(Geo g, Walls<double> wa, Coef<double> co, const double *__restrict__ ia, const double *__restrict__ corr2,
                         double nu, const double *__restrict__ f, int nc, double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 F{f, g.N3, wa};
    const double i2 = ia[k] * ia[k];
    for (int c = 0; c < nc; c++) {
        const double f0 = F(c, t);
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double m = (d == 2) ? i2 : 1.0;
            double s = 0.0;
#pragma unroll
            for (int l = 0; l < H; l++)
                s = fma(co.b[d][l] * m, at(F, g, c, i, j, k, d, l + 1) + at(F, g, c, i, j, k, d, -l - 1), s);
            r += fma(-co.b2[d] * m, f0, s);
        }
        double az[H];
#pragma unroll
        for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[k];
        const double dz = dd1<H>(F, g, c, i, j, k, 2, az);
        out[(long long)c * g.N3 + t] = nu * fma(-corr2[k], dz, r);
    }
}

// ex::div(Field<tensor>) (src/ex/div/div.hxx:258-285) and ex::div(Field<symmTensor>)
// (div.hxx:222-255; storage xx xy xz yy yz zz): out_c = sum_d D_d T[c*3+d],
// without the z metric, as in the reference
template <int H>
__global__ void k_op_div_t(Geo g, Walls<double> wa, Coef<double> co, const double *__restrict__ T, int symm,
                           double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 F{T, g.N3, wa};
    const int S[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int c = 0; c < 3; c++) {
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) r += dd1<H>(F, g, symm ? S[c * 3 + d] : c * 3 + d, i, j, k, d, co.a[d]);
        out[(long long)c * g.N3 + t] = r;
    }
}

// ex::div(Field<scalar> s, Field<tensor> T) (div.hxx:173-207): sum_d D_d (s T[c*3+d])
template <int H>
__global__ void k_op_div_st(Geo g, Walls<double> wa, Walls<double> wb, Coef<double> co, const double *__restrict__ s,
                            const double *__restrict__ T, double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 Sf{s, g.N3, wa}, F{T, g.N3, wb};
    for (int c = 0; c < 3; c++) {
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double q = 0.0;
#pragma unroll
            for (int l = 0; l < H; l++)
                q = fma(co.a[d][l],
                        at(Sf, g, 0, i, j, k, d, l + 1) * at(F, g, c * 3 + d, i, j, k, d, l + 1)
                            - at(Sf, g, 0, i, j, k, d, -l - 1) * at(F, g, c * 3 + d, i, j, k, d, -l - 1),
                        q);
            r += q;
        }
        out[(long long)c * g.N3 + t] = r;
    }
}

// ex::laplacian(Field<scalar> nu, Field<T>) (src/ex/laplacian/laplacian.hxx:64-127):
// the + neighbour at 1+l weighted by nu at offset l, the - neighbour at -1-l
// by nu at -1-l, both against the centre; z terms over dzdxi^2 and the
// stretched-z term -nu(0) D_z f d2zdxi2/dzdxi^3
template <int H>
__global__ void k_op_lap_f(Geo g, Walls<double> wa, Walls<double> wb, Coef<double> co, const double *__restrict__ ia,
                           const double *__restrict__ corr2, const double *__restrict__ nu, const double *__restrict__ f,
                           int nc, double *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    Ld64 NU{nu, g.N3, wa}, F{f, g.N3, wb};
    const double i2 = ia[k] * ia[k];
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[k];
    const double nu0 = NU(0, t);
    for (int c = 0; c < nc; c++) {
        const double f0 = F(c, t);
        double r = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double m = (d == 2) ? i2 : 1.0;
#pragma unroll
            for (int l = 0; l < H; l++) {
                const double np = l == 0 ? nu0 : at(NU, g, 0, i, j, k, d, l);
                const double nm = at(NU, g, 0, i, j, k, d, -l - 1);
                const double fp = at(F, g, c, i, j, k, d, l + 1), fm = at(F, g, c, i, j, k, d, -l - 1);
                r = fma(co.b[d][l] * m, fma(np, fp - f0, nm * (fm - f0)), r);
            }
        }
        const double dz = dd1<H>(F, g, c, i, j, k, 2, az);
        out[(long long)c * g.N3 + t] = fma(-nu0 * corr2[k], dz, r);
    }
}

// ------------------------------------------------------------------ layout --
// reference ghosted AoS (n0, n1, n2, nc) -> unique SoA
__global__ void k_aos_to_soa(Geo g, int h, int n1, int n2, int nc, const double *__restrict__ aos,
                             double *__restrict__ d64, float *__restrict__ hi, float *__restrict__ lo)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= g.N3) return;
    int i, j, k;
    pt_index(g, t, i, j, k);
    const long long src = (((long long)(i + h) * n1 + (j + h)) * n2 + (k + h)) * nc;
    for (int c = 0; c < nc; c++) {
        const double x = aos[src + c];
        if (d64) {
            d64[(long long)c * g.N3 + t] = x;
        } else {
            const float xh = (float)x;
            hi[(long long)c * g.N3 + t] = xh;
            lo[(long long)c * g.N3 + t] = (float)(x - (double)xh);
        }
    }
}

// unique SoA -> ghosted AoS with every slot filled by periodic wrap
// (interior incl. the duplicate node as periodicBC::update leaves it)
__global__ void k_soa_to_aos(Geo g, Walls<double> wl, int h, int n0, int n1, int n2, int nc,
                             const double *__restrict__ d64, const float *__restrict__ hi,
                             const float *__restrict__ lo, double *__restrict__ aos)
{
    const long long tot = (long long)n0 * n1 * n2;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= tot) return;
    const int kk = (int)(t % n2);
    const long long r = t / n2;
    const int jj = (int)(r % n1);
    const int ii = (int)(r / n1);
    int j = jj - h, side = -1, l = 0;
    if (wl.on) {
        if (j < 0) {
            side = 0;
            l = min(-j, g.N1 - 1);
            j = l;
        } else if (j >= g.N1) {
            side = 1;
            l = min(j - (g.N1 - 1), g.N1 - 1);
            j = (g.N1 - 1) - l;
        }
    } else {
        j = wrapi(j, g.N1);
    }
    const long long s = (long long)wrapi(ii - h, g.N0) * g.N12 + (long long)j * g.N2 + wrapi(kk - h, g.N2);
    for (int c = 0; c < nc; c++) {
        const long long o = (long long)c * g.N3 + s;
        const double v = d64 ? d64[o] : (double)hi[o] + (double)lo[o];
        aos[t * nc + c] = side < 0 ? v : wall_ghost(wl, side, c, l, v);
    }
}

// Wall-node overwrite of neumannBC / dirichletBC::update (src/BC/neumannBC.hxx:8-26,
// src/BC/dirichletBC.hxx:8-24): south f(0) = f(1) - val dy | val, north
// f(N1-1) = f(N1-2) + val dy | val, per component.
template <typename T>
__global__ void k_wall_fix(Geo g, WallFix wf, T *__restrict__ f, float *__restrict__ lo)
{
    const long long plane = (long long)g.N0 * g.N2;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= plane * wf.nc) return;
    const int c = (int)(t / plane);
    const long long r = t % plane;
    const int i = (int)(r / g.N2), k = (int)(r % g.N2);
    const long long base = (long long)c * g.N3 + (long long)i * g.N12 + k;
    auto get = [&](int j) -> double {
        const long long o = base + (long long)j * g.N2;
        return lo ? (double)f[o] + (double)lo[o] : (double)f[o];
    };
    auto put = [&](int j, double x) {
        const long long o = base + (long long)j * g.N2;
        if (lo) {
            const float h = (float)x;
            f[o] = (T)h;
            lo[o] = (float)(x - (double)h);
        } else {
            f[o] = (T)x;
        }
    };
    // north face (bc index 0) is applied before south (1), as correctBoundaryConditions orders them
    const int jn = g.N1 - 1;
    if (wf.type[1][c] == 1)
        put(jn, sizeof(T) == 4 && !lo ? (double)((float)get(jn - 1) + (float)(wf.val[1][c] * wf.dy))
                                      : get(jn - 1) + wf.val[1][c] * wf.dy);
    else if (wf.type[1][c] == 2)
        put(jn, wf.val[1][c]);
    if (wf.type[0][c] == 1)
        put(0, sizeof(T) == 4 && !lo ? (double)((float)get(1) - (float)(wf.val[0][c] * wf.dy))
                                     : get(1) - wf.val[0][c] * wf.dy);
    else if (wf.type[0][c] == 2)
        put(0, wf.val[0][c]);
}

__global__ void k_split(long long n, const double *__restrict__ x, float *__restrict__ hi, float *__restrict__ lo)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double v = x[t];
    const float h = (float)v;
    hi[t] = h;
    lo[t] = (float)(v - (double)h);
}

__global__ void k_join(long long n, const float *__restrict__ hi, const float *__restrict__ lo, double *__restrict__ x)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    x[t] = (double)hi[t] + (double)lo[t];
}

inline unsigned nblocks(long long n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// ----------------------------------------------------------------- launchers --
#define NOVA_DISPATCH_H(h, ...)                 \
    switch (h) {                                \
    case 1: { constexpr int HH = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int HH = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int HH = 3; __VA_ARGS__; } break; \
    default: { constexpr int HH = 4; __VA_ARGS__; } break; \
    }

cudaError_t launch_div_proj(int h, const Geo &g, const Walls<double> &wl, const Coef<double> &co, const double *ia,
                            const double *U64, const float *hi, const float *lo, double divisor, double *rhs,
                            cudaStream_t st, const StageExec &ex)
{
    if (ex.err && h == 3 && ex.impl != STAGE_MARCH && proj_tma_fits(g, wl.on))
        return launch_div_tma(g, co, wl, ia, U64, hi, lo, divisor, rhs, ex.err, st);
    const int ch = pick_ichunk(g, 3);
    const dim3 grid = tile_grid(g, ch), block(kTK, kTJ);
#define NOVA_DIV(LDT, LDV, W)                                                                             \
    NOVA_DISPATCH_H(h, {                                                                                  \
        constexpr size_t sb = tile_smem_bytes<double, HH, 3>();                                           \
        k_div_tiled<HH, LDT, W><<<grid, block, sb, st>>>(g, co, ia, LDV, divisor, rhs, ch);                \
    })
    if (U64) {
        if (wl.on) { NOVA_DIV(Ld64, (Ld64{U64, g.N3, wl}), true); } else { NOVA_DIV(Ld64, (Ld64{U64, g.N3, wl}), false); }
    } else {
        if (wl.on) {
            NOVA_DIV(LdSplit, (LdSplit{hi, lo, g.N3, wl}), true);
        } else {
            NOVA_DIV(LdSplit, (LdSplit{hi, lo, g.N3, wl}), false);
        }
    }
#undef NOVA_DIV
    return cudaSuccess;
}

void launch_scale(const Geo &g, int ny, void *spec, const double *kx2, const double *ky2, const double *kz2,
                  double invN3, cudaStream_t st)
{
    const long long tot = (long long)g.N0 * ny * (g.N2 / 2 + 1);
    k_scale<<<nblocks(tot, 256), 256, 0, st>>>(g, ny, (cuDoubleComplex *)spec, kx2, ky2, kz2, invN3);
}

cudaError_t launch_correct(int h, const Geo &g, const Walls<double> &pw, const Coef<double> &co, const double *ia,
                           const double *p, double s, const double *Us64, double *U64, const float *Ushi,
                           const float *Uslo, float *hi, float *lo, cudaStream_t st, const StageExec &ex)
{
    if (ex.err && h == 3 && ex.impl != STAGE_MARCH && proj_tma_fits(g, pw.on))
        return launch_correct_tma(g, co, pw, ia, p, s, Us64, U64, Ushi, Uslo, hi, lo, ex.err, st);
    const int ch = pick_ichunk(g, 4);
    const dim3 grid = tile_grid(g, ch), block(kTK, kTJ);
#define NOVA_CORR(SPL, W)                                                                                 \
    NOVA_DISPATCH_H(h, {                                                                                  \
        constexpr size_t sb = tile_smem_bytes<double, HH, 1>();                                           \
        k_correct_tiled<HH, SPL, W><<<grid, block, sb, st>>>(g, pw, co, ia, p, s, Us64, U64, Ushi, Uslo, hi, lo, ch); \
    })
    // SPLIT: (hi, lo) output, from an FP64 U* (Us64) or a (hi, lo) one
    if (U64) {
        if (pw.on) { NOVA_CORR(false, true); } else { NOVA_CORR(false, false); }
    } else {
        if (pw.on) { NOVA_CORR(true, true); } else { NOVA_CORR(true, false); }
    }
#undef NOVA_CORR
    return cudaSuccess;
}

int diag_blocks(const Geo &g)
{
    const dim3 gr = tile_grid(g, pick_ichunk(g, 2));
    const long long tiled = (long long)gr.x * gr.y * gr.z;
    return (int)(tiled > 1184 ? tiled : 1184);
}

DiagFinal diag_final_of(const Geo &g, const DiagPhys &ph, double step, double time, const double *U64,
                        const float *Uhi, const float *Ulo)
{
    DiagFinal f{};
    f.invN3 = 1.0 / (double)((long long)g.N0 * (g.N1 - g.wallY) * g.N2);
    f.step = step;
    f.time = time;
    f.nu = ph.nu;
    f.eta = ph.eta;
    f.dt = ph.dt;
    f.dx = ph.dx;
    f.dy = ph.dy;
    f.dz = ph.dz;
    f.U64 = U64;
    f.Uhi = Uhi;
    f.Ulo = Ulo;
    f.N3 = g.N3;
    // the reference's interior node (N0, N1, N2): periodic axes wrap to 0, a
    // wall axis stores it (the north wall row)
    f.last = g.wallY ? (long long)(g.N1 - 1) * g.N2 : 0;
    return f;
}

void launch_diag(int h, const Geo &g, const Walls<double> &wl, const Coef<double> &co, const double *ia,
                 const double *U64, const float *Uhi, const float *Ulo, const double *B64, const float *Bhi,
                 const float *Blo, int hasB, double *part, double step, double time, double *row, int *flag,
                 cudaStream_t st, const DiagPhys &ph)
{
    const int ch = pick_ichunk(g, 2);
    const dim3 grid = tile_grid(g, ch), block(kTK, kTJ);
    const int nb = (int)(grid.x * grid.y * grid.z);
#define NOVA_DIAG(NC, LDT, UU, BB, W)                                                                     \
    NOVA_DISPATCH_H(h, {                                                                                  \
        constexpr size_t sb = tile_smem_bytes<double, HH, NC>();                                          \
        if (sb > 48 * 1024)                                                                               \
            cudaFuncSetAttribute(k_diag_tiled<HH, NC, LDT, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb); \
        k_diag_tiled<HH, NC, LDT, W><<<grid, block, sb, st>>>(g, wl, co, ia, UU, BB, ch, part);            \
    })
    if (U64) {
        Ld64 U{U64, g.N3, wl}, B{hasB ? B64 : U64, g.N3, wl};
        if (hasB) {
            if (wl.on) { NOVA_DIAG(6, Ld64, U, B, true); } else { NOVA_DIAG(6, Ld64, U, B, false); }
        } else {
            if (wl.on) { NOVA_DIAG(3, Ld64, U, B, true); } else { NOVA_DIAG(3, Ld64, U, B, false); }
        }
    } else {
        LdSplit U{Uhi, Ulo, g.N3, wl}, B{hasB ? Bhi : Uhi, hasB ? Blo : Ulo, g.N3, wl};
        if (hasB) {
            if (wl.on) { NOVA_DIAG(6, LdSplit, U, B, true); } else { NOVA_DIAG(6, LdSplit, U, B, false); }
        } else {
            if (wl.on) { NOVA_DIAG(3, LdSplit, U, B, true); } else { NOVA_DIAG(3, LdSplit, U, B, false); }
        }
    }
#undef NOVA_DIAG
    k_diag_final<<<1, 256, 0, st>>>(part, nb, diag_final_of(g, ph, step, time, U64, Uhi, Ulo), row, flag);
}

void launch_diag_final(const double *part, int nb, const DiagFinal &fin, double *row, int *flag, cudaStream_t st)
{
    k_diag_final<<<1, 256, 0, st>>>(part, nb, fin, row, flag);
}

void launch_maxabs(const Geo &g, const double *s, double *part, double *out, cudaStream_t st)
{
    const int nb = diag_blocks(g);
    k_maxabs_part<<<nb, 256, 0, st>>>(g.N3, Ld64{s, g.N3}, part);
    k_max_final<<<1, 256, 0, st>>>(part, nb, out);
}

// The allocation-free reduction's scratch: kMaxabsStaticParts partials, then
// the result slot (64 KiB per device, part of the library image).  Nothing in
// it has to start at zero: k_maxabs_chunks writes every partial that
// k_max_final reads, and k_max_final writes the result before it is copied out.
static __device__ __align__(256) double g_maxabs_scratch[kMaxabsStaticParts + 1];
static_assert((long long)kMaxabsChunk * kMaxabsStaticParts == NOVA_MAXABS_NOALLOC_MAX_NODES,
              "the static scratch must cover the advertised node limit");

// The scratch's device address, looked up on every call with the caller's
// device current: a cached address would go stale when the primary context
// is destroyed and made again (cudaDeviceReset), and the lookup is cheap once
// the module is loaded.
cudaError_t maxabs_noalloc_scratch(double **scratch)
{
    double *q = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&q, g_maxabs_scratch);
    if (e != cudaSuccess) return e;
    *scratch = q;
    return cudaSuccess;
}

void launch_maxabs_noalloc(long long n, const double *s, double *scratch, cudaStream_t st)
{
    const int np = (int)((n + kMaxabsChunk - 1) / kMaxabsChunk);
    k_maxabs_chunks<<<np, 256, 0, st>>>(n, s, scratch);
    k_max_final<<<1, 256, 0, st>>>(scratch, np, scratch + kMaxabsStaticParts);
}

void launch_op(int op, int h, const Geo &g, const Walls<double> &wa, const Walls<double> &wb, const Coef<double> &co,
               const double *ia, const double *corr2, const double *a, const double *b, int nc, double nu, double *out,
               cudaStream_t st)
{
    const unsigned nb = nblocks(g.N3, 128);
    switch (op) {
    case OP_GRAD_S: NOVA_DISPATCH_H(h, (k_op_grad_s<HH><<<nb, 128, 0, st>>>(g, wa, co, ia, a, out))); break;
    case OP_GRAD_V: NOVA_DISPATCH_H(h, (k_op_grad_v<HH><<<nb, 128, 0, st>>>(g, wa, co, ia, a, out))); break;
    case OP_DIV_V: NOVA_DISPATCH_H(h, (k_op_div_v<HH><<<nb, 128, 0, st>>>(g, wa, co, ia, a, out))); break;
    case OP_CURL: NOVA_DISPATCH_H(h, (k_op_curl<HH><<<nb, 128, 0, st>>>(g, wa, co, ia, a, out))); break;
    case OP_DIV_VF: NOVA_DISPATCH_H(h, (k_op_div_vf<HH><<<nb, 128, 0, st>>>(g, wa, wb, co, ia, a, b, nc, out))); break;
    case OP_DIV_T: NOVA_DISPATCH_H(h, (k_op_div_t<HH><<<nb, 128, 0, st>>>(g, wa, co, a, nc == 6, out))); break;
    case OP_DIV_ST: NOVA_DISPATCH_H(h, (k_op_div_st<HH><<<nb, 128, 0, st>>>(g, wa, wb, co, a, b, out))); break;
    case OP_LAP_F:
        NOVA_DISPATCH_H(h, (k_op_lap_f<HH><<<nb, 128, 0, st>>>(g, wa, wb, co, ia, corr2, a, b, nc, out)));
        break;
    default: NOVA_DISPATCH_H(h, (k_op_lap<HH><<<nb, 128, 0, st>>>(g, wa, co, ia, corr2, nu, a, nc, out))); break;
    }
}

void launch_aos_to_soa(const Geo &g, int h, const int n[3], int nc, const double *aos, double *d64, float *hi,
                       float *lo, cudaStream_t st)
{
    k_aos_to_soa<<<nblocks(g.N3, 256), 256, 0, st>>>(g, h, n[1], n[2], nc, aos, d64, hi, lo);
}

void launch_soa_to_aos(const Geo &g, const Walls<double> &wl, int h, const int n[3], int nc, const double *d64,
                       const float *hi, const float *lo, double *aos, cudaStream_t st)
{
    const long long tot = (long long)n[0] * n[1] * n[2];
    k_soa_to_aos<<<nblocks(tot, 256), 256, 0, st>>>(g, wl, h, n[0], n[1], n[2], nc, d64, hi, lo, aos);
}

void launch_wall_fix64(const Geo &g, const WallFix &wf, double *f, cudaStream_t st)
{
    k_wall_fix<double><<<nblocks((long long)g.N0 * g.N2 * wf.nc, 256), 256, 0, st>>>(g, wf, f, nullptr);
}

void launch_wall_fix32(const Geo &g, const WallFix &wf, float *f, cudaStream_t st)
{
    k_wall_fix<float><<<nblocks((long long)g.N0 * g.N2 * wf.nc, 256), 256, 0, st>>>(g, wf, f, nullptr);
}

void launch_wall_fix_split(const Geo &g, const WallFix &wf, float *hi, float *lo, cudaStream_t st)
{
    k_wall_fix<float><<<nblocks((long long)g.N0 * g.N2 * wf.nc, 256), 256, 0, st>>>(g, wf, hi, lo);
}

void launch_even_extend(const Geo &g, int ny, const double *rhs, double *ext, cudaStream_t st)
{
    k_even_extend<<<nblocks((long long)g.N0 * 2 * ny * g.N2, 256), 256, 0, st>>>(g, ny, rhs, ext);
}

void launch_restrict_rows(const Geo &g, int ny, const double *ext, double *p, cudaStream_t st)
{
    k_restrict_rows<<<nblocks(g.N3, 256), 256, 0, st>>>(g, ny, ext, p);
}

void launch_split(long long n, const double *x, float *hi, float *lo, cudaStream_t st)
{
    k_split<<<nblocks(n, 256), 256, 0, st>>>(n, x, hi, lo);
}

void launch_join(long long n, const float *hi, const float *lo, double *x, cudaStream_t st)
{
    k_join<<<nblocks(n, 256), 256, 0, st>>>(n, hi, lo, x);
}

}  // namespace nova
