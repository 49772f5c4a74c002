// Fused Runge-Kutta stage kernels: one kernel computes the whole right-hand
// side of one stage and applies the stage update in its epilogue.
//
//   NS    (app/TG_Piosson/RKLoop.H:17-28, app/OT_Poisson/UEqn.H:16-30):
//         dU = dt*( -div(U,U) + laplacian(nu,U) )
//   MHD U (app/OT_Poisson/UEqn.H:16-23):
//         dU = dt*( -div(U,U) + laplacian(nu,U) + div(B,B) - grad(0.5*(B&B)) )
//   MHD B (app/OT_Poisson/BEqn.H:72-78):
//         dB = dt*( -div(U,B) + div(B,U) + laplacian(eta,B) )
//
// with ex::div(V,F) the skew form of src/ex/div/div.hxx:84-172,
//   div(V,F)_c = 1/2 sum_d [ D_d(V_d F_c) + V_d D_d F_c + F_c D_d V_d ],
// ex::laplacian(nu,F) of src/ex/laplacian/laplacian.hxx:130-191 including its
// stretched-z term, and ex::grad of src/ex/grad/grad.cpp:25-62; the z
// derivatives carry the Mesh::dzdxi_ metric (src/Mesh/Mesh.cpp:147-179).
//
// Tiling (2.5-D): a block owns a 32(k) x 8(j) column of the grid and marches
// along i.  Each thread keeps its column's 2H+1 planes in a register queue (the
// i-direction stencil), the current plane plus its j/k halo sits in shared
// memory (the j- and k-direction stencils).  Periodic ghosts are synthesised by
// wrapping indices at load time, which replaces periodicBC::update.
//
// Epilogue (stage s of the classical RK4 of src/settings/settings.cpp:44-51,
// association order of app/TG_Piosson/RKLoop.H:24-28 kept):
//   s=0: Y1 = U0 + dU*1/2   A = U0 + dU*1/6
//   s=1: Y2 = U0 + dU*1/2   A = A  + dU*1/3
//   s=2: Y3 = U0 + dU       A = A  + dU*1/3
//   s=3: U* = A  + dU*1/6
//   s=4 (the reference loop as written, U not refreshed between stages, so
//        all four dU are equal): U* = (((U0 + dU/6) + dU/3) + dU/3) + dU/6
// The FP32-split variant keeps A as an FP32 sum of increments and adds it to
// the (hi, lo) base in FP64 at the last stage.
#include "nova_internal.cuh"

#include <type_traits>

namespace nova {

namespace {

template <typename T, int H, int PHYS, int STAGE, class Args>
__global__ void __launch_bounds__(kThreads) k_stage(Geo g, Coef<T> co, const T *__restrict__ ia,
                                                      const T *__restrict__ corr2, T dt, T visc, Args args,
                                                      int ichunk)
{
    constexpr int NC = (PHYS == PHYS_NS) ? 3 : 6;
    constexpr int W = kTK + 2 * H;
    constexpr int R = kTJ + 2 * H;
    constexpr int NJH = 2 * H * kTK;
    constexpr int NKH = 2 * H * kTJ;
    constexpr int NH = NJH + NKH;
    constexpr int HS = (NH + kThreads - 1) / kThreads;
    __shared__ T sm[NC][R][W];

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTK + tx;
    const int k0 = blockIdx.x * kTK, j0 = blockIdx.y * kTJ;
    const int k = k0 + tx, j = j0 + ty;
    const bool valid = (k < g.N2) && (j < g.N1);
    const int kw = wrapi(k, g.N2), jw = wrapi(j, g.N1);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);

    const T *src[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
        const T *base;
        if constexpr (std::is_same<Args, StageArgs64>::value)
            base = (c < 3) ? args.Y : args.X;
        else
            base = (c < 3) ? args.Y : args.X;
        src[c] = base + (long long)(c % 3) * g.N3;
    }

    // halo cells of the current plane owned by this thread
    int hrow[HS], hcol[HS];
    long long hoff[HS];
    bool hon[HS];
#pragma unroll
    for (int s = 0; s < HS; s++) {
        const int t = tid + s * kThreads;
        hon[s] = t < NH;
        int row, col;
        if (t < NJH) {
            const int r = t / kTK;
            row = r < H ? r : kTJ + r;
            col = H + t % kTK;
        } else {
            const int u = t - NJH;
            row = H + u / (2 * H);
            const int cc = u % (2 * H);
            col = cc < H ? cc : kTK + cc;
        }
        if (!hon[s]) { row = 0; col = 0; }
        hrow[s] = row;
        hcol[s] = col;
        hoff[s] = (long long)wrapi(j0 + row - H, g.N1) * g.N2 + wrapi(k0 + col - H, g.N2);
    }

    // z metric of this thread's column (src/ex/*: terms divided by dzdxi(k))
    const T iak = ia[kw];
    const T c2k = corr2[kw];
    T az[H], bz[H];
#pragma unroll
    for (int l = 0; l < H; l++) {
        az[l] = co.a[2][l] * iak;
        bz[l] = co.b[2][l] * iak * iak;
    }
    const T b2z = co.b2[2] * iak * iak;

    const long long colOff = (long long)jw * g.N2 + kw;
    T q[2 * H + 1][NC];
#pragma unroll
    for (int s = 0; s < 2 * H; s++) {
        const long long p = (long long)wrapi(ib - H + s, g.N0) * g.N12 + colOff;
#pragma unroll
        for (int c = 0; c < NC; c++) q[s + 1][c] = src[c][p];
    }

    for (int i = ib; i < ie; i++) {
#pragma unroll
        for (int s = 0; s < 2 * H; s++)
#pragma unroll
            for (int c = 0; c < NC; c++) q[s][c] = q[s + 1][c];
        {
            const long long p = (long long)wrapi(i + H, g.N0) * g.N12 + colOff;
#pragma unroll
            for (int c = 0; c < NC; c++) q[2 * H][c] = src[c][p];
        }
        const long long plane = (long long)i * g.N12;
        __syncthreads();
#pragma unroll
        for (int c = 0; c < NC; c++) sm[c][ty + H][tx + H] = q[H][c];
#pragma unroll
        for (int s = 0; s < HS; s++)
            if (hon[s])
#pragma unroll
                for (int c = 0; c < NC; c++) sm[c][hrow[s]][hcol[s]] = src[c][plane + hoff[s]];
        __syncthreads();
        if (!valid) continue;

        auto vx = [&](int c, int s) -> T { return q[H + s][c]; };
        auto vy = [&](int c, int s) -> T { return sm[c][ty + H + s][tx + H]; };
        auto vz = [&](int c, int s) -> T { return sm[c][ty + H][tx + H + s]; };

        T rhs[3];
        if constexpr (PHYS == PHYS_NS) {
            T u0[3] = {q[H][0], q[H][1], q[H][2]};
            T adv[3] = {0, 0, 0}, lap[3] = {0, 0, 0}, div = 0, duz[3];
            auto dir = [&](const auto &v, int d, const T *a, const T *b, T b2, T *du_keep) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T du = d1<T, H>(v, c, a);
                    adv[c] += fma(u0[d], du, d1p<T, H>(v, d, c, a));
                    lap[c] += d2<T, H>(v, c, b, b2);
                    if (c == d) div += du;
                    if (du_keep) du_keep[c] = du;
                }
            };
            dir(vx, 0, co.a[0], co.b[0], co.b2[0], nullptr);
            dir(vy, 1, co.a[1], co.b[1], co.b2[1], nullptr);
            dir(vz, 2, az, bz, b2z, duz);
#pragma unroll
            for (int c = 0; c < 3; c++)
                rhs[c] = T(-0.5) * fma(u0[c], div, adv[c]) + visc * fma(-c2k, duz[c], lap[c]);
        } else if constexpr (PHYS == PHYS_MHD_U) {
            // comps 0-2: U (stage state), 3-5: B (frozen)
            T u0[3] = {q[H][0], q[H][1], q[H][2]};
            T b0[3] = {q[H][3], q[H][4], q[H][5]};
            T advU[3] = {0, 0, 0}, advB[3] = {0, 0, 0}, lap[3] = {0, 0, 0}, gb[3], divU = 0, divB = 0, duz[3];
            auto dir = [&](const auto &v, int d, const T *a, const T *b, T b2, T *du_keep) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T du = d1<T, H>(v, c, a);
                    const T db = d1<T, H>(v, 3 + c, a);
                    advU[c] += fma(u0[d], du, d1p<T, H>(v, d, c, a));
                    advB[c] += fma(b0[d], db, d1p<T, H>(v, 3 + d, 3 + c, a));
                    lap[c] += d2<T, H>(v, c, b, b2);
                    if (c == d) { divU += du; divB += db; }
                    if (du_keep) du_keep[c] = du;
                }
                // grad(0.5*(B&B)) along d (src/ex/grad/grad.cpp:43-54 on the product field)
                auto e = [&](int, int s) -> T {
                    return (v(3, s) * v(3, s) + v(4, s) * v(4, s) + v(5, s) * v(5, s)) * T(0.5);
                };
                gb[d] = d1<T, H>(e, 0, a);
            };
            dir(vx, 0, co.a[0], co.b[0], co.b2[0], nullptr);
            dir(vy, 1, co.a[1], co.b[1], co.b2[1], nullptr);
            dir(vz, 2, az, bz, b2z, duz);
#pragma unroll
            for (int c = 0; c < 3; c++)
                rhs[c] = T(-0.5) * fma(u0[c], divU, advU[c]) + visc * fma(-c2k, duz[c], lap[c])
                         + T(0.5) * fma(b0[c], divB, advB[c]) - gb[c];
        } else {
            // comps 0-2: B (stage state), 3-5: U (frozen)
            T b0[3] = {q[H][0], q[H][1], q[H][2]};
            T u0[3] = {q[H][3], q[H][4], q[H][5]};
            T advUB[3] = {0, 0, 0}, advBU[3] = {0, 0, 0}, lap[3] = {0, 0, 0}, divU = 0, divB = 0, dbz[3];
            auto dir = [&](const auto &v, int d, const T *a, const T *b, T b2, T *db_keep) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T db = d1<T, H>(v, c, a);
                    const T du = d1<T, H>(v, 3 + c, a);
                    advUB[c] += fma(u0[d], db, d1p<T, H>(v, 3 + d, c, a));
                    advBU[c] += fma(b0[d], du, d1p<T, H>(v, d, 3 + c, a));
                    lap[c] += d2<T, H>(v, c, b, b2);
                    if (c == d) { divU += du; divB += db; }
                    if (db_keep) db_keep[c] = db;
                }
            };
            dir(vx, 0, co.a[0], co.b[0], co.b2[0], nullptr);
            dir(vy, 1, co.a[1], co.b[1], co.b2[1], nullptr);
            dir(vz, 2, az, bz, b2z, dbz);
#pragma unroll
            for (int c = 0; c < 3; c++)
                rhs[c] = T(-0.5) * fma(b0[c], divU, advUB[c]) + T(0.5) * fma(u0[c], divB, advBU[c])
                         + visc * fma(-c2k, dbz[c], lap[c]);
        }

        const long long idx = plane + colOff;
        if constexpr (std::is_same<T, double>::value) {
            // RK4a weights (src/settings/settings.cpp:44-50)
            const double w6 = 1.0 / 6.0, w3 = 1.0 / 3.0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const long long o = (long long)c * g.N3 + idx;
                const double du = dt * rhs[c];
                const double y0 = q[H][c];
                if constexpr (STAGE == 4) {
                    args.Ynext[o] = (((y0 + du * w6) + du * w3) + du * w3) + du * w6;
                } else if constexpr (STAGE == 0) {
                    args.Ynext[o] = y0 + du * 0.5;
                    args.A[o] = y0 + du * w6;
                } else if constexpr (STAGE == 1) {
                    args.Ynext[o] = args.U0[o] + du * 0.5;
                    args.A[o] = args.A[o] + du * w3;
                } else if constexpr (STAGE == 2) {
                    args.Ynext[o] = args.U0[o] + du * 1.0;
                    args.A[o] = args.A[o] + du * w3;
                } else {
                    args.Ynext[o] = args.A[o] + du * w6;
                }
            }
        } else {
            const float w6 = 1.0f / 6.0f, w3 = 1.0f / 3.0f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const long long o = (long long)c * g.N3 + idx;
                const float du = dt * rhs[c];
                if constexpr (STAGE == 4) {
                    const float inc = ((du * w6 + du * w3) + du * w3) + du * w6;
                    const double x = ((double)q[H][c] + (double)args.U0lo[o]) + (double)inc;
                    const float hi = (float)x;
                    args.outhi[o] = hi;
                    args.outlo[o] = (float)(x - (double)hi);
                } else if constexpr (STAGE == 0) {
                    args.Ynext[o] = q[H][c] + du * 0.5f;
                    args.A[o] = du * w6;
                } else if constexpr (STAGE == 1) {
                    args.Ynext[o] = args.U0hi[o] + du * 0.5f;
                    args.A[o] = args.A[o] + du * w3;
                } else if constexpr (STAGE == 2) {
                    args.Ynext[o] = args.U0hi[o] + du;
                    args.A[o] = args.A[o] + du * w3;
                } else {
                    const float inc = args.A[o] + du * w6;
                    const double x = ((double)args.U0hi[o] + (double)args.U0lo[o]) + (double)inc;
                    const float hi = (float)x;
                    args.outhi[o] = hi;
                    args.outlo[o] = (float)(x - (double)hi);
                }
            }
        }
    }
}

constexpr int kH = 3;

int pick_ichunk(const Geo &g)
{
    // aim for >= 4 waves of ~2 resident blocks on 148 SMs while keeping the
    // 2H-plane warm-up small against the chunk length
    const long long tiles = (long long)((g.N2 + kTK - 1) / kTK) * ((g.N1 + kTJ - 1) / kTJ);
    int ch = g.N0;
    while (ch > 16 && tiles * ((g.N0 + ch - 1) / ch) < 148 * 8) ch /= 2;
    return ch;
}

template <typename T, int PHYS, int STAGE, class Args>
void launch_one(const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc, const Args &a,
                cudaStream_t st)
{
    const int ch = pick_ichunk(g);
    dim3 block(kTK, kTJ);
    dim3 grid((g.N2 + kTK - 1) / kTK, (g.N1 + kTJ - 1) / kTJ, (g.N0 + ch - 1) / ch);
    k_stage<T, kH, PHYS, STAGE, Args><<<grid, block, 0, st>>>(g, co, ia, corr2, dt, visc, a, ch);
}

template <typename T, int PHYS, class Args>
void launch_phys(int stage, const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc,
                 const Args &a, cudaStream_t st)
{
    switch (stage) {
    case 0: launch_one<T, PHYS, 0>(g, co, ia, corr2, dt, visc, a, st); break;
    case 1: launch_one<T, PHYS, 1>(g, co, ia, corr2, dt, visc, a, st); break;
    case 2: launch_one<T, PHYS, 2>(g, co, ia, corr2, dt, visc, a, st); break;
    case 3: launch_one<T, PHYS, 3>(g, co, ia, corr2, dt, visc, a, st); break;
    default: launch_one<T, PHYS, 4>(g, co, ia, corr2, dt, visc, a, st); break;
    }
}

}  // namespace

void launch_stage64(int phys, int stage, const Geo &g, const Coef<double> &co, const double *ia,
                    const double *corr2, double dt, double visc, const StageArgs64 &a, cudaStream_t st)
{
    switch (phys) {
    case PHYS_NS: launch_phys<double, PHYS_NS>(stage, g, co, ia, corr2, dt, visc, a, st); break;
    case PHYS_MHD_U: launch_phys<double, PHYS_MHD_U>(stage, g, co, ia, corr2, dt, visc, a, st); break;
    default: launch_phys<double, PHYS_MHD_B>(stage, g, co, ia, corr2, dt, visc, a, st); break;
    }
}

void launch_stage32(int phys, int stage, const Geo &g, const Coef<float> &co, const float *ia,
                    const float *corr2, float dt, float visc, const StageArgs32 &a, cudaStream_t st)
{
    switch (phys) {
    case PHYS_NS: launch_phys<float, PHYS_NS>(stage, g, co, ia, corr2, dt, visc, a, st); break;
    case PHYS_MHD_U: launch_phys<float, PHYS_MHD_U>(stage, g, co, ia, corr2, dt, visc, a, st); break;
    default: launch_phys<float, PHYS_MHD_B>(stage, g, co, ia, corr2, dt, visc, a, st); break;
    }
}

}  // namespace nova
