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
// ex::div(V,F) is the skew form of src/ex/div/div.hxx:84-172,
//   div(V,F)_c = 1/2 sum_d [ D_d(V_d F_c) + V_d D_d F_c + F_c D_d V_d ],
// evaluated here as 1/2 sum_d [ A_d(V,F)_c + F_c D_d V_d ] with
//   A_d(V,F)_c = sum_l a_l [ F_c(+l) (V_d(+l) + V_d(0)) - F_c(-l) (V_d(-l) + V_d(0)) ],
// which equals D_d(V_d F_c) + V_d(0) D_d F_c and costs one product per node
// pair instead of three.  ex::laplacian(nu,F) follows
// src/ex/laplacian/laplacian.hxx:130-191 (centre terms of the three
// directions folded into one), the stretched-z term included when the mesh is
// stretched; ex::grad follows src/ex/grad/grad.cpp:25-62.  z derivatives carry
// the Mesh::dzdxi_ metric (src/Mesh/Mesh.cpp:147-179).
//
// Epilogue (stage s of the classical RK4 of src/settings/settings.cpp:44-51,
// association order of app/TG_Piosson/RKLoop.H:24-28 kept):
//   s=0: Y1 = U0 + dU*1/2   A = U0 + dU*1/6
//   s=1: Y2 = U0 + dU*1/2   A = A  + dU*1/3
//   s=2: Y3 = U0 + dU       A = A  + dU*1/3
//   s=3: U* = A  + dU*1/6
//   s=4 (the reference loop as written, U not refreshed between stages, so
//        all four dU are equal): U* = (((U0 + dU/6) + dU/3) + dU/3) + dU/6
//   s=5 (app/shearLayer/UEqn.H:28-29): U* = U0 + dU*w, w the stage's weight
// The FP32-split variant keeps A as an FP32 sum of increments and adds it to
// the (hi, lo) base in FP64 at the last stage.
#include "nova_internal.cuh"
#include "nova_stage_math.cuh"
#include "nova_tile.cuh"

#include <type_traits>

// minimum resident blocks per SM requested from the register allocator for
// the Navier-Stokes kernels (FP64, FP32); the MHD kernels (6 halo'd
// components) ask for one
#ifndef NOVA_STAGE_MINB
#define NOVA_STAGE_MINB 2
#endif
#ifndef NOVA_STAGE_MINB32
#define NOVA_STAGE_MINB32 2
#endif

template <typename T, int PHYS> constexpr int stage_minb()
{
    return PHYS != 0 ? 1 : (sizeof(T) == 8 ? NOVA_STAGE_MINB : NOVA_STAGE_MINB32);
}

namespace nova {

namespace {

template <typename T, int H, int PHYS, int STAGE, bool STRETCH, bool WALLS, class Args>
__global__ void __launch_bounds__(kThreads, (stage_minb<T, PHYS>())) k_stage(Geo g, Walls<T> wl, Coef<T> co,
                                                      StageCoef<T> sc, const T *__restrict__ ia,
                                                      const T *__restrict__ corr2, T dt, T visc, Args args, int ichunk)
{
    constexpr int NC = (PHYS == PHYS_NS) ? 3 : 6;
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<T, H, NC> *>(smraw);

    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);

    // z metric of this thread's column (src/ex/*: terms divided by dzdxi(k))
    const T iak = ia[kw];
    const T c2k = STRETCH ? corr2[kw] : T(0);

    const T *src[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) src[c] = ((c < 3) ? args.Y : args.X) + (long long)(c % 3) * g.N3;

    // pointwise epilogue operands (base, accumulator): prefetched one plane
    // ahead in FP64 and in the FP32 shear-layer stage (5: base hi and lo, the
    // latter in the accumulator's place); the other FP32 stages load them at
    // the start of the plane (measured faster there: fewer live registers)
    constexpr bool kSplit5 = !std::is_same<T, double>::value && STAGE == 5;
    constexpr bool kE0 = (STAGE == 1 || STAGE == 2 || STAGE == 5) || (!std::is_same<T, double>::value && STAGE == 3);
    constexpr bool kE1 = (STAGE >= 1 && STAGE <= 3) || kSplit5;
    constexpr bool kAhead = std::is_same<T, double>::value || kSplit5;
    const T *e0p = nullptr, *e1p = nullptr;
    if constexpr (std::is_same<T, double>::value) {
        e0p = args.U0;
        e1p = args.A;
    } else {
        e0p = args.U0hi;
        e1p = kSplit5 ? args.U0lo : args.A;
    }
    T e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, e0n[3] = {0, 0, 0}, e1n[3] = {0, 0, 0};
    auto pre = [&](long long nidx, bool load) {
        if constexpr (kAhead) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                e0[c] = e0n[c];
                e1[c] = e1n[c];
                if (load) {
                    const long long o = (long long)c * g.N3 + nidx;
                    if constexpr (kE0) e0n[c] = e0p[o];
                    if constexpr (kE1) e1n[c] = e1p[o];
                }
            }
        }
    };

    tile_march<T, H, NC, WALLS>(
        g, wl, sm, [&](int c, long long o) { return src[c][o]; }, ib, ie, pre,
        [&](long long idx, auto &q, const auto &vx, const auto &vy, const auto &vz) {
            if constexpr (!kAhead) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const long long o = (long long)c * g.N3 + idx;
                    if constexpr (kE0) e0[c] = e0p[o];
                    if constexpr (kE1) e1[c] = e1p[o];
                }
            }
            T rhs[3], divu;
            if constexpr (PHYS == PHYS_NS) {
                const T u0[3] = {q[H][0], q[H][1], q[H][2]};
                ns_rhs<T, H, STRETCH>(vx, vy, vz, u0, co, sc, iak, c2k, visc, rhs, divu);
            } else if constexpr (PHYS == PHYS_MHD_U) {
                // comps 0-2: U (stage state), 3-5: B (frozen)
                const T u0[3] = {q[H][0], q[H][1], q[H][2]};
                const T b0[3] = {q[H][3], q[H][4], q[H][5]};
                mhd_rhs<T, H, STRETCH, true>(vx, vy, vz, u0, b0, co, sc, iak, c2k, visc, rhs);
            } else {
                // comps 0-2: B (stage state), 3-5: U (frozen)
                const T b0[3] = {q[H][0], q[H][1], q[H][2]};
                const T u0[3] = {q[H][3], q[H][4], q[H][5]};
                mhd_rhs<T, H, STRETCH, false>(vx, vy, vz, b0, u0, co, sc, iak, c2k, visc, rhs);
            }

            if constexpr (std::is_same<T, double>::value) {
#pragma unroll
                for (int c = 0; c < 3; c++)
                    rk_store64<STAGE>(args, (long long)c * g.N3 + idx, q[H][c], e0[c], e1[c], dt * rhs[c]);
            } else {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const long long o = (long long)c * g.N3 + idx;
                    const float lo = kSplit5 ? e1[c] : ((STAGE >= 3) ? args.U0lo[o] : 0.0f);
                    rk_store32<STAGE>(args, o, q[H][c], e0[c], e1[c], lo, dt * rhs[c]);
                }
            }
        });
}

constexpr int kH = 3;

template <typename T, int PHYS, int STAGE, bool STRETCH, bool WALLS, class Args>
void launch_one(const Geo &g, const Walls<T> &wl, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc,
                const Args &a, cudaStream_t st)
{
    constexpr int NC = (PHYS == PHYS_NS) ? 3 : 6;
    constexpr size_t smem = tile_smem_bytes<T, kH, NC>();
    auto kern = k_stage<T, kH, PHYS, STAGE, STRETCH, WALLS, Args>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int bps = stage_minb<T, PHYS>();
    const int ch = pick_ichunk(g, bps);
    kern<<<tile_grid(g, ch), dim3(kTK, kTJ), smem, st>>>(g, wl, co, stage_coef(co, visc), ia, corr2, dt, visc, a, ch);
}

template <typename T, int PHYS, bool STRETCH, bool WALLS, class Args>
void launch_stage_t(int stage, const Geo &g, const Walls<T> &wl, const Coef<T> &co, const T *ia, const T *corr2, T dt,
                    T visc, const Args &a, cudaStream_t st)
{
    switch (stage) {
    case 0: launch_one<T, PHYS, 0, STRETCH, WALLS>(g, wl, co, ia, corr2, dt, visc, a, st); break;
    case 1: launch_one<T, PHYS, 1, STRETCH, WALLS>(g, wl, co, ia, corr2, dt, visc, a, st); break;
    case 2: launch_one<T, PHYS, 2, STRETCH, WALLS>(g, wl, co, ia, corr2, dt, visc, a, st); break;
    case 3: launch_one<T, PHYS, 3, STRETCH, WALLS>(g, wl, co, ia, corr2, dt, visc, a, st); break;
    case 5: launch_one<T, PHYS, 5, STRETCH, WALLS>(g, wl, co, ia, corr2, dt, visc, a, st); break;
    default: launch_one<T, PHYS, 4, STRETCH, WALLS>(g, wl, co, ia, corr2, dt, visc, a, st); break;
    }
}

template <typename T, class Args>
void launch_stage_any(int phys, int stage, bool stretch, const Geo &g, const Walls<T> &wl, const Coef<T> &co,
                      const T *ia, const T *corr2, T dt, T visc, const Args &a, cudaStream_t st)
{
    // walls are built for the Navier-Stokes stage only (the C ABI refuses MHD with walls)
    const bool walls = wl.on != 0;
#define NOVA_STAGE_CASE(P, S, W) launch_stage_t<T, P, S, W>(stage, g, wl, co, ia, corr2, dt, visc, a, st)
    if (phys == PHYS_NS) {
        if (stretch) {
            if (walls) NOVA_STAGE_CASE(PHYS_NS, true, true); else NOVA_STAGE_CASE(PHYS_NS, true, false);
        } else {
            if (walls) NOVA_STAGE_CASE(PHYS_NS, false, true); else NOVA_STAGE_CASE(PHYS_NS, false, false);
        }
    } else if (phys == PHYS_MHD_U) {
        if (stretch) NOVA_STAGE_CASE(PHYS_MHD_U, true, false); else NOVA_STAGE_CASE(PHYS_MHD_U, false, false);
    } else {
        if (stretch) NOVA_STAGE_CASE(PHYS_MHD_B, true, false); else NOVA_STAGE_CASE(PHYS_MHD_B, false, false);
    }
#undef NOVA_STAGE_CASE
}

}  // namespace

cudaError_t launch_stage64(int phys, int stage, bool stretch, const Geo &g, const Walls<double> &wl,
                           const Coef<double> &co, const double *ia, const double *corr2, double dt, double visc,
                           const StageArgs64 &a, cudaStream_t st, const StageExec &ex, const StageDiag *dg,
                           bool *dg_done)
{
    if (phys == PHYS_NS && ex.impl != STAGE_MARCH && ex.err && stage_tma_fits(g, true))
        return launch_stage_tma64(stage, stretch, g, wl, co, ia, corr2, dt, visc, a, ex.err, st, dg, dg_done);
    if (phys != PHYS_NS && !wl.on && ex.impl != STAGE_MARCH && ex.err && stage <= 4 && mhd_tma_fits(g, true))
        return launch_mhd_tma64(phys, stage, stretch, g, co, ia, corr2, dt, visc, a, ex.err, st);
    if (ex.impl == STAGE_TMA && (phys == PHYS_NS || stage <= 4)) return cudaErrorNotSupported;
    launch_stage_any<double>(phys, stage, stretch, g, wl, co, ia, corr2, dt, visc, a, st);
    return cudaSuccess;
}

cudaError_t launch_stage32(int phys, int stage, bool stretch, const Geo &g, const Walls<float> &wl,
                           const Coef<float> &co, const float *ia, const float *corr2, float dt, float visc,
                           const StageArgs32 &a, cudaStream_t st, const StageExec &ex)
{
    if (phys == PHYS_NS && ex.impl != STAGE_MARCH && ex.err && stage_tma_fits(g, false))
        return launch_stage_tma32(stage, stretch, g, wl, co, ia, corr2, dt, visc, a, ex.err, st);
    if (phys != PHYS_NS && !wl.on && ex.impl != STAGE_MARCH && ex.err && stage <= 4 && mhd_tma_fits(g, false))
        return launch_mhd_tma32(phys, stage, stretch, g, co, ia, corr2, dt, visc, a, ex.err, st);
    if (ex.impl == STAGE_TMA && (phys == PHYS_NS || stage <= 4)) return cudaErrorNotSupported;
    launch_stage_any<float>(phys, stage, stretch, g, wl, co, ia, corr2, dt, visc, a, st);
    return cudaSuccess;
}

}  // namespace nova
