// Point arithmetic of the fused Navier-Stokes stage, shared by the two stage
// kernels (the register-queue march of nova_stage.cu and the TMA pipeline of
// nova_stage_tma.cu) so that both produce the same bits.
//
//   dU = dt*( -div(U,U) + laplacian(nu,U) )        (app/TG_Piosson/RKLoop.H:17-28)
//
// div(U,U) is the skew form of src/ex/div/div.hxx:84-172 evaluated as
// 1/2 sum_d [ A_d(U,U)_c + U_c D_d U_d ] (adv1 in nova_internal.cuh);
// laplacian follows src/ex/laplacian/laplacian.hxx:130-191 with the centre
// terms of the three directions folded into bsum and the stretched-z term
// -corr2 * dU/dz when the mesh is stretched.
#pragma once

#include "nova_internal.cuh"

namespace nova {

// vx/vy/vz(c, s): component c at offset s along i, j, k; u0 = U at the node;
// iak = 1/dzdxi(k): the z sums run with the uniform weights co.a[2], co.b[2]
// and are scaled by iak (first derivatives) or iak^2 (the Laplacian) once,
// which keeps the per-thread z weights out of the registers
template <typename T, int H, bool STRETCH, class VX, class VY, class VZ>
__device__ __forceinline__ void ns_rhs(const VX &vx, const VY &vy, const VZ &vz, const T (&u0)[3], const Coef<T> &co,
                                       T iak, T c2k, T visc, T (&rhs)[3])
{
    T adv[3] = {0, 0, 0}, lap[3] = {0, 0, 0}, div = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        adv[c] = adv1<T, H>(vx, c, 0, u0[0], co.a[0]) + adv1<T, H>(vy, c, 1, u0[1], co.a[1]);
        lap[c] = lsum<T, H>(vx, c, co.b[0]) + lsum<T, H>(vy, c, co.b[1]);
    }
    div = d1<T, H>(vx, 0, co.a[0]) + d1<T, H>(vy, 1, co.a[1]);
    const T iak2 = iak * iak;
    T duz[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        adv[c] = fma(iak, adv1<T, H>(vz, c, 2, u0[2], co.a[2]), adv[c]);
        lap[c] = fma(iak2, lsum<T, H>(vz, c, co.b[2]), lap[c]);
        if (STRETCH) duz[c] = iak * d1<T, H>(vz, c, co.a[2]);
    }
    div = fma(iak, d1<T, H>(vz, 2, co.a[2]), div);
    const T bsum = co.b2[0] + co.b2[1] + co.b2[2] * iak2;
#pragma unroll
    for (int c = 0; c < 3; c++)
        rhs[c] = T(-0.5) * fma(u0[c], div, adv[c]) + visc * (fma(-bsum, u0[c], lap[c]) - c2k * duz[c]);
}

// Stage update of one component at node o (classical RK4 of
// src/settings/settings.cpp:44-51 in the association order of
// app/TG_Piosson/RKLoop.H:24-28; STAGE 4 = the loop as written, one dU):
//   s=0: Y1 = U0 + dU*1/2   A = U0 + dU*1/6
//   s=1: Y2 = U0 + dU*1/2   A = A  + dU*1/3
//   s=2: Y3 = U0 + dU       A = A  + dU*1/3
//   s=3: U* = A  + dU*1/6
// y0: the stage state at the node; e0: U0 (stages 1, 2); e1: A (stages 1-3)
template <int STAGE>
__device__ __forceinline__ void rk_store64(const StageArgs64 &a, long long o, double y0, double e0, double e1, double du)
{
    const double w6 = 1.0 / 6.0, w3 = 1.0 / 3.0;
    if constexpr (STAGE == 4) {
        a.Ynext[o] = (((y0 + du * w6) + du * w3) + du * w3) + du * w6;
    } else if constexpr (STAGE == 0) {
        a.Ynext[o] = y0 + du * 0.5;
        a.A[o] = y0 + du * w6;
    } else if constexpr (STAGE == 1) {
        a.Ynext[o] = e0 + du * 0.5;
        a.A[o] = e1 + du * w3;
    } else if constexpr (STAGE == 2) {
        a.Ynext[o] = e0 + du * 1.0;
        a.A[o] = e1 + du * w3;
    } else {
        a.Ynext[o] = e1 + du * w6;
    }
}

// FP32-split: A is an FP32 sum of increments; the last stage adds it to the
// (hi, lo) base in FP64.  e0: U0hi (stages 1-3), e1: A, lo: U0lo (stages 3, 4)
template <int STAGE>
__device__ __forceinline__ void rk_store32(const StageArgs32 &a, long long o, float y0, float e0, float e1, float lo,
                                           float du)
{
    const float w6 = 1.0f / 6.0f, w3 = 1.0f / 3.0f;
    if constexpr (STAGE == 4) {
        const float inc = ((du * w6 + du * w3) + du * w3) + du * w6;
        const double x = ((double)y0 + (double)lo) + (double)inc;
        const float hi = (float)x;
        a.outhi[o] = hi;
        a.outlo[o] = (float)(x - (double)hi);
    } else if constexpr (STAGE == 0) {
        a.Ynext[o] = y0 + du * 0.5f;
        a.A[o] = du * w6;
    } else if constexpr (STAGE == 1) {
        a.Ynext[o] = e0 + du * 0.5f;
        a.A[o] = e1 + du * w3;
    } else if constexpr (STAGE == 2) {
        a.Ynext[o] = e0 + du;
        a.A[o] = e1 + du * w3;
    } else {
        const float inc = e1 + du * w6;
        const double x = ((double)e0 + (double)lo) + (double)inc;
        const float hi = (float)x;
        a.outhi[o] = hi;
        a.outlo[o] = (float)(x - (double)hi);
    }
}

}  // namespace nova
