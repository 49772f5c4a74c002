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

// One direction of the fused sum  -1/2 A_d(U,U)_c + visc * lsum_d(U_c),
// accumulated onto s[c]:
//   s[c] += sum_l [ U_c(+l) W+_l + U_c(-l) W-_l ],
//   W+_l = -a_l/2 (U_d(+l) + U_d(0)) + vb_l,   W-_l = a_l/2 (U_d(-l) + U_d(0)) + vb_l
// The weights depend on the direction only, so the three components share
// them: one product per neighbour instead of one for the advective and one for
// the diffusive term.  dd += D_d U_d (the divergence term).
template <typename T, int H, class V>
__device__ __forceinline__ void ns_dir(const V &v, int d, T v0, const T *ha, const T *a, const T (&vb)[H], T (&s)[3],
                                       T &dd)
{
    T wp[H], wm[H];
#pragma unroll
    for (int l = 0; l < H; l++) {
        const T p = v(d, l + 1), m = v(d, -l - 1);
        wp[l] = fma(-ha[l], p + v0, vb[l]);
        wm[l] = fma(ha[l], m + v0, vb[l]);
        dd = fma(a[l], p - m, dd);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        T r = s[c];
#pragma unroll
        for (int l = 0; l < H; l++) {
            r = fma(v(c, l + 1), wp[l], r);
            r = fma(v(c, -l - 1), wm[l], r);
        }
        s[c] = r;
    }
}

// vx/vy/vz(c, s): component c at offset s along i, j, k; u0 = U at the node;
// divu receives sum_d D_d U_d at the node (the divergence of the stage state);
// iak = 1/dzdxi(k): the z weights are a_l iak and b_l iak^2, applied as the
// uniform weights with vb = visc iak b_l and the z sum scaled by iak (it is
// evaluated first), so no per-node weight tables live in registers.
// Algebraically the skew form and Laplacian above; rounding differs from the
// term-by-term order at the level of a few ulps of the largest term.
template <typename T, int H, bool STRETCH, class VX, class VY, class VZ>
__device__ __forceinline__ void ns_rhs(const VX &vx, const VY &vy, const VZ &vz, const T (&u0)[3], const Coef<T> &co,
                                       const StageCoef<T> &sc, T iak, T c2k, T visc, T (&rhs)[3], T &divu)
{
    T s[3] = {0, 0, 0}, dv = 0;
    {
        T vb[H];
        const T viak = visc * iak;
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = viak * co.b[2][l];
        ns_dir<T, H>(vz, 2, u0[2], sc.ha[2], co.a[2], vb, s, dv);
#pragma unroll
        for (int c = 0; c < 3; c++) s[c] *= iak;
        dv *= iak;
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = sc.vb[0][l];
        ns_dir<T, H>(vx, 0, u0[0], sc.ha[0], co.a[0], vb, s, dv);
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = sc.vb[1][l];
        ns_dir<T, H>(vy, 1, u0[1], sc.ha[1], co.a[1], vb, s, dv);
    }
    divu = dv;
    const T bsum = fma(co.b2[2], iak * iak, co.b2[0] + co.b2[1]);
    const T K = fma(T(-0.5), dv, -visc * bsum);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        T r = s[c];
        if (STRETCH) r = fma(-visc * c2k, iak * d1<T, H>(vz, c, co.a[2]), r);
        rhs[c] = fma(u0[c], K, r);
    }
}

// The MHD right-hand sides (comps 0-2 of the accessors: the evolved field E,
// 3-5: the frozen one F), ex::div(V,F) in the skew form above:
//   U loop (app/OT_Poisson/UEqn.H:16-23), E = U, F = B:
//     -div(U,U) + laplacian(nu,U) + div(B,B) - grad(0.5*(B&B))
//   B loop (app/OT_Poisson/BEqn.H:72-78), E = B, F = U:
//     -div(U,B) + div(B,U) + laplacian(eta,B)
// Both are, per direction d, shared-weight sums over the neighbours (the
// ns_dir form): -1/2 A_d(U,E)_c + visc lsum_d(E_c) = sum_l E_c(+-l) W+-_l with
// W+-_l = -+(a_l/2)(U_d(+-l) + U_d(0)) + visc b_l, and +1/2 A_d(B,F)_c =
// sum_l F_c(+-l) V+-_l with V+-_l = +-(a_l/2)(B_d(+-l) + B_d(0)); the
// remaining skew terms are -1/2 E_c div U + 1/2 F_c div B.  So
//   rhs_c = sum_d [E-sum + F-sum] + E_c(0) K1 + F_c(0) K2 (- d_c 0.5|B|^2, U loop),
//   K1 = -div U / 2 - visc bsum,  K2 = div B / 2,
// with the stretched-z term -visc c2k dE_c/dz.  z is evaluated first with the
// uniform weights (and vb = visc iak b_l) and scaled by iak = 1/dzdxi, as in
// ns_rhs.  About 310 operations per node for the U loop (the term-by-term
// form: about 430).

// one direction d: s[c] += the E- and F-sums; du += D_d U_d, db += D_d B_d,
// gb (GRADB) = D_d 0.5|B|^2.  uo, bo: the component offsets of U and B.
template <typename T, int H, bool GRADB, class V>
__device__ __forceinline__ void mhd_dir(const V &v, int d, int uo, int bo, T ud0, T bd0, const T *ha, const T *a,
                                        const T (&vb)[H], T (&s)[3], T &du, T &db, T &gb)
{
    T wp[H], wm[H], xp[H], xm[H];
#pragma unroll
    for (int l = 0; l < H; l++) {
        const T up = v(uo + d, l + 1), um = v(uo + d, -l - 1);
        wp[l] = fma(-ha[l], up + ud0, vb[l]);
        wm[l] = fma(ha[l], um + ud0, vb[l]);
        du = fma(a[l], up - um, du);
        const T bp = v(bo + d, l + 1), bm = v(bo + d, -l - 1);
        xp[l] = ha[l] * (bp + bd0);
        xm[l] = -ha[l] * (bm + bd0);
        db = fma(a[l], bp - bm, db);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        T r = s[c];
#pragma unroll
        for (int l = 0; l < H; l++) {
            r = fma(v(c, l + 1), wp[l], r);
            r = fma(v(c, -l - 1), wm[l], r);
        }
#pragma unroll
        for (int l = 0; l < H; l++) {
            r = fma(v(3 + c, l + 1), xp[l], r);
            r = fma(v(3 + c, -l - 1), xm[l], r);
        }
        s[c] = r;
    }
    if constexpr (GRADB) {
        auto e = [&](int, int t) -> T {
            return (v(bo, t) * v(bo, t) + v(bo + 1, t) * v(bo + 1, t) + v(bo + 2, t) * v(bo + 2, t)) * T(0.5);
        };
        gb = d1<T, H>(e, 0, a);
    }
}

// PHYS_MHD_U (E = U, F = B) or PHYS_MHD_B (E = B, F = U); e0, f0 = E, F at the
// node; iak, c2k the column's metric terms (as ns_rhs)
template <typename T, int H, bool STRETCH, bool ULOOP, class VX, class VY, class VZ>
__device__ __forceinline__ void mhd_rhs(const VX &vx, const VY &vy, const VZ &vz, const T (&e0)[3], const T (&f0)[3],
                                        const Coef<T> &co, const StageCoef<T> &sc, T iak, T c2k, T visc,
                                        T (&rhs)[3])
{
    constexpr int uo = ULOOP ? 0 : 3, bo = ULOOP ? 3 : 0;
    const T (&u0)[3] = ULOOP ? e0 : f0;
    const T (&b0)[3] = ULOOP ? f0 : e0;
    T s[3] = {0, 0, 0}, du = 0, db = 0, gb[3] = {0, 0, 0};
    {
        T vb[H];
        const T viak = visc * iak;
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = viak * co.b[2][l];
        mhd_dir<T, H, ULOOP>(vz, 2, uo, bo, u0[2], b0[2], sc.ha[2], co.a[2], vb, s, du, db, gb[2]);
#pragma unroll
        for (int c = 0; c < 3; c++) s[c] *= iak;
        du *= iak;
        db *= iak;
        gb[2] *= iak;
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = sc.vb[0][l];
        mhd_dir<T, H, ULOOP>(vx, 0, uo, bo, u0[0], b0[0], sc.ha[0], co.a[0], vb, s, du, db, gb[0]);
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = sc.vb[1][l];
        mhd_dir<T, H, ULOOP>(vy, 1, uo, bo, u0[1], b0[1], sc.ha[1], co.a[1], vb, s, du, db, gb[1]);
    }
    const T bsum = fma(co.b2[2], iak * iak, co.b2[0] + co.b2[1]);
    const T K1 = fma(T(-0.5), du, -visc * bsum), K2 = T(0.5) * db;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        T r = fma(f0[c], K2, s[c]);
        if constexpr (ULOOP) r -= gb[c];
        if (STRETCH) r = fma(-visc * c2k, iak * d1<T, H>(vz, c, co.a[2]), r);
        rhs[c] = fma(e0[c], K1, r);
    }
}

// Stage update of one component at node o (classical RK4 of
// src/settings/settings.cpp:44-51 in the association order of
// app/TG_Piosson/RKLoop.H:24-28; STAGE 4 = the loop as written, one dU):
//   s=0: Y1 = U0 + dU*1/2   A = U0 + dU*1/6
//   s=1: Y2 = U0 + dU*1/2   A = A  + dU*1/3
//   s=2: Y3 = U0 + dU       A = A  + dU*1/3
//   s=3: U* = A  + dU*1/6
//   s=5: U* = U0 + dU*w   (app/shearLayer/UEqn.H:28-29, w = RK4[rk] of the stage)
// y0: the stage state at the node; e0: U0 (stages 1, 2, 5); e1: A (stages 1-3)
// (every product-sum an explicit fma and the stage-2 sum unfused, so the
// result does not depend on the compiler's contraction choices)
template <int STAGE> struct RK64 {
    // the (Ynext, A) values of one node
    __device__ __forceinline__ static void eval(const StageArgs64 &a, double y0, double e0, double e1, double du,
                                                double &yn, double &an)
    {
        const double w6 = 1.0 / 6.0, w3 = 1.0 / 3.0;
        if constexpr (STAGE == 5) {
            yn = fma(du, a.w, e0);
        } else if constexpr (STAGE == 4) {
            yn = fma(du, w6, fma(du, w3, fma(du, w3, fma(du, w6, y0))));
        } else if constexpr (STAGE == 0) {
            yn = fma(du, 0.5, y0);
            an = fma(du, w6, y0);
        } else if constexpr (STAGE == 1) {
            yn = fma(du, 0.5, e0);
            an = fma(du, w3, e1);
        } else if constexpr (STAGE == 2) {
            yn = __dadd_rn(e0, du);  // not contracted with du = dt * rhs
            an = fma(du, w3, e1);
        } else {
            yn = fma(du, w6, e1);
        }
    }
    static constexpr bool kA = STAGE <= 2;  // the stage writes the accumulator
};

template <int STAGE>
__device__ __forceinline__ void rk_store64(const StageArgs64 &a, long long o, double y0, double e0, double e1, double du)
{
    double yn, an;
    RK64<STAGE>::eval(a, y0, e0, e1, du, yn, an);
    a.Ynext[o] = yn;
    if constexpr (RK64<STAGE>::kA) a.A[o] = an;
}

// FP32-split: A is an FP32 sum of increments; the last stage (3, 4, or the
// shear-layer stage 5) adds it to the (hi, lo) base in FP64 and stores U* as a
// (hi, lo) pair, or in FP64 for the projection (a.out64).  e0: U0hi (stages
// 1-3, 5), e1: A, lo: U0lo (stages 3-5)
template <int STAGE>
__device__ __forceinline__ void rk_store32(const StageArgs32 &a, long long o, float y0, float e0, float e1, float lo,
                                           float du)
{
    // every product-sum is an explicit fmaf, so that the paired form
    // (rk_store32x2) reproduces these bits
    const float w6 = 1.0f / 6.0f, w3 = 1.0f / 3.0f;
    if constexpr (STAGE == 5) {
        const double x = ((double)e0 + (double)lo) + (double)(du * a.w);
        if (a.out64) {
            a.out64[o] = x;
            return;
        }
        const float hi = (float)x;
        a.outhi[o] = hi;
        a.outlo[o] = (float)(x - (double)hi);
    } else if constexpr (STAGE == 4) {
        const float inc = fmaf(du, w6, fmaf(du, w3, fmaf(du, w3, du * w6)));
        const double x = ((double)y0 + (double)lo) + (double)inc;
        if (a.out64) {
            a.out64[o] = x;
            return;
        }
        const float hi = (float)x;
        a.outhi[o] = hi;
        a.outlo[o] = (float)(x - (double)hi);
    } else if constexpr (STAGE == 0) {
        a.Ynext[o] = fmaf(du, 0.5f, y0);
        a.A[o] = du * w6;
    } else if constexpr (STAGE == 1) {
        a.Ynext[o] = fmaf(du, 0.5f, e0);
        a.A[o] = fmaf(du, w3, e1);
    } else if constexpr (STAGE == 2) {
        a.Ynext[o] = __fadd_rn(e0, du);  // not contracted with du = dt * rhs
        a.A[o] = fmaf(du, w3, e1);
    } else {
        const float inc = fmaf(du, w6, e1);
        const double x = ((double)e0 + (double)lo) + (double)inc;
        if (a.out64) {
            a.out64[o] = x;
            return;
        }
        const float hi = (float)x;
        a.outhi[o] = hi;
        a.outlo[o] = (float)(x - (double)hi);
    }
}

// ---------------------------------------------------------------------------
// Paired FP32: two adjacent k nodes per thread in the sm_100 f32x2
// instructions (one FFMA2 / FADD2 / FMUL2 per pair).  Each function is the
// scalar one above operation for operation (fma for fma, product for product,
// p - m as fma(m, -1, p), which rounds identically), so the pair produces the
// bits of two scalar evaluations.
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

template <int H, class V>
__device__ __forceinline__ void ns_dir2(const V &v, int d, float2 v0, const float *ha, const float *a,
                                        const float2 (&vb)[H], float2 (&s)[3], float2 &dd)
{
    float2 wp[H], wm[H];
#pragma unroll
    for (int l = 0; l < H; l++) {
        const float2 p = v(d, l + 1), m = v(d, -l - 1);
        wp[l] = fma2(f2(-ha[l]), add2(p, v0), vb[l]);
        wm[l] = fma2(f2(ha[l]), add2(m, v0), vb[l]);
        dd = fma2(f2(a[l]), sub2(p, m), dd);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float2 r = s[c];
#pragma unroll
        for (int l = 0; l < H; l++) {
            r = fma2(v(c, l + 1), wp[l], r);
            r = fma2(v(c, -l - 1), wm[l], r);
        }
        s[c] = r;
    }
}

template <int H, class V> __device__ __forceinline__ float2 d1x2(const V &v, int c, const float *a)
{
    float2 r = mul2(f2(a[0]), sub2(v(c, 1), v(c, -1)));
#pragma unroll
    for (int l = 1; l < H; l++) r = fma2(f2(a[l]), sub2(v(c, l + 1), v(c, -l - 1)), r);
    return r;
}

// ns_rhs for a pair: accessors return float2 pairs; iak, c2k the columns' metric terms
template <int H, bool STRETCH, class VX, class VY, class VZ>
__device__ __forceinline__ void ns_rhs2(const VX &vx, const VY &vy, const VZ &vz, const float2 (&u0)[3],
                                        const Coef<float> &co, const StageCoef<float> &sc, float2 iak, float2 c2k,
                                        float visc, float2 (&rhs)[3])
{
    const float2 z = f2(0.0f);
    float2 s[3] = {z, z, z}, dv = z;
    {
        float2 vb[H];
        const float2 viak = mul2(f2(visc), iak);
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = mul2(viak, f2(co.b[2][l]));
        ns_dir2<H>(vz, 2, u0[2], sc.ha[2], co.a[2], vb, s, dv);
#pragma unroll
        for (int c = 0; c < 3; c++) s[c] = mul2(s[c], iak);
        dv = mul2(dv, iak);
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = f2(sc.vb[0][l]);
        ns_dir2<H>(vx, 0, u0[0], sc.ha[0], co.a[0], vb, s, dv);
#pragma unroll
        for (int l = 0; l < H; l++) vb[l] = f2(sc.vb[1][l]);
        ns_dir2<H>(vy, 1, u0[1], sc.ha[1], co.a[1], vb, s, dv);
    }
    const float2 bsum = fma2(f2(co.b2[2]), mul2(iak, iak), f2(co.b2[0] + co.b2[1]));
    const float2 K = fma2(f2(-0.5f), dv, mul2(f2(-visc), bsum));
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float2 r = s[c];
        if (STRETCH) r = fma2(mul2(f2(-visc), c2k), mul2(iak, d1x2<H>(vz, c, co.a[2])), r);
        rhs[c] = fma2(u0[c], K, r);
    }
}

__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }

// U* = (hi, lo) base + FP32 increment, per node in FP64 (rk_store32's last step)
__device__ __forceinline__ void store_split2(const StageArgs32 &a, long long o, float2 base, float2 lo, float2 inc)
{
    const double x0 = ((double)base.x + (double)lo.x) + (double)inc.x;
    const double x1 = ((double)base.y + (double)lo.y) + (double)inc.y;
    if (a.out64) {
        *reinterpret_cast<double2 *>(a.out64 + o) = make_double2(x0, x1);
        return;
    }
    const float h0 = (float)x0, h1 = (float)x1;
    st2(a.outhi + o, make_float2(h0, h1));
    st2(a.outlo + o, make_float2((float)(x0 - (double)h0), (float)(x1 - (double)h1)));
}

// rk_store32 for the pair of nodes o, o + 1
template <int STAGE>
__device__ __forceinline__ void rk_store32x2(const StageArgs32 &a, long long o, float2 y0, float2 e0, float2 e1,
                                             float2 lo, float2 du)
{
    static_assert(STAGE >= 0 && STAGE <= 5, "stages 0-5");
    const float2 w6 = f2(1.0f / 6.0f), w3 = f2(1.0f / 3.0f), h = f2(0.5f);
    if constexpr (STAGE == 5) {
        store_split2(a, o, e0, lo, mul2(du, f2(a.w)));
    } else if constexpr (STAGE == 4) {
        store_split2(a, o, y0, lo, fma2(du, w6, fma2(du, w3, fma2(du, w3, mul2(du, w6)))));
    } else if constexpr (STAGE == 0) {
        st2(a.Ynext + o, fma2(du, h, y0));
        st2(a.A + o, mul2(du, w6));
    } else if constexpr (STAGE == 1) {
        st2(a.Ynext + o, fma2(du, h, e0));
        st2(a.A + o, fma2(du, w3, e1));
    } else if constexpr (STAGE == 2) {
        st2(a.Ynext + o, add2(e0, du));
        st2(a.A + o, fma2(du, w3, e1));
    } else {
        store_split2(a, o, e0, lo, fma2(du, w6, e1));
    }
}

}  // namespace nova
