// Per-node terms of the diagnostics history, shared by the diagnostics kernel
// (nova_ops.cu) and the fused first stage (nova_stage_tma.cu).
//
// A history row restates the per-step diagnostics of the apps:
//   app/OT_Poisson/OT.cpp:132-176  Ek, Em, Jav = mean|J|, Jmax = max|J|,
//                                  omega = mean|ex::curl(U)|, epsilon, Umax
//                                  (J = ex::curl(B), BEqn.H:97-98; means and
//                                  maxima over the unique nodes)
//   src/Tools/Tools.cpp:9-41       tools::CFL (cfl_y and cfl_z keep only the
//                                  last node's value against cfl_x)
//   tools::maximum(ex::div(U)), (ex::div(B))
//                                  app/TG_Piosson/RKLoop.H:42-51, OT_Poisson/BEqn.H:46-54
// plus 1/2 <|curl U|^2> and 1/2 <|curl B|^2> with the central 6th-order curl
// (the enstrophy; ex::curl is the Q1 stencil of ex::grad(vector),
// src/ex/grad/grad.cpp:82-94, whose magnitude the apps average).
#pragma once

#include "nova_internal.cuh"

namespace nova {

// Q1 derivative of ex::grad(Field<vector>): sum_l c_l/(l+1)/delta (f(+l) - f(-1-l)),
// a[l] = c_l / (2 (l+1) delta) (z weights already divided by dzdxi)
template <int H, class V>
__device__ __forceinline__ double q1d(const V &v, int c, const double *a)
{
    double r = 0.0;
#pragma unroll
    for (int l = 0; l < H; l++) r = fma(2.0 * a[l], v(c, l) - v(c, -1 - l), r);
    return r;
}

// |ex::curl(F)| and 1/2 |curl F|^2 (central) of the vector at components c0..c0+2;
// z derivatives are taken with the weights az and then scaled by iz
template <int H, class VX, class VY, class VZ>
__device__ __forceinline__ void curl_terms(const VX &vx, const VY &vy, const VZ &vz, int c0, const double *ax,
                                           const double *ay, const double *az, double iz, double &q1mag,
                                           double &half_sq)
{
    // one curl component at a time (few values live at once)
    double w2, c2, w, c;
    w = q1d<H>(vy, c0 + 2, ay) - q1d<H>(vz, c0 + 1, az) * iz;
    c = d1<double, H>(vy, c0 + 2, ay) - d1<double, H>(vz, c0 + 1, az) * iz;
    w2 = w * w;
    c2 = c * c;
    w = q1d<H>(vz, c0 + 0, az) * iz - q1d<H>(vx, c0 + 2, ax);
    c = d1<double, H>(vz, c0 + 0, az) * iz - d1<double, H>(vx, c0 + 2, ax);
    w2 = fma(w, w, w2);
    c2 = fma(c, c, c2);
    w = q1d<H>(vx, c0 + 1, ax) - q1d<H>(vy, c0 + 0, ay);
    c = d1<double, H>(vx, c0 + 1, ax) - d1<double, H>(vy, c0 + 0, ay);
    w2 = fma(w, w, w2);
    c2 = fma(c, c, c2);
    q1mag = sqrt(w2);
    half_sq = 0.5 * c2;
}

// the U terms only (6 running values: the fused stage's register budget),
// expanded to the kDiagParts layout with zero B terms by part()
struct DiagAccU {
    double ek = 0.0, om = 0.0, ens = 0.0, umax = 0.0, mdu = 0.0, ux = 0.0;
    __device__ __forceinline__ void add(const double (&u)[3], double divu, double q1, double hs)
    {
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        ek += 0.5 * uu;
        om += q1;
        ens += hs;
        umax = fmax(umax, sqrt(uu));
        mdu = fmax(mdu, fabs(divu));
        ux = fmax(ux, u[0]);
    }
    __device__ __forceinline__ void warp_reduce()
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ek += __shfl_down_sync(0xffffffffu, ek, o);
            om += __shfl_down_sync(0xffffffffu, om, o);
            ens += __shfl_down_sync(0xffffffffu, ens, o);
            umax = fmax(umax, __shfl_down_sync(0xffffffffu, umax, o));
            mdu = fmax(mdu, __shfl_down_sync(0xffffffffu, mdu, o));
            ux = fmax(ux, __shfl_down_sync(0xffffffffu, ux, o));
        }
    }
    __device__ __forceinline__ double part(int q) const
    {
        switch (q) {
        case DP_EK: return ek;
        case DP_OMEGA: return om;
        case DP_ENSU: return ens;
        case DP_UMAX: return umax;
        case DP_DIVU: return mdu;
        case DP_UX: return ux;
        default: return 0.0;
        }
    }
};

// DiagAccU's six values kept in shared memory, one column per thread (slot q
// of thread t at m[q * stride + t]), for a kernel whose registers are taken
// (the fused FP64 stage)
struct DiagAccSm {
    double *m;
    int stride;
    __device__ __forceinline__ void init()
    {
#pragma unroll
        for (int q = 0; q < 6; q++) m[q * stride] = 0.0;
    }
    __device__ __forceinline__ void add(const double (&u)[3], double divu, double q1, double hs)
    {
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        m[0] += 0.5 * uu;
        m[stride] += q1;
        m[2 * stride] += hs;
        m[3 * stride] = fmax(m[3 * stride], sqrt(uu));
        m[4 * stride] = fmax(m[4 * stride], fabs(divu));
        m[5 * stride] = fmax(m[5 * stride], u[0]);
    }
    __device__ __forceinline__ DiagAccU load() const
    {
        DiagAccU a;
        a.ek = m[0];
        a.om = m[stride];
        a.ens = m[2 * stride];
        a.umax = m[3 * stride];
        a.mdu = m[4 * stride];
        a.ux = m[5 * stride];
        return a;
    }
};

// running per-thread values of the kDiagParts partials (layout in nova_internal.cuh)
struct DiagAcc {
    double v[kDiagParts];
    __device__ DiagAcc()
    {
#pragma unroll
        for (int q = 0; q < kDiagParts; q++) v[q] = 0.0;
    }
    // the U terms of a node: u the vector, divu its divergence, q1/hs its curl
    // terms; unique = the node is one of the unique nodes the means cover
    __device__ __forceinline__ void add_u(const double (&u)[3], double divu, double q1, double hs, bool unique)
    {
        const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        if (unique) {
            v[DP_EK] += 0.5 * uu;
            v[DP_OMEGA] += q1;
            v[DP_ENSU] += hs;
            v[DP_UMAX] = fmax(v[DP_UMAX], sqrt(uu));
        }
        v[DP_DIVU] = fmax(v[DP_DIVU], fabs(divu));
        v[DP_UX] = fmax(v[DP_UX], u[0]);
    }
    __device__ __forceinline__ void add_b(const double (&b)[3], double divb, double q1, double hs, bool unique)
    {
        if (unique) {
            v[DP_EM] += 0.5 * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
            v[DP_JAV] += q1;
            v[DP_ENSB] += hs;
            v[DP_JMAX] = fmax(v[DP_JMAX], q1);
        }
        v[DP_DIVB] = fmax(v[DP_DIVB], fabs(divb));
    }
    // warp reduction (fixed order); the result is valid in lane 0
    __device__ __forceinline__ void warp_reduce()
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < kDiagParts; q++) {
                const double x = __shfl_down_sync(0xffffffffu, v[q], o);
                v[q] = q >= DP_DIVU ? fmax(v[q], x) : v[q] + x;
            }
    }
};

}  // namespace nova
