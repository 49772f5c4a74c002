// Point arithmetic of the Navier-Stokes adjoint stage, shared by the tiled
// march (nova_adjoint.cu) and the TMA pipeline (nova_adj_tma.cu).
//
// Forward right-hand side F(U)_c = -N(U)_c + nu L U_c with the skew form
// N(U)_c = 1/2 sum_d [ D_d(U_d U_c) + U_d D_d U_c + U_c D_d U_d ]
// (app/TG_Piosson/RKLoop.H:17-22, src/ex/div/div.hxx:84-172).  With periodic
// central differences D_d^T = -D_d and L^T = L, for a direction g at the
// forward stage state Y:
//   xi_e = dt [ S_e - 1/2 At_e - 1/2 g_e div Y - nu bsum g_e ],
//   S_e  = sum_d sum_l [ g_e(+l) V+_l + g_e(-l) V-_l ],
//          V+-_l = +-(a_l/2)(Y_d(+-l) + Y_d(0)) + nu b_l
//          (the transposed advection A_d(Y, g) and the Laplacian, with weights
//          shared by the three components as in the forward stage),
//   At_d = sum_l a_l sum_c [ g_c(-l)(Y_c(0) + Y_c(-l)) - g_c(+l)(Y_c(0) + Y_c(+l))
//                            + g_c(0)(Y_c(+l) - Y_c(-l)) ]
//          (= -sum_c Y_c D_d g_c + sum_c g_c D_d Y_c - D_d(Y.g), the e = d terms),
// and xi is linear in g.
#pragma once

#include "nova_internal.cuh"

namespace nova {

// adjoint stage kinds: the MHD coupling transposes (numbered as launch_adj_mhd's
// kind) and the Navier-Stokes stage
enum AdjKind { ADJ_UB = 0, ADJ_BU = 1, ADJ_BB = 2, ADJ_NS = 3 };

// Building blocks at one node for a field P (comps 0-2 of vx/vy/vz, the
// forward stage state Y of the Navier-Stokes stage) and a direction g (comps
// 3-5), each vx/vy/vz(c, s) the component c at offset s along i, j, k:
//   Sx_e   = sum_d sum_l [ g_e(+l) V+_l + g_e(-l) V-_l ],  V+-_l = +-(a_l/2)(P_d(+-l) + P_d(0)) + nu b_l
//            (1/2 sum_d A_d(P, g)_e + nu lap(g)_e without its centre term)
//   At_d   = -sum_c P_c D_d g_c + sum_c g_c D_d P_c - D_d(P.g)
//   divP   = sum_d D_d P_d,  divG = sum_d D_d g_d (with DIVG)
// az, bz: the z weights a_l / dzdxi, b_l / dzdxi^2
template <typename T, int H, bool DIVG, class VX, class VY, class VZ>
__device__ __forceinline__ void adj_terms(const VX &vx, const VY &vy, const VZ &vz, const T (&p0)[3], const T (&g0)[3],
                                          const Coef<T> &co, const T *az, const T *bz, T nu, T (&Sx)[3], T (&At)[3],
                                          T &divP, T &divG)
{
    divP = 0;
    divG = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) Sx[c] = 0;
    auto dir = [&](const auto &v, int d, const T *aa, const T *bb) {
        T vp[H], vm[H];
        T at = 0;
#pragma unroll
        for (int l = 0; l < H; l++) {
            const T p = v(d, l + 1), m = v(d, -l - 1);
            const T ha = T(0.5) * aa[l], nb = nu * bb[l];
            vp[l] = fma(ha, p0[d] + p, nb);
            vm[l] = fma(-ha, p0[d] + m, nb);
            divP = fma(aa[l], p - m, divP);
            if (DIVG) divG = fma(aa[l], v(3 + d, l + 1) - v(3 + d, -l - 1), divG);
            T t = 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const T yp = v(c, l + 1), ym = v(c, -l - 1), gp = v(3 + c, l + 1), gm = v(3 + c, -l - 1);
                t = fma(-gp, p0[c] + yp, t);
                t = fma(gm, p0[c] + ym, t);
                t = fma(g0[c], yp - ym, t);
            }
            at = fma(aa[l], t, at);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            T r = Sx[c];
#pragma unroll
            for (int l = 0; l < H; l++) {
                r = fma(v(3 + c, l + 1), vp[l], r);
                r = fma(v(3 + c, -l - 1), vm[l], r);
            }
            Sx[c] = r;
        }
        At[d] = at;
    };
    dir(vx, 0, co.a[0], co.b[0]);
    dir(vy, 1, co.a[1], co.b[1]);
    dir(vz, 2, az, bz);
}

// the Navier-Stokes stage: xi = dt [ Sx - 1/2 At - 1/2 g divY - nu bsum g ] (P = Y)
template <typename T, int H, class VX, class VY, class VZ>
__device__ __forceinline__ void adj_xi(const VX &vx, const VY &vy, const VZ &vz, const T (&y0)[3], const T (&g0)[3],
                                       const Coef<T> &co, const T *az, const T *bz, T nu, T dt, T bsum, T (&xi)[3])
{
    T Sx[3], At[3], divY, divG;
    adj_terms<T, H, false>(vx, vy, vz, y0, g0, co, az, bz, nu, Sx, At, divY, divG);
#pragma unroll
    for (int e = 0; e < 3; e++) xi[e] = dt * (Sx[e] - T(0.5) * fma(g0[e], divY, At[e]) - nu * bsum * g0[e]);
}

// the z weights of adj_xi for the node column k (iak = 1/dzdxi(k))
template <typename T, int H>
__device__ __forceinline__ void adj_zweights(const Coef<T> &co, T iak, T (&az)[H], T (&bz)[H], T &bsum)
{
#pragma unroll
    for (int l = 0; l < H; l++) {
        az[l] = co.a[2][l] * iak;
        bz[l] = co.b[2][l] * iak * iak;
    }
    bsum = co.b2[0] + co.b2[1] + co.b2[2] * iak * iak;
}

// Reverse RK4 recursion of the classical stage loop (forward stages k_s =
// dt F(Y_s), Y1 = U, Y2 = U + k1/2, Y3 = U + k2/2, Y4 = U + k3,
// U* = U + (k1 + 2k2 + 2k3 + k4)/6), given mu = dJ/dU*:
//   s=4: g4 = mu/6        xi4 -> g3 = mu/3 + xi4        Lam = xi4
//   s=3:                  xi3 -> g2 = mu/3 + xi3/2      Lam += xi3
//   s=2:                  xi2 -> g1 = mu/6 + xi2/2      Lam += xi2
//   s=1:                  xi1 -> dJ/dU = mu + Lam + xi1
// A: AdjArgs (FP64: dJ/dU into Gout at s = 1) or AdjArgs32 (into lam, FP64)
template <typename T, int S, class A>
__device__ __forceinline__ void adj_store(const A &a, long long o, double mu, T lam, T xi)
{
    if constexpr (S == 4) {
        a.Gout[o] = (T)(mu * (1.0 / 3.0)) + xi;
        a.LamOut[o] = xi;
    } else if constexpr (S == 3) {
        a.Gout[o] = (T)(mu * (1.0 / 3.0)) + T(0.5) * xi;
        a.LamOut[o] = lam + xi;
    } else if constexpr (S == 2) {
        a.Gout[o] = (T)(mu * (1.0 / 6.0)) + T(0.5) * xi;
        a.LamOut[o] = lam + xi;
    } else if constexpr (sizeof(T) == 8) {
        a.Gout[o] = mu + (lam + xi);
    } else {
        a.lam[o] = mu + (double)(lam + xi);
    }
}

}  // namespace nova
