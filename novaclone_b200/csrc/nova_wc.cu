// Weakly-compressible time advance: the compressible loop bodies of app/TG
// (rhoEqn.H, pEqn.H, UEqn.H) and app/shearLayerWC (UEqn.H, rhoEqn.H, pEqn.H,
// TEqn.H), each RK loop fused into one kernel per stage on the 2.5-D tile
// march of nova_tile.cuh (FP64, periodic meshes).
//
// Every loop is the reference's classical RK4 on a conserved quantity q*rho
// with rho frozen during the U and T loops (RK4W = 1/6, 1/3, 1/3, 1/6):
//   d   = dt * RHS(stage state)
//   acc = acc + RK4W[s] d                       (acc starts at rho*q0)
//   s<3: q = (rho*q0)/rho + c_s (d/rho),  c_s = (int(s/2)+1)/2 = 1/2, 1/2, 1
//   s=3: q = acc/rho
// (app/shearLayerWC/UEqn.H:11-41, TEqn.H:91-117; for rho itself, rhoEqn.H:53-78,
// q = rhoOld + c_s d and acc/1).
//   U:   RHS = -div(rho U, U) - grad p + laplacian(mu, U) [- (rho T) g]
//   rho: RHS = -div(rho U)
//   T:   RHS = -div(rho U, T) + laplacian(ka, T)
// div(V, F) is the skew form of src/ex/div/div.hxx:84-172 with V = rho U
// formed node by node from the halo'd rho and U; div(V) is src/ex/div/div.hxx:22-80.
// The EOS of pEqn.H is applied in the last rho stage: SHEAR p = (K rho) rho
// (app/shearLayerWC/pEqn.H:2), TG p = K (rho rho) with K = 50 (app/TG/pEqn.H:2).
#include "nova_internal.cuh"
#include "nova_tile.cuh"
#include "nova_wc.cuh"

namespace nova {

namespace {

constexpr int kH = 3;

__device__ __forceinline__ double rk4w(int s) { return s == 0 || s == 3 ? 1.0 / 6.0 : 1.0 / 3.0; }
__device__ __forceinline__ double stage_c(int s) { return (double)(int(s / 2) + 1) / 2.0; }

struct ZMetric {
    double iak, az[kH], bz[kH], bsum, c2k;
};

template <bool STRETCH>
__device__ __forceinline__ ZMetric zmetric(const Coef<double> &co, const double *ia, const double *corr2, int kw)
{
    ZMetric z;
    z.iak = ia[kw];
#pragma unroll
    for (int l = 0; l < kH; l++) {
        z.az[l] = co.a[2][l] * z.iak;
        z.bz[l] = co.b[2][l] * z.iak * z.iak;
    }
    z.bsum = co.b2[0] + co.b2[1] + co.b2[2] * z.iak * z.iak;
    z.c2k = STRETCH ? corr2[kw] : 0.0;
    return z;
}

// ---------------------------------------------------------------- U loop --
// halo'd comps: 0-2 U (stage state), 3 rho, 4 p; 5+d: rho U_d formed per node
template <int STAGE, bool STRETCH, bool BUOY>
__global__ void __launch_bounds__(kThreads, 1) k_wc_u(Geo g, Coef<double> co, const double *__restrict__ ia,
                                                      const double *__restrict__ corr2, WcArgs a, int ichunk)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, kH, 5> *>(smraw);
    const int ib = blockIdx.z * ichunk, ie = min(ib + ichunk, g.N0);
    const ZMetric zm = zmetric<STRETCH>(co, ia, corr2, wrapi(blockIdx.x * kTK + threadIdx.x, g.N2));
    const Walls<double> wl{};
    auto ld = [&](int c, long long o) -> double {
        return c < 3 ? a.Y[(long long)c * g.N3 + o] : (c == 3 ? a.rho[o] : a.p[o]);
    };
    // the pointwise operands (base, accumulator, T) of the next plane load
    // while this plane computes
    double q0n[3] = {0, 0, 0}, accn[3] = {0, 0, 0}, Tn = 0.0, q0c[3], accc[3], Tc = 0.0;
    auto pre = [&](long long nidx, bool load) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            q0c[c] = q0n[c];
            accc[c] = accn[c];
            if (STAGE > 0 && load) {
                q0n[c] = a.Q0[(long long)c * g.N3 + nidx];
                accn[c] = a.acc[(long long)c * g.N3 + nidx];
            }
        }
        Tc = Tn;
        if (BUOY && load) Tn = a.T[nidx];
    };
    tile_march<double, kH, 5, false>(g, wl, sm, ld, ib, ie, pre, [&](long long idx, auto &q, const auto &vx,
                                                                    const auto &vy, const auto &vz) {
        const double u0[3] = {q[kH][0], q[kH][1], q[kH][2]};
        const double r0 = q[kH][3];
        const double V0[3] = {r0 * u0[0], r0 * u0[1], r0 * u0[2]};
        double adv[3] = {0, 0, 0}, lap[3] = {0, 0, 0}, gp[3], duz[3] = {0, 0, 0}, divV = 0.0;
        auto dir = [&](const auto &v, int d, const double *aa, const double *bb, bool zdir) {
            auto vv = [&](int c, int s) -> double { return c < 5 ? v(c, s) : v(3, s) * v(c - 5, s); };
#pragma unroll
            for (int c = 0; c < 3; c++) {
                adv[c] += adv1<double, kH>(vv, c, 5 + d, V0[d], aa);
                lap[c] += lsum<double, kH>(v, c, bb);
                if (STRETCH && zdir) duz[c] = d1<double, kH>(v, c, aa);
            }
            divV += d1<double, kH>(vv, 5 + d, aa);
            gp[d] = d1<double, kH>(v, 4, aa);
        };
        dir(vx, 0, co.a[0], co.b[0], false);
        dir(vy, 1, co.a[1], co.b[1], false);
        dir(vz, 2, zm.az, zm.bz, true);
        const double T0 = BUOY ? Tc : 0.0;
        const double ir = 1.0 / r0;  // the divisions by rho below as products (within an ulp)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long o = (long long)c * g.N3 + idx;
            double e = -(0.5 * fma(u0[c], divV, adv[c]));
            e = e - gp[c];
            e = e + a.visc * (fma(-zm.bsum, u0[c], lap[c]) - zm.c2k * duz[c]);
            if (BUOY) e = e - (r0 * T0) * a.g[c];
            const double d = a.dt * e;
            const double q0 = STAGE == 0 ? u0[c] : q0c[c];
            const double acc = (STAGE == 0 ? r0 * q0 : accc[c]) + rk4w(STAGE) * d;
            if (STAGE < 3) {
                a.acc[o] = acc;
                a.Ynext[o] = (r0 * q0) * ir + stage_c(STAGE) * (d * ir);
            } else {
                a.Ynext[o] = acc * ir;
            }
        }
    });
}

// -------------------------------------------------------------- rho loop --
// halo'd comps: 0 rho (stage state), 1-3 U; 4+d: rho U_d formed per node
template <int STAGE, bool STRETCH, int EOS>
__global__ void __launch_bounds__(kThreads, 2) k_wc_rho(Geo g, Coef<double> co, const double *__restrict__ ia,
                                                        const double *__restrict__ corr2, WcArgs a, int ichunk)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, kH, 4> *>(smraw);
    const int ib = blockIdx.z * ichunk, ie = min(ib + ichunk, g.N0);
    const ZMetric zm = zmetric<STRETCH>(co, ia, corr2, wrapi(blockIdx.x * kTK + threadIdx.x, g.N2));
    const Walls<double> wl{};
    auto ld = [&](int c, long long o) -> double { return c == 0 ? a.Y[o] : a.U[(long long)(c - 1) * g.N3 + o]; };
    double q0n = 0.0, accn = 0.0, q0c = 0.0, accc = 0.0;  // next plane's base and accumulator, loading ahead
    auto pre = [&](long long nidx, bool load) {
        q0c = q0n;
        accc = accn;
        if (STAGE > 0 && load) {
            q0n = a.Q0[nidx];
            accn = a.acc[nidx];
        }
    };
    tile_march<double, kH, 4, false>(g, wl, sm, ld, ib, ie, pre, [&](long long idx, auto &q, const auto &vx,
                                                                    const auto &vy, const auto &vz) {
        double divV = 0.0;
        auto dir = [&](const auto &v, int d, const double *aa) {
            auto vv = [&](int c, int s) -> double { return v(0, s) * v(1 + c, s); };
            divV += d1<double, kH>(vv, d, aa);
        };
        dir(vx, 0, co.a[0]);
        dir(vy, 1, co.a[1]);
        dir(vz, 2, zm.az);
        const double d = a.dt * (-divV);
        const double r = q[kH][0];
        const double rold = STAGE == 0 ? r : q0c;
        const double acc = (STAGE == 0 ? r : accc) + rk4w(STAGE) * d;
        if (STAGE < 3) {
            a.acc[idx] = acc;
            a.Ynext[idx] = rold + stage_c(STAGE) * d;
        } else {
            a.Ynext[idx] = acc;
            a.p[idx] = EOS == NOVA_WC_SHEAR ? (a.eos_k * acc) * acc : a.eos_k * (acc * acc);
        }
    });
}

// ---------------------------------------------------------------- T loop --
// halo'd comps: 0 T (stage state), 1 rho, 2-4 U; 5+d: rho U_d formed per node
template <int STAGE, bool STRETCH>
__global__ void __launch_bounds__(kThreads, 2) k_wc_t(Geo g, Coef<double> co, const double *__restrict__ ia,
                                                      const double *__restrict__ corr2, WcArgs a, int ichunk)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, kH, 5> *>(smraw);
    const int ib = blockIdx.z * ichunk, ie = min(ib + ichunk, g.N0);
    const ZMetric zm = zmetric<STRETCH>(co, ia, corr2, wrapi(blockIdx.x * kTK + threadIdx.x, g.N2));
    const Walls<double> wl{};
    auto ld = [&](int c, long long o) -> double {
        return c == 0 ? a.Y[o] : (c == 1 ? a.rho[o] : a.U[(long long)(c - 2) * g.N3 + o]);
    };
    double q0n = 0.0, accn = 0.0, q0c = 0.0, accc = 0.0;  // next plane's base and accumulator, loading ahead
    auto pre = [&](long long nidx, bool load) {
        q0c = q0n;
        accc = accn;
        if (STAGE > 0 && load) {
            q0n = a.Q0[nidx];
            accn = a.acc[nidx];
        }
    };
    tile_march<double, kH, 5, false>(g, wl, sm, ld, ib, ie, pre, [&](long long idx, auto &q, const auto &vx,
                                                                    const auto &vy, const auto &vz) {
        const double t0 = q[kH][0], r0 = q[kH][1];
        const double V0[3] = {r0 * q[kH][2], r0 * q[kH][3], r0 * q[kH][4]};
        double adv = 0.0, lap = 0.0, duz = 0.0, divV = 0.0;
        auto dir = [&](const auto &v, int d, const double *aa, const double *bb, bool zdir) {
            auto vv = [&](int c, int s) -> double { return c < 5 ? v(c, s) : v(1, s) * v(c - 3, s); };
            adv += adv1<double, kH>(vv, 0, 5 + d, V0[d], aa);
            lap += lsum<double, kH>(v, 0, bb);
            if (STRETCH && zdir) duz = d1<double, kH>(v, 0, aa);
            divV += d1<double, kH>(vv, 5 + d, aa);
        };
        dir(vx, 0, co.a[0], co.b[0], false);
        dir(vy, 1, co.a[1], co.b[1], false);
        dir(vz, 2, zm.az, zm.bz, true);
        const double e = -(0.5 * fma(t0, divV, adv)) + a.visc * (fma(-zm.bsum, t0, lap) - zm.c2k * duz);
        const double d = a.dt * e;
        const double q0 = STAGE == 0 ? t0 : q0c;
        const double acc = (STAGE == 0 ? r0 * q0 : accc) + rk4w(STAGE) * d;
        const double ir = 1.0 / r0;  // the divisions by rho below as products (within an ulp)
        if (STAGE < 3) {
            a.acc[idx] = acc;
            a.Ynext[idx] = (r0 * q0) * ir + stage_c(STAGE) * (d * ir);
        } else {
            a.Ynext[idx] = acc * ir;
        }
    });
}

// ------------------------------------------------- hydrostatic initial p --
// app/shearLayerWC/shearLayer.cpp:114-150 with hydrostaticP.H:1-38: one thread
// per (i, j) column sums T dz g_z rho0 from the top node down.
__global__ void k_wc_hydrostatic(Geo g, double dz, double gz, double rho0, double K, const double *__restrict__ T,
                                 double *__restrict__ p, double *__restrict__ rho)
{
    const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (col >= (long long)g.N0 * g.N1) return;
    const long long base = col * g.N2;
    const double p0 = __dmul_rn(__dmul_rn(K, rho0), rho0);
    double cum = 0.0;
    for (int k = g.N2 - 1; k >= 0; k--) {
        // rounded term by term as the reference's host code (no fused multiply-add)
        cum = __dadd_rn(cum, __dmul_rn(__dmul_rn(__dmul_rn(T[base + k], dz), gz), rho0));
        const double pk = __dadd_rn(p0, cum);
        p[base + k] = pk;
        rho[base + k] = pow(pk / K, 0.5);
    }
}

}  // namespace

void launch_wc_stage(int loop, int stage, int wc_case, bool stretch, const Geo &g, const Coef<double> &co,
                     const double *ia, const double *corr2, const WcArgs &a, cudaStream_t st)
{
    // the rho and T loops fit 2 blocks per SM (128 registers), the U loop 1
    const int bps = loop == WC_LOOP_U ? 1 : 2;
    auto go = [&](auto kern, size_t smem) {
        static bool attr = false;  // once per kernel instantiation
        if (!attr) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            attr = true;
        }
        const int ch = pick_ichunk(g, bps);
        kern<<<tile_grid(g, ch), dim3(kTK, kTJ), smem, st>>>(g, co, ia, corr2, a, ch);
    };
    constexpr size_t s5 = tile_smem_bytes<double, kH, 5>(), s4 = tile_smem_bytes<double, kH, 4>();
#define WC_STAGES(EXPR)                                                                                 \
    switch (stage) {                                                                                    \
    case 0: { constexpr int S = 0; EXPR; } break;                                                      \
    case 1: { constexpr int S = 1; EXPR; } break;                                                      \
    case 2: { constexpr int S = 2; EXPR; } break;                                                      \
    default: { constexpr int S = 3; EXPR; } break;                                                     \
    }
    if (loop == WC_LOOP_U) {
        const bool buoy = wc_case == NOVA_WC_SHEAR;
        if (stretch) {
            if (buoy) { WC_STAGES(go(k_wc_u<S, true, true>, s5)) } else { WC_STAGES(go(k_wc_u<S, true, false>, s5)) }
        } else {
            if (buoy) { WC_STAGES(go(k_wc_u<S, false, true>, s5)) } else { WC_STAGES(go(k_wc_u<S, false, false>, s5)) }
        }
    } else if (loop == WC_LOOP_RHO) {
        if (stretch) {
            if (wc_case == NOVA_WC_SHEAR) { WC_STAGES(go(k_wc_rho<S, true, NOVA_WC_SHEAR>, s4)) }
            else { WC_STAGES(go(k_wc_rho<S, true, NOVA_WC_TG>, s4)) }
        } else {
            if (wc_case == NOVA_WC_SHEAR) { WC_STAGES(go(k_wc_rho<S, false, NOVA_WC_SHEAR>, s4)) }
            else { WC_STAGES(go(k_wc_rho<S, false, NOVA_WC_TG>, s4)) }
        }
    } else {
        if (stretch) { WC_STAGES(go(k_wc_t<S, true>, s5)) } else { WC_STAGES(go(k_wc_t<S, false>, s5)) }
    }
#undef WC_STAGES
}

void launch_wc_hydrostatic(const Geo &g, double dz, double gz, double rho0, double K, const double *T, double *p,
                           double *rho, cudaStream_t st)
{
    const long long cols = (long long)g.N0 * g.N1;
    k_wc_hydrostatic<<<(unsigned)((cols + 127) / 128), 128, 0, st>>>(g, dz, gz, rho0, K, T, p, rho);
}

}  // namespace nova
