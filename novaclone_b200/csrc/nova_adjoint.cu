// Discrete adjoint of the Navier-Stokes stage: xi = dt * J_F(Y)^T g, fused
// with the reverse recursion of the classical RK4 stage loop (the point
// arithmetic and the recursion are in nova_adj_math.cuh); tiled march, used
// where the TMA pipeline of nova_adj_tma.cu does not fit the mesh and for the
// FP32-split adjoint.  The MHD coupling transposes follow below.
#include "nova_adj_math.cuh"
#include "nova_internal.cuh"
#include "nova_tile.cuh"

namespace nova {

namespace {

// T: the arithmetic and storage type of the stage states, the directions g
// and the running sum Lam (double, or float for the FP32-split adjoint, A =
// AdjArgs32); mu and the resulting dJ/dU are FP64 in both.
template <typename T, int H, int S, class A>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 8 ? 1 : 2)
    k_adj_stage(Geo g, Coef<T> co, const T *__restrict__ ia, T dt, T nu, A a, int ichunk)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<T, H, 6> *>(smraw);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);
    T az[H], bz[H], bsum;
    adj_zweights<T, H>(co, ia[kw], az, bz, bsum);
    // comps 0-2: forward stage state Y, 3-5: adjoint stage direction g (= mu/6 at s=4)
    auto ld = [&](int c, long long o) -> T {
        if (c < 3) return a.Y[(long long)c * g.N3 + o];
        if constexpr (S == 4) return (T)(a.mu[(long long)(c - 3) * g.N3 + o] * (1.0 / 6.0));
        return a.G[(long long)(c - 3) * g.N3 + o];
    };
    const Walls<T> wl{};  // the adjoint is built for periodic meshes
    tile_march<T, H, 6, false>(g, wl, sm, ld, ib, ie, [&](long long idx, auto &q, const auto &vx, const auto &vy,
                                                  const auto &vz) {
        double mu[3];
        T lam[3] = {0, 0, 0};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            mu[c] = a.mu[(long long)c * g.N3 + idx];
            if (S != 4) lam[c] = a.Lam[(long long)c * g.N3 + idx];
        }
        const T y0[3] = {q[H][0], q[H][1], q[H][2]};
        const T g0[3] = {q[H][3], q[H][4], q[H][5]};
        T xi[3];
        adj_xi<T, H>(vx, vy, vz, y0, g0, co, az, bz, nu, dt, bsum, xi);
#pragma unroll
        for (int e = 0; e < 3; e++) adj_store<T, S>(a, (long long)e * g.N3 + idx, mu[e], lam[e], xi[e]);
    });
}

template <typename T, int S, class A>
void launch_s(const Geo &g, const Coef<T> &co, const T *ia, T dt, T nu, const A &a, cudaStream_t st)
{
    constexpr size_t smem = tile_smem_bytes<T, 3, 6>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_adj_stage<T, 3, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int ch = pick_ichunk(g, sizeof(T) == 8 ? 1 : 2);
    k_adj_stage<T, 3, S, A><<<tile_grid(g, ch), dim3(kTK, kTJ), smem, st>>>(g, co, ia, dt, nu, a, ch);
}

template <typename T, class A>
void launch_adj(int s, const Geo &g, const Coef<T> &co, const T *ia, T dt, T nu, const A &a, cudaStream_t st)
{
    switch (s) {
    case 4: launch_s<T, 4>(g, co, ia, dt, nu, a, st); break;
    case 3: launch_s<T, 3>(g, co, ia, dt, nu, a, st); break;
    case 2: launch_s<T, 2>(g, co, ia, dt, nu, a, st); break;
    default: launch_s<T, 1>(g, co, ia, dt, nu, a, st); break;
    }
}

// ----------------------------------------------------------- MHD adjoint --
// Building blocks for div(V,F)_c = 1/2 sum_d [D_d(V_d F_c) + V_d D_d F_c + F_c D_d V_d]
// with D_d^T = -D_d (periodic central differences), for an adjoint direction g:
//   T_F(V; g)_c = (d div(V,F)/dF)^T g = 1/2 [ -sum_d A_d(V,g)_c + g_c sum_d D_d V_d ]
//   T_V(F; g)_e = (d div(V,F)/dV)^T g = 1/2 [ -sum_c F_c D_e g_c + sum_c g_c D_e F_c - D_e(sum_c F_c g_c) ]
// (for the Navier-Stokes term div(U,U) the transpose is T_F(U) + T_V(U), k_adj_stage).
// MHD right-hand sides (app/OT_Poisson/UEqn.H:16-23, BEqn.H:72-78):
//   F_U = -div(U,U) + nu L U + div(B,B) - grad(1/2 |B|^2)   (B frozen in the U loop)
//   F_B = -div(U,B) + div(B,U) + eta L B                    (U frozen in the B loop)
// with (d grad(1/2|B|^2)/dB)^T g = -B_e div g, the kernels compute, for the
// stage direction g_S and the field P in comps 0-2 of the march:
//   KIND_UB: lambda_B += dt [T_F(B) + T_V(B) + B div g]     P = B^n (dF_U/dB)
//   KIND_BU: lambda_U += dt [T_F(B) - T_V(B)]               P = Z_S, the B stage state (dF_B/dU)
//   KIND_BB: xi = dt [-T_F(U') + T_V(U') + eta L g]          P = U^{n+1} (dF_B/dB; F_B is linear in B)
//            with the reverse RK4 recursion of k_adj_stage in the epilogue
enum AdjMhdKind { KIND_UB = 0, KIND_BU = 1, KIND_BB = 2 };

template <int KIND, int S>
__global__ void __launch_bounds__(kThreads, 1) k_adj_mhd(Geo g, Coef<double> co, const double *__restrict__ ia,
                                                         double dt, double visc, AdjArgs a, double *acc, int ichunk)
{
    constexpr int H = 3;
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<double, H, 6> *>(smraw);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);
    const double iak = ia[kw];
    double az[H], bz[H];
#pragma unroll
    for (int l = 0; l < H; l++) {
        az[l] = co.a[2][l] * iak;
        bz[l] = co.b[2][l] * iak * iak;
    }
    const double bsum = co.b2[0] + co.b2[1] + co.b2[2] * iak * iak;
    const double gs = (S == 4) ? 1.0 / 6.0 : 1.0;
    auto ld = [&](int c, long long o) -> double {
        return c < 3 ? a.Y[(long long)c * g.N3 + o] : a.G[(long long)(c - 3) * g.N3 + o] * gs;
    };
    const Walls<double> wl{};
    tile_march<double, H, 6, false>(g, wl, sm, ld, ib, ie, [&](long long idx, auto &q, const auto &vx, const auto &vy,
                                                          const auto &vz) {
        const double p0[3] = {q[H][0], q[H][1], q[H][2]};
        const double g0[3] = {q[H][3], q[H][4], q[H][5]};
        double At[3] = {0, 0, 0}, Bt[3] = {0, 0, 0}, lap[3] = {0, 0, 0}, divP = 0.0, divg = 0.0;
        auto dir = [&](const auto &v, int d, const double *aa, const double *bb) {
            double dP[3], dG[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                dP[c] = d1<double, H>(v, c, aa);
                dG[c] = d1<double, H>(v, 3 + c, aa);
                Bt[c] -= adv1<double, H>(v, 3 + c, d, p0[d], aa);
                if (KIND == KIND_BB) lap[c] += lsum<double, H>(v, 3 + c, bb);
            }
            divP += dP[d];
            divg += dG[d];
            auto sdot = [&](int, int s) -> double {
                return v(0, s) * v(3, s) + v(1, s) * v(4, s) + v(2, s) * v(5, s);
            };
            At[d] = -(p0[0] * dG[0] + p0[1] * dG[1] + p0[2] * dG[2]) + (g0[0] * dP[0] + g0[1] * dP[1] + g0[2] * dP[2])
                    - d1<double, H>(sdot, 0, aa);
        };
        dir(vx, 0, co.a[0], co.b[0]);
        dir(vy, 1, co.a[1], co.b[1]);
        dir(vz, 2, az, bz);
#pragma unroll
        for (int e = 0; e < 3; e++) {
            const double TF = 0.5 * fma(g0[e], divP, Bt[e]), TV = 0.5 * At[e];
            const long long o = (long long)e * g.N3 + idx;
            if constexpr (KIND == KIND_UB) {
                acc[o] += dt * (TF + TV + p0[e] * divg);
            } else if constexpr (KIND == KIND_BU) {
                acc[o] += dt * (TF - TV);
            } else {
                const double xi = dt * (-TF + TV + visc * fma(-bsum, g0[e], lap[e]));
                const double mu = a.mu[o];
                if constexpr (S == 4) {
                    a.Gout[o] = mu * (1.0 / 3.0) + xi;
                    a.LamOut[o] = xi;
                } else if constexpr (S == 3) {
                    a.Gout[o] = mu * (1.0 / 3.0) + 0.5 * xi;
                    a.LamOut[o] = a.Lam[o] + xi;
                } else if constexpr (S == 2) {
                    a.Gout[o] = mu * (1.0 / 6.0) + 0.5 * xi;
                    a.LamOut[o] = a.Lam[o] + xi;
                } else {
                    a.Gout[o] = mu + (a.Lam[o] + xi);
                }
            }
        }
    });
}

template <int KIND, int S>
void launch_mhd_s(const Geo &g, const Coef<double> &co, const double *ia, double dt, double visc, const AdjArgs &a,
                  double *acc, cudaStream_t st)
{
    constexpr size_t smem = tile_smem_bytes<double, 3, 6>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_adj_mhd<KIND, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int ch = pick_ichunk(g, 1);
    k_adj_mhd<KIND, S><<<tile_grid(g, ch), dim3(kTK, kTJ), smem, st>>>(g, co, ia, dt, visc, a, acc, ch);
}

template <int KIND>
void launch_mhd_k(int s, const Geo &g, const Coef<double> &co, const double *ia, double dt, double visc,
                  const AdjArgs &a, double *acc, cudaStream_t st)
{
    switch (s) {
    case 4: launch_mhd_s<KIND, 4>(g, co, ia, dt, visc, a, acc, st); break;
    case 3: launch_mhd_s<KIND, 3>(g, co, ia, dt, visc, a, acc, st); break;
    case 2: launch_mhd_s<KIND, 2>(g, co, ia, dt, visc, a, acc, st); break;
    default: launch_mhd_s<KIND, 1>(g, co, ia, dt, visc, a, acc, st); break;
    }
}

__global__ void k_axpby(long long n, double a, const double *__restrict__ x, double *__restrict__ y)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) y[t] = a * x[t];
}

__global__ void k_axpy(long long n, double a, const double *__restrict__ x, double *__restrict__ y)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n) y[t] = fma(a, x[t], y[t]);
}

}  // namespace

void launch_axpy(long long n, double a, const double *x, double *y, cudaStream_t st)
{
    k_axpy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, a, x, y);
}

cudaError_t launch_adj_stage64(int s, const Geo &g, const Coef<double> &co, const double *ia, double dt, double nu,
                               const AdjArgs &a, cudaStream_t st, int *err)
{
    if (err && adj_tma_fits(g)) return launch_adj_tma64(ADJ_NS, s, g, co, ia, dt, nu, a, nullptr, err, st);
    launch_adj<double>(s, g, co, ia, dt, nu, a, st);
    return cudaSuccess;
}

void launch_adj_stage32(int s, const Geo &g, const Coef<float> &co, const float *ia, float dt, float nu,
                        const AdjArgs32 &a, cudaStream_t st)
{
    launch_adj<float>(s, g, co, ia, dt, nu, a, st);
}

cudaError_t launch_adj_mhd(int kind, int s, const Geo &g, const Coef<double> &co, const double *ia, double dt,
                           double visc, const AdjArgs &a, double *acc, cudaStream_t st, int *err)
{
    if (err && adj_tma_fits(g)) return launch_adj_tma64(kind, s, g, co, ia, dt, visc, a, acc, err, st);
    if (kind == 0)
        launch_mhd_k<KIND_UB>(s, g, co, ia, dt, visc, a, acc, st);
    else if (kind == 1)
        launch_mhd_k<KIND_BU>(s, g, co, ia, dt, visc, a, acc, st);
    else
        launch_mhd_k<KIND_BB>(s, g, co, ia, dt, visc, a, acc, st);
    return cudaSuccess;
}

void launch_scale_copy(long long n, double a, const double *x, double *y, cudaStream_t st)
{
    k_axpby<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, a, x, y);
}

}  // namespace nova
