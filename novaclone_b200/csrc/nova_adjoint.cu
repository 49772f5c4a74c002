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
    // the pointwise operands (mu, lambda) of the next plane load while this plane computes
    double mun[3] = {0, 0, 0}, mu[3];
    T lamn[3] = {0, 0, 0}, lam[3];
    auto pre = [&](long long nidx, bool load) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            mu[c] = mun[c];
            lam[c] = lamn[c];
            if (load) {
                mun[c] = a.mu[(long long)c * g.N3 + nidx];
                if (S != 4) lamn[c] = a.Lam[(long long)c * g.N3 + nidx];
            }
        }
    };
    tile_march<T, H, 6, false>(g, wl, sm, ld, ib, ie, pre, [&](long long idx, auto &q, const auto &vx,
                                                       const auto &vy, const auto &vz) {
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
// MHD right-hand sides (app/OT_Poisson/UEqn.H:16-23, BEqn.H:72-78):
//   F_U = -div(U,U) + nu L U + div(B,B) - grad(1/2 |B|^2)   (B frozen in the U loop)
//   F_B = -div(U,B) + div(B,U) + eta L B                    (U frozen in the B loop)
// The coupling transposes, from the building blocks of nova_adj_math.cuh for
// the field P in comps 0-2 and the stage direction g_S in comps 3-5
// ((d grad(1/2|B|^2)/dB)^T g = -B div g):
//   ADJ_UB: acc += dt [ 1/2 g divP - Sx + 1/2 At + P divG ]   P = B^n        (dF_U/dB into lambda_B)
//   ADJ_BU: acc += dt [ 1/2 g divP - Sx - 1/2 At ]            P = Z_S        (dF_B/dU into lambda_U)
//   ADJ_BB: xi   = dt [ Sx + 1/2 At - 1/2 g divP - eta bsum g ] P = U^{n+1}  (dF_B/dB, with the recursion)
// (Sx with the Laplacian weight eta for BB only).  Tiled march; T = float with
// A = AdjArgs32 for the FP32-split adjoint (acc and mu stay FP64).  At s = 4
// the direction is mu/6, read from a.mu.
template <typename T, int KIND, int S, class A>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 8 ? 1 : 2)
    k_adj_mhd(Geo g, Coef<T> co, const T *__restrict__ ia, T dt, T visc, A a, double *acc, int ichunk)
{
    constexpr int H = 3;
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &sm = *reinterpret_cast<TileSmem<T, H, 6> *>(smraw);
    const int ib = blockIdx.z * ichunk;
    const int ie = min(ib + ichunk, g.N0);
    const int kw = wrapi(blockIdx.x * kTK + threadIdx.x, g.N2);
    T az[H], bz[H], bsum;
    adj_zweights<T, H>(co, ia[kw], az, bz, bsum);
    auto ld = [&](int c, long long o) -> T {
        if (c < 3) return a.Y[(long long)c * g.N3 + o];
        if constexpr (S == 4) return (T)(a.mu[(long long)(c - 3) * g.N3 + o] * (1.0 / 6.0));
        return a.G[(long long)(c - 3) * g.N3 + o];
    };
    const Walls<T> wl{};
    // the pointwise operands of the next plane load while this plane computes:
    // BB mu and lambda, UB and BU the FP64 accumulator they add to
    double pn[3] = {0, 0, 0}, pc[3];
    T lamn[3] = {0, 0, 0}, lamc[3];
    auto pre = [&](long long nidx, bool load) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            pc[c] = pn[c];
            lamc[c] = lamn[c];
            if (load) {
                const long long o = (long long)c * g.N3 + nidx;
                pn[c] = KIND == ADJ_BB ? a.mu[o] : acc[o];
                if (KIND == ADJ_BB && S != 4) lamn[c] = a.Lam[o];
            }
        }
    };
    tile_march<T, H, 6, false>(g, wl, sm, ld, ib, ie, pre, [&](long long idx, auto &q, const auto &vx,
                                                       const auto &vy, const auto &vz) {
        const T p0[3] = {q[H][0], q[H][1], q[H][2]};
        const T g0[3] = {q[H][3], q[H][4], q[H][5]};
        T Sx[3], At[3], divP, divG;
        adj_terms<T, H, KIND == ADJ_UB>(vx, vy, vz, p0, g0, co, az, bz, KIND == ADJ_BB ? visc : T(0), Sx, At, divP,
                                        divG);
#pragma unroll
        for (int e = 0; e < 3; e++) {
            const long long o = (long long)e * g.N3 + idx;
            if constexpr (KIND == ADJ_BB) {
                const T xi = dt * (Sx[e] + T(0.5) * fma(-g0[e], divP, At[e]) - visc * bsum * g0[e]);
                adj_store<T, S>(a, o, pc[e], S == 4 ? T(0) : lamc[e], xi);
            } else if constexpr (KIND == ADJ_UB) {
                acc[o] = pc[e] + (double)(dt * (fma(T(0.5) * g0[e], divP, -Sx[e]) + fma(T(0.5), At[e], p0[e] * divG)));
            } else {
                acc[o] = pc[e] + (double)(dt * (fma(T(0.5) * g0[e], divP, -Sx[e]) - T(0.5) * At[e]));
            }
        }
    });
}

template <typename T, int KIND, int S, class A>
void launch_mhd_s(const Geo &g, const Coef<T> &co, const T *ia, T dt, T visc, const A &a, double *acc, cudaStream_t st)
{
    constexpr size_t smem = tile_smem_bytes<T, 3, 6>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_adj_mhd<T, KIND, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int ch = pick_ichunk(g, sizeof(T) == 8 ? 1 : 2);
    k_adj_mhd<T, KIND, S, A><<<tile_grid(g, ch), dim3(kTK, kTJ), smem, st>>>(g, co, ia, dt, visc, a, acc, ch);
}

template <typename T, int KIND, class A>
void launch_mhd_k(int s, const Geo &g, const Coef<T> &co, const T *ia, T dt, T visc, const A &a, double *acc,
                  cudaStream_t st)
{
    switch (s) {
    case 4: launch_mhd_s<T, KIND, 4>(g, co, ia, dt, visc, a, acc, st); break;
    case 3: launch_mhd_s<T, KIND, 3>(g, co, ia, dt, visc, a, acc, st); break;
    case 2: launch_mhd_s<T, KIND, 2>(g, co, ia, dt, visc, a, acc, st); break;
    default: launch_mhd_s<T, KIND, 1>(g, co, ia, dt, visc, a, acc, st); break;
    }
}

template <typename T, class A>
void launch_mhd_any(int kind, int s, const Geo &g, const Coef<T> &co, const T *ia, T dt, T visc, const A &a,
                    double *acc, cudaStream_t st)
{
    if (kind == ADJ_UB)
        launch_mhd_k<T, ADJ_UB>(s, g, co, ia, dt, visc, a, acc, st);
    else if (kind == ADJ_BU)
        launch_mhd_k<T, ADJ_BU>(s, g, co, ia, dt, visc, a, acc, st);
    else
        launch_mhd_k<T, ADJ_BB>(s, g, co, ia, dt, visc, a, acc, st);
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
    launch_mhd_any<double>(kind, s, g, co, ia, dt, visc, a, acc, st);
    return cudaSuccess;
}

void launch_adj_mhd32(int kind, int s, const Geo &g, const Coef<float> &co, const float *ia, float dt, float visc,
                      const AdjArgs32 &a, double *acc, cudaStream_t st)
{
    launch_mhd_any<float>(kind, s, g, co, ia, dt, visc, a, acc, st);
}

void launch_scale_copy(long long n, double a, const double *x, double *y, cudaStream_t st)
{
    k_axpby<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, a, x, y);
}

namespace {

__global__ void k_dot_part(long long n, const double *__restrict__ x, const double *__restrict__ y,
                           double *__restrict__ part)
{
    __shared__ double sh[32];
    double a = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        a = fma(x[t], y[t], a);
    a = block_reduce_sum(a, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
}

__global__ void k_sum_final(const double *__restrict__ part, int nb, double scale, double *__restrict__ out)
{
    __shared__ double sh[32];
    double a = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) a += part[q];
    a = block_reduce_sum(a, sh);
    if (threadIdx.x == 0) *out = a * scale;
}

}  // namespace

void launch_dot(long long n, const double *x, const double *y, double scale, double *part, int nb, double *out,
                cudaStream_t st)
{
    k_dot_part<<<nb, 256, 0, st>>>(n, x, y, part);
    k_sum_final<<<1, 256, 0, st>>>(part, nb, scale, out);
}

}  // namespace nova
