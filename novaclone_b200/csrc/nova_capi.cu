// C ABI of libnova_b200 (include/nova_gpu.h): contexts, fields, the ex::
// drop-in operators, the cuFFT projection and the fused time advance.
#include "nova_gpu.h"
#include "nova_internal.cuh"
#include "nova_mesh.cuh"
#include "nova_ops.cuh"
#include "nova_wc.cuh"

#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace nova;

struct nova_field {
    int nc;
    int prec;
    long long n3;
    double *d64;
    float *hi, *lo;
    nova_bc bc;  // setBC of the reference field: index face + 6*comp
};

namespace {

// settings::coef_ (src/settings/settings.cpp:25-31)
const double kCoef[4][4] = {
    {1.0, 0.0, 0.0, 0.0},
    {4.0 / 3.0, -1.0 / 3.0, 0.0, 0.0},
    {6.0 / 4.0, -12.0 / 20.0, 1.0 / 10.0, 0.0},
    {8.0 / 5.0, -4.0 / 5.0, 24.0 / 105.0, -8.0 / 280.0},
};

struct ProfRec {
    int cls;
    cudaEvent_t a, b;
};

}  // namespace

struct nova_ctx {
    nova_mesh_desc md{};
    int h = 3;
    int local_n[3] = {0, 0, 0};
    Geo g{};
    Coef<double> co64{};
    Coef<float> co32{};
    std::vector<double> dzdxi, d2zdxi2;  // ghosted length n2 (Mesh::dzdxi_)
    double *d_ia64 = nullptr, *d_corr64 = nullptr;
    float *d_ia32 = nullptr, *d_corr32 = nullptr;
    double *d_kx2 = nullptr, *d_ky2 = nullptr, *d_kz2 = nullptr;
    cufftHandle plan_f = 0, plan_b = 0;
    bool plans = false;
    // periodic meshes with N0 = 64 or 256: plan_f/plan_b are batched 2-D (j, k)
    // transforms and the i direction runs fused with the scale (k_pois_i)
    bool pois_i = false;
    double *d_twN = nullptr;  // W_N0^m, m = 0..N0-1 (re, im)
    // N1 = N2 = 256 as well and NOVA_FFT=cluster: the (j, k) planes by the
    // one-pass cluster kernels (nova_fft2d.cu) instead of the cuFFT plans
    bool fft2 = false;
    bool fft_cluster = false;
    bool pois_direct = false;  // NOVA_POIS_I=direct: k_pois_i also where k_pois_tma fits
    bool fft_ready = false;
    double *d_tw256 = nullptr;
    cufftHandle dct_f = 0, dct_b = 0;  // wall Poisson on the even extension in y
    bool dct_plans = false;
    double *d_ext = nullptr, *d_ky2e = nullptr;
    void *d_spec2 = nullptr;
    // wall Poisson with N[1] = 256: batched 2-D (i, k) transforms of the stored
    // rows and k_pois_dct (DCT-I along y); NOVA_DCT=extend keeps the even extension
    cufftHandle dct2_f = 0, dct2_b = 0;
    bool dct2_plans = false;
    bool dct_extend = false;
    void *d_spec3 = nullptr;
    double *d_t512 = nullptr;
    void *d_spec = nullptr;
    double *d_rhs = nullptr;
    double *w64[3] = {nullptr, nullptr, nullptr};
    float *w32[3] = {nullptr, nullptr, nullptr};
    double *d_part = nullptr;
    double *d_scalar = nullptr;
    int *d_flag = nullptr;
    double *d_hist = nullptr;
    long long hist_cap = 0;
    double *d_stage = nullptr;
    size_t stage_cap = 0;
    double *adj_pool = nullptr;  // adjoint checkpoints, segment states, adjoint fields
    size_t adj_cap = 0;
    double *d_row = nullptr;     // two diagnostics rows (adjoint objectives)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    bool prof = false;
    std::vector<ProfRec> prof_live;
    std::vector<cudaEvent_t> ev_pool;
    double prof_ms[NOVA_K_COUNT] = {0};
    long prof_n[NOVA_K_COUNT] = {0};
    long launches = 0;
    int stage_impl = STAGE_AUTO;  // NOVA_STAGE_IMPL=march|tma at nova_create
};

namespace {

// default BCs: periodic faces; Neumann 0 on wall faces
void default_bc(const nova_ctx *ctx, nova_bc *bc)
{
    for (int q = 0; q < 18; q++) {
        const int face = q % 6;
        const bool ywall = ctx->g.wallY && (face == NOVA_NORTH || face == NOVA_SOUTH);
        bc->type[q] = ywall ? NOVA_BC_NEUMANN : NOVA_BC_PERIODIC;
        bc->val[q] = 0.0;
    }
}

// ghosts of a field's components beyond the y walls (Walls<T>, nova_internal.cuh)
template <typename T>
void add_walls(const nova_ctx *ctx, const nova_field *f, Walls<T> &w, int c0)
{
    if (!ctx->g.wallY || !f) return;
    w.on = 1;
    w.dy = (T)(ctx->md.L[1] / ctx->md.N[1]);
    for (int c = 0; c < f->nc && c0 + c < 9; c++) {
        for (int side = 0; side < 2; side++) {
            const int q = (side == 0 ? NOVA_SOUTH : NOVA_NORTH) + 6 * (c < 3 ? c : 0);
            w.dir[side][c0 + c] = f->bc.type[q] == NOVA_BC_DIRICHLET ? 1 : 0;
            w.val[side][c0 + c] = (T)f->bc.val[q];
        }
    }
}

template <typename T> Walls<T> walls_of(const nova_ctx *ctx, const nova_field *a, const nova_field *b = nullptr)
{
    Walls<T> w{};
    add_walls<T>(ctx, a, w, 0);
    add_walls<T>(ctx, b, w, 3);
    return w;
}

// the reference's wall-node overwrite for a field (k_wall_fix)
WallFix wall_fix_of(const nova_ctx *ctx, const nova_field *f)
{
    WallFix wf{};
    if (!ctx->g.wallY) return wf;
    wf.on = 1;
    wf.nc = f->nc;
    wf.dy = ctx->md.L[1] / ctx->md.N[1];
    for (int c = 0; c < f->nc && c < 9; c++)
        for (int side = 0; side < 2; side++) {
            const int q = (side == 0 ? NOVA_SOUTH : NOVA_NORTH) + 6 * (c < 3 ? c : 0);
            wf.type[side][c] = f->bc.type[q];
            wf.val[side][c] = f->bc.val[q];
        }
    return wf;
}

nova_status fail(nova_ctx *c, nova_status s, const std::string &msg)
{
    if (c) c->err = msg;
    return s;
}

nova_status cuda_check(nova_ctx *c, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return NOVA_OK;
    if (e == cudaErrorMemoryAllocation) return fail(c, NOVA_E_OOM, std::string(what) + ": out of device memory");
    return fail(c, NOVA_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                        \
    do {                                                                \
        nova_status _s = cuda_check(ctx, (call), #call);                \
        if (_s != NOVA_OK) return _s;                                   \
    } while (0)

#define CKL(what)                                                       \
    do {                                                                \
        nova_status _s = cuda_check(ctx, cudaGetLastError(), what);     \
        if (_s != NOVA_OK) return _s;                                   \
    } while (0)

nova_status fft_check(nova_ctx *ctx, cufftResult r, const char *what)
{
    if (r == CUFFT_SUCCESS) return NOVA_OK;
    if (r == CUFFT_ALLOC_FAILED) return fail(ctx, NOVA_E_OOM, std::string(what) + ": cuFFT allocation failed");
    return fail(ctx, NOVA_E_CUDA, std::string(what) + ": cuFFT error " + std::to_string((int)r));
}

template <typename T>
nova_status dalloc(nova_ctx *ctx, T **p, size_t n)
{
    if (*p) return NOVA_OK;
    return cuda_check(ctx, cudaMalloc((void **)p, sizeof(T) * (n ? n : 1)), "cudaMalloc");
}

// Mesh::dzdxi_, d2zdxi2_ (src/Mesh/Mesh.cpp:146-179)
void mesh_metrics(const nova_mesh_desc &m, std::vector<double> &dz1, std::vector<double> &dz2)
{
    const int h = m.m / 2;
    const int nk = m.N[2] + 1 + m.m;
    const double *c = kCoef[(m.m - 2) / 2];
    const double dz = m.L[2] / m.N[2];
    const double b = mesh_hyp_b(m);
    dz1.assign(nk, 0.0);
    dz2.assign(nk, 0.0);
    for (int k = h; k < nk - h; k++) {
        double s = 0.0, s2 = 0.0;
        for (int l = 0; l < h; l++) {
            s += (c[l] / 2.0 / (l + 1) / dz * mesh_z(m, h, b, k + 1 + l)
                  - c[l] / 2.0 / (l + 1) / dz * mesh_z(m, h, b, k - 1 - l));
            s2 += (c[l] / std::pow((l + 1) * dz, 2) * mesh_z(m, h, b, k + 1 + l)
                   + c[l] / std::pow((l + 1) * dz, 2) * mesh_z(m, h, b, k - 1 - l)
                   + (-2.0 * c[l] / std::pow((l + 1) * dz, 2)) * mesh_z(m, h, b, k));
        }
        dz1[k] = s;
        dz2[k] = s2;
    }
}

// squared modified wavenumbers along one axis (poisson::wavenumbersFFT_, poisson.cpp:352-391)
std::vector<double> kp2_table(int n, double L, double delta, int h, const double *coef, bool fold, int count)
{
    std::vector<double> t(count);
    const double pi = M_PI, eps = 1.0e-16;
    for (int i = 0; i < count; i++) {
        double kk;
        if (!fold || 2 * i < n)
            kk = 2.0 * pi * (i) / L;
        else
            kk = 2.0 * pi * (n - i) / L;
        double kp = 0.0;
        if (kk > eps)
            for (int ll = 0; ll < h; ll++) kp += kk * coef[ll] / (ll + 1) * std::sin((ll + 1) * kk * delta) / (kk * delta);
        t[i] = kp * kp;
    }
    return t;
}

void prof_begin(nova_ctx *ctx, int cls, cudaEvent_t *a)
{
    *a = nullptr;
    if (!ctx->prof) return;
    if (ctx->ev_pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->ev_pool.push_back(e);
    }
    *a = ctx->ev_pool.back();
    ctx->ev_pool.pop_back();
    cudaEventRecord(*a, ctx->stream);
    (void)cls;
}

void prof_end(nova_ctx *ctx, int cls, cudaEvent_t a)
{
    if (!ctx->prof || !a) return;
    if (ctx->ev_pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->ev_pool.push_back(e);
    }
    cudaEvent_t b = ctx->ev_pool.back();
    ctx->ev_pool.pop_back();
    cudaEventRecord(b, ctx->stream);
    ctx->prof_live.push_back({cls, a, b});
}

void prof_collect(nova_ctx *ctx)
{
    if (ctx->prof_live.empty()) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto &r : ctx->prof_live) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        ctx->prof_ms[r.cls] += ms;
        ctx->prof_n[r.cls] += 1;
        ctx->ev_pool.push_back(r.a);
        ctx->ev_pool.push_back(r.b);
    }
    ctx->prof_live.clear();
}

struct ProfScope {
    nova_ctx *ctx;
    int cls;
    cudaEvent_t a;
    ProfScope(nova_ctx *c, int k) : ctx(c), cls(k) { prof_begin(ctx, cls, &a); }
    ~ProfScope() { prof_end(ctx, cls, a); }
};

// W_N^m = exp(-2 pi i m / N), m = 0..N-1, rounded from extended precision
std::vector<double> twiddles(int N)
{
    std::vector<double> tw(2 * (size_t)N);
    const long double pi_l = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < N; m++) {
        const long double a = 2.0L * pi_l * (long double)m / (long double)N;
        tw[2 * m] = (double)cosl(a);
        tw[2 * m + 1] = (double)-sinl(a);
    }
    return tw;
}

nova_status ensure_fft(nova_ctx *ctx)
{
    if (ctx->fft_ready) return NOVA_OK;
    const Geo &g = ctx->g;
    nova_status s;
    if (pois_i_fits(g) && ctx->fft_cluster && fft2_fits(g)) {
        // the (j, k) planes by the cluster kernels, the i direction by k_pois_i
        std::vector<double> tw = twiddles(g.N0), t256 = twiddles(256);
        if ((s = dalloc(ctx, &ctx->d_twN, tw.size())) != NOVA_OK) return s;
        CK(cudaMemcpy(ctx->d_twN, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice));
        if ((s = dalloc(ctx, &ctx->d_tw256, t256.size())) != NOVA_OK) return s;
        CK(cudaMemcpy(ctx->d_tw256, t256.data(), sizeof(double) * t256.size(), cudaMemcpyHostToDevice));
        ctx->pois_i = true;
        ctx->fft2 = true;
        const size_t nspec = (size_t)g.N0 * g.N1 * (g.N2 / 2 + 1);
        if ((s = dalloc(ctx, (double **)&ctx->d_spec, 2 * nspec)) != NOVA_OK) return s;
        if ((s = dalloc(ctx, &ctx->d_rhs, (size_t)g.N3)) != NOVA_OK) return s;
        ctx->fft_ready = true;
        return NOVA_OK;
    }
    // the transform runs over the N[1] unique y nodes of poisson::rhs (poisson.cpp:167-181),
    // which with walls are the first N[1] of the N[1]+1 stored rows
    const int ny = ctx->md.N[1];
    const bool pi = pois_i_fits(g);
    if (pi) {
        std::vector<double> tw = twiddles(g.N0);
        if ((s = dalloc(ctx, &ctx->d_twN, tw.size())) != NOVA_OK) return s;
        CK(cudaMemcpy(ctx->d_twN, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice));
    }
    // 3-D transform, or for k_pois_i the (j, k) planes batched over i; both
    // give the half spectrum [i][j][kz]
    const int rank = pi ? 2 : 3, batch = pi ? g.N0 : 1;
    int n3d[3] = {g.N0, ny, g.N2}, n2d[2] = {ny, g.N2};
    int rembed3[3] = {g.N0, g.N1, g.N2}, rembed2[2] = {g.N1, g.N2};
    int cembed3[3] = {g.N0, ny, g.N2 / 2 + 1}, cembed2[2] = {ny, g.N2 / 2 + 1};
    int *n = pi ? n2d : n3d, *rembed = pi ? rembed2 : rembed3, *cembed = pi ? cembed2 : cembed3;
    const int rdist = (pi ? 1 : g.N0) * g.N1 * g.N2, cdist = (pi ? 1 : g.N0) * ny * (g.N2 / 2 + 1);
    if ((s = fft_check(ctx, cufftPlanMany(&ctx->plan_f, rank, n, rembed, 1, rdist, cembed, 1, cdist, CUFFT_D2Z, batch),
                       "cufftPlanMany D2Z")) != NOVA_OK)
        return s;
    if ((s = fft_check(ctx, cufftPlanMany(&ctx->plan_b, rank, n, cembed, 1, cdist, rembed, 1, rdist, CUFFT_Z2D, batch),
                       "cufftPlanMany Z2D")) != NOVA_OK) {
        cufftDestroy(ctx->plan_f);
        return s;
    }
    ctx->plans = true;
    ctx->pois_i = pi;
    const size_t nspec = (size_t)g.N0 * ny * (g.N2 / 2 + 1);
    if ((s = dalloc(ctx, (double **)&ctx->d_spec, 2 * nspec)) != NOVA_OK) return s;
    if ((s = dalloc(ctx, &ctx->d_rhs, (size_t)g.N3)) != NOVA_OK) return s;
    ctx->fft_ready = true;
    return NOVA_OK;
}

nova_status ensure_red(nova_ctx *ctx)
{
    nova_status s;
    if ((s = dalloc(ctx, &ctx->d_part, (size_t)diag_blocks(ctx->g) * kDiagParts)) != NOVA_OK) return s;
    if ((s = dalloc(ctx, &ctx->d_scalar, 1)) != NOVA_OK) return s;
    // [0] non-finite diagnostics, [1] a stage pipeline wait timed out
    if ((s = dalloc(ctx, &ctx->d_flag, 2)) != NOVA_OK) return s;
    return NOVA_OK;
}

nova_status stage_fail(nova_ctx *ctx, cudaError_t e)
{
    if (e == cudaErrorNotSupported)
        return fail(ctx, NOVA_E_UNSUPPORTED,
                    "NOVA_STAGE_IMPL=tma: the TMA stage kernel needs N2 % 32 == 0 and N1 at least twice the tile height (16 rows FP64, 8 FP32), with periodic y a multiple of it; walls in y only in FP32");
    if (e == cudaErrorInvalidValue) return fail(ctx, NOVA_E_CUDA, "stage kernel: cuTensorMapEncodeTiled failed");
    return cuda_check(ctx, e, "stage kernel");
}

// rhs (device, N3 doubles) -> p: spectral inverse of div(grad(.)) (poisson::solve)
nova_status poisson_device(nova_ctx *ctx, const double *rhs, double *p)
{
    nova_status s;
    if ((s = ensure_fft(ctx)) != NOVA_OK) return s;
    if ((s = ensure_red(ctx)) != NOVA_OK) return s;  // the error word of k_pois_tma
    ProfScope ps(ctx, NOVA_K_FFT);
    const long long nuniq = (long long)ctx->g.N0 * ctx->md.N[1] * ctx->g.N2;
    if (ctx->fft2) {
        launch_fft2_fwd(ctx->g, rhs, ctx->d_spec, ctx->d_tw256, ctx->stream);
        launch_pois_i(ctx->g, ctx->md.N[1], ctx->d_spec, ctx->d_twN, ctx->d_kx2, ctx->d_ky2, ctx->d_kz2,
                      1.0 / (double)nuniq, ctx->pois_direct ? nullptr : ctx->d_flag + 1, ctx->stream);
        launch_fft2_inv(ctx->g, ctx->d_spec, p, ctx->d_tw256, ctx->stream);
        ctx->launches += 3;
        CKL("cluster FFT / k_pois_i");
        return NOVA_OK;
    }
    cufftSetStream(ctx->plan_f, ctx->stream);
    cufftSetStream(ctx->plan_b, ctx->stream);
    if ((s = fft_check(ctx, cufftExecD2Z(ctx->plan_f, (cufftDoubleReal *)rhs, (cufftDoubleComplex *)ctx->d_spec),
                       "cufftExecD2Z")) != NOVA_OK)
        return s;
    if (ctx->pois_i) {
        launch_pois_i(ctx->g, ctx->md.N[1], ctx->d_spec, ctx->d_twN, ctx->d_kx2, ctx->d_ky2, ctx->d_kz2,
                      1.0 / (double)nuniq, ctx->pois_direct ? nullptr : ctx->d_flag + 1, ctx->stream);
        ctx->launches += 1;
        CKL("k_pois_i");
    } else {
        launch_scale(ctx->g, ctx->md.N[1], ctx->d_spec, ctx->d_kx2, ctx->d_ky2, ctx->d_kz2, 1.0 / (double)nuniq,
                     ctx->stream);
        ctx->launches += 1;
        CKL("k_scale");
    }
    if ((s = fft_check(ctx, cufftExecZ2D(ctx->plan_b, (cufftDoubleComplex *)ctx->d_spec, (cufftDoubleReal *)p),
                       "cufftExecZ2D")) != NOVA_OK)
        return s;
    return NOVA_OK;
}

// the y modified wavenumbers of the wall solve: period 2 L_y on 2 N[1] points
// (the even extension's), folded
std::vector<double> ky2_walls(const nova_ctx *ctx)
{
    const int ny = ctx->md.N[1];
    const double *c = kCoef[(ctx->md.m - 2) / 2];
    return kp2_table(2 * ny, 2.0 * ctx->md.L[1], ctx->md.L[1] / ny, ctx->h, c, true, 2 * ny);
}

// the wall Poisson with DCT-I along y on the N[1] + 1 stored rows (N[1] = 256):
// batched 2-D D2Z over (i, k), k_pois_dct (DCT-I, scale, DCT-I), 2-D Z2D
nova_status poisson_device_dct1(nova_ctx *ctx, const double *rhs, double *p)
{
    const Geo &g = ctx->g;
    const int ny = ctx->md.N[1], nzh = g.N2 / 2 + 1;
    nova_status s;
    if (!ctx->dct2_plans) {
        // element (i, j, k) of a batch-j plane at j N2 + i N1 N2 + k; spectrum at (i N1 + j) nzh + kz
        int n[2] = {g.N0, g.N2}, rin[2] = {g.N0, (int)g.N12}, cin[2] = {g.N0, g.N1 * nzh};
        if ((s = fft_check(ctx, cufftPlanMany(&ctx->dct2_f, 2, n, rin, 1, g.N2, cin, 1, nzh, CUFFT_D2Z, g.N1),
                           "cufftPlanMany D2Z (walls, DCT)")) != NOVA_OK)
            return s;
        if ((s = fft_check(ctx, cufftPlanMany(&ctx->dct2_b, 2, n, cin, 1, nzh, rin, 1, g.N2, CUFFT_Z2D, g.N1),
                           "cufftPlanMany Z2D (walls, DCT)")) != NOVA_OK) {
            cufftDestroy(ctx->dct2_f);
            return s;
        }
        ctx->dct2_plans = true;
        if ((s = dalloc(ctx, (double **)&ctx->d_spec3, 2 * (size_t)g.N0 * g.N1 * nzh)) != NOVA_OK) return s;
        const std::vector<double> t256 = twiddles(256), t512 = twiddles(512), ky2e = ky2_walls(ctx);
        if (!ctx->d_tw256) {
            if ((s = dalloc(ctx, &ctx->d_tw256, t256.size())) != NOVA_OK) return s;
            CK(cudaMemcpy(ctx->d_tw256, t256.data(), sizeof(double) * t256.size(), cudaMemcpyHostToDevice));
        }
        if ((s = dalloc(ctx, &ctx->d_t512, 512)) != NOVA_OK) return s;  // W_512^n, n < 256
        CK(cudaMemcpy(ctx->d_t512, t512.data(), sizeof(double) * 512, cudaMemcpyHostToDevice));
        if (!ctx->d_ky2e) {
            if ((s = dalloc(ctx, &ctx->d_ky2e, ky2e.size())) != NOVA_OK) return s;
            CK(cudaMemcpy(ctx->d_ky2e, ky2e.data(), sizeof(double) * ky2e.size(), cudaMemcpyHostToDevice));
        }
    }
    ProfScope ps(ctx, NOVA_K_FFT);
    cufftSetStream(ctx->dct2_f, ctx->stream);
    cufftSetStream(ctx->dct2_b, ctx->stream);
    if ((s = fft_check(ctx, cufftExecD2Z(ctx->dct2_f, const_cast<double *>(rhs), (cufftDoubleComplex *)ctx->d_spec3),
                       "cufftExecD2Z")) != NOVA_OK)
        return s;
    launch_pois_dct(g, ctx->d_spec3, ctx->d_tw256, ctx->d_t512, ctx->d_kx2, ctx->d_ky2e, ctx->d_kz2,
                    1.0 / ((double)g.N0 * 2.0 * ny * g.N2), ctx->stream);
    if ((s = fft_check(ctx, cufftExecZ2D(ctx->dct2_b, (cufftDoubleComplex *)ctx->d_spec3, p), "cufftExecZ2D")) !=
        NOVA_OK)
        return s;
    ctx->launches += 1;
    CKL("wall poisson (DCT-I)");
    return NOVA_OK;
}

// the wall Poisson of NOVA_POISSON_DCT: even extension in y, periodic solve on
// the doubled domain (modified wavenumbers of period 2 L_y), restriction to
// the stored rows
nova_status poisson_device_dct(nova_ctx *ctx, const double *rhs, double *p)
{
    const Geo &g = ctx->g;
    const int ny = ctx->md.N[1];
    nova_status s;
    if (!ctx->dct_extend && pois_dct_fits(g, ny)) return poisson_device_dct1(ctx, rhs, p);
    if (!ctx->dct_plans) {
        if ((s = fft_check(ctx, cufftPlan3d(&ctx->dct_f, g.N0, 2 * ny, g.N2, CUFFT_D2Z), "cufftPlan3d D2Z (walls)")) !=
            NOVA_OK)
            return s;
        if ((s = fft_check(ctx, cufftPlan3d(&ctx->dct_b, g.N0, 2 * ny, g.N2, CUFFT_Z2D), "cufftPlan3d Z2D (walls)")) !=
            NOVA_OK) {
            cufftDestroy(ctx->dct_f);
            return s;
        }
        ctx->dct_plans = true;
        const size_t next = (size_t)g.N0 * 2 * ny * g.N2;
        if ((s = dalloc(ctx, &ctx->d_ext, next)) != NOVA_OK) return s;
        if ((s = dalloc(ctx, (double **)&ctx->d_spec2, 2 * (size_t)g.N0 * 2 * ny * (g.N2 / 2 + 1))) != NOVA_OK) return s;
        const std::vector<double> ky2e = ky2_walls(ctx);
        if ((s = dalloc(ctx, &ctx->d_ky2e, ky2e.size())) != NOVA_OK) return s;
        CK(cudaMemcpy(ctx->d_ky2e, ky2e.data(), sizeof(double) * ky2e.size(), cudaMemcpyHostToDevice));
    }
    ProfScope ps(ctx, NOVA_K_FFT);
    cufftSetStream(ctx->dct_f, ctx->stream);
    cufftSetStream(ctx->dct_b, ctx->stream);
    launch_even_extend(g, ny, rhs, ctx->d_ext, ctx->stream);
    if ((s = fft_check(ctx, cufftExecD2Z(ctx->dct_f, ctx->d_ext, (cufftDoubleComplex *)ctx->d_spec2), "cufftExecD2Z")) !=
        NOVA_OK)
        return s;
    launch_scale(g, 2 * ny, ctx->d_spec2, ctx->d_kx2, ctx->d_ky2e, ctx->d_kz2,
                 1.0 / ((double)g.N0 * 2.0 * ny * g.N2), ctx->stream);
    if ((s = fft_check(ctx, cufftExecZ2D(ctx->dct_b, (cufftDoubleComplex *)ctx->d_spec2, ctx->d_ext), "cufftExecZ2D")) !=
        NOVA_OK)
        return s;
    launch_restrict_rows(g, ny, ctx->d_ext, p, ctx->stream);
    ctx->launches += 3;
    CKL("wall poisson");
    return NOVA_OK;
}

// a field of this context's mesh: its buffers hold the context's N3 nodes per
// component (a field made by a context of another mesh would be read or
// written past its end)
bool on_mesh(const nova_ctx *ctx, const nova_field *f)
{
    return f && f->n3 == ctx->g.N3;
}

bool valid_field(const nova_ctx *ctx, const nova_field *f, int nc)
{
    return on_mesh(ctx, f) && f->nc == nc;
}

nova_status ensure_stage(nova_ctx *ctx, size_t n)
{
    if (ctx->stage_cap >= n) return NOVA_OK;
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    ctx->d_stage = nullptr;
    ctx->stage_cap = 0;
    nova_status s = dalloc(ctx, &ctx->d_stage, n);
    if (s == NOVA_OK) ctx->stage_cap = n;
    return s;
}

}  // namespace

// ================================================================== context ==
extern "C" nova_status nova_create(const nova_mesh_desc *md, nova_ctx **out)
{
    if (!md || !out) return NOVA_E_INVALID;
    *out = nullptr;
    if (md->m != 2 && md->m != 4 && md->m != 6 && md->m != 8) return NOVA_E_INVALID;
    for (int a = 0; a < 3; a++)
        if (md->N[a] < 1 || !(md->L[a] > 0.0) || (md->walls[a] != 0 && md->walls[a] != 1)) return NOVA_E_INVALID;
    if (md->walls[0] || md->walls[2]) return NOVA_E_UNSUPPORTED;  // walls in y only
    if (md->walls[1] && md->N[1] < md->m) return NOVA_E_INVALID;   // the mirrored halo needs m/2 nodes per wall
    nova_ctx *ctx = new (std::nothrow) nova_ctx();
    if (!ctx) return NOVA_E_OOM;
    ctx->md = *md;
    ctx->h = md->m / 2;
    if (const char *impl = std::getenv("NOVA_STAGE_IMPL")) {
        if (!std::strcmp(impl, "march")) ctx->stage_impl = STAGE_MARCH;
        if (!std::strcmp(impl, "tma")) ctx->stage_impl = STAGE_TMA;
    }
    if (const char *f = std::getenv("NOVA_FFT")) ctx->fft_cluster = !std::strcmp(f, "cluster");
    if (const char *f = std::getenv("NOVA_POIS_I")) ctx->pois_direct = !std::strcmp(f, "direct");
    if (const char *f = std::getenv("NOVA_DCT")) ctx->dct_extend = !std::strcmp(f, "extend");
    for (int a = 0; a < 3; a++) ctx->local_n[a] = md->N[a] + 1 + md->m;
    Geo &g = ctx->g;
    g.wallY = md->walls[1];
    g.N0 = md->N[0];
    g.N1 = md->N[1] + g.wallY;
    g.N2 = md->N[2];
    g.N12 = (long long)g.N1 * g.N2;
    g.N3 = (long long)g.N0 * g.N12;
    const double *c = kCoef[(md->m - 2) / 2];
    for (int d = 0; d < 3; d++) {
        const double del = md->L[d] / md->N[d];
        double b2 = 0.0;
        for (int l = 0; l < 4; l++) {
            const double a = (l < ctx->h) ? c[l] / 2.0 / (l + 1) / del : 0.0;
            const double b = (l < ctx->h) ? c[l] / std::pow((l + 1) * del, 2) : 0.0;
            ctx->co64.a[d][l] = a;
            ctx->co64.b[d][l] = b;
            ctx->co32.a[d][l] = (float)a;
            ctx->co32.b[d][l] = (float)b;
            b2 += 2.0 * b;
        }
        ctx->co64.b2[d] = b2;
        ctx->co32.b2[d] = (float)b2;
    }
    mesh_metrics(*md, ctx->dzdxi, ctx->d2zdxi2);
    std::vector<double> ia(g.N2), cr(g.N2);
    std::vector<float> ia32(g.N2), cr32(g.N2);
    for (int k = 0; k < g.N2; k++) {
        const double d1 = ctx->dzdxi[k + ctx->h], d2 = ctx->d2zdxi2[k + ctx->h];
        ia[k] = 1.0 / d1;
        cr[k] = d2 / (d1 * d1);
        ia32[k] = (float)ia[k];
        cr32[k] = (float)cr[k];
    }
    const double dx = md->L[0] / md->N[0], dy = md->L[1] / md->N[1], dz = md->L[2] / md->N[2];
    std::vector<double> kx2 = kp2_table(g.N0, md->L[0], dx, ctx->h, c, true, g.N0);
    std::vector<double> ky2 = kp2_table(md->N[1], md->L[1], dy, ctx->h, c, true, md->N[1]);
    std::vector<double> kz2 = kp2_table(g.N2, md->L[2], dz, ctx->h, c, false, g.N2 / 2 + 1);

    nova_status s = NOVA_OK;
    auto up = [&](auto **dptr, const auto &vec) {
        if (s != NOVA_OK) return;
        using T = typename std::remove_reference<decltype(vec)>::type::value_type;
        s = dalloc(ctx, (T **)dptr, vec.size());
        if (s == NOVA_OK)
            s = cuda_check(ctx, cudaMemcpy(*dptr, vec.data(), sizeof(T) * vec.size(), cudaMemcpyHostToDevice),
                           "cudaMemcpy");
    };
    up(&ctx->d_ia64, ia);
    up(&ctx->d_corr64, cr);
    up(&ctx->d_ia32, ia32);
    up(&ctx->d_corr32, cr32);
    up(&ctx->d_kx2, kx2);
    up(&ctx->d_ky2, ky2);
    up(&ctx->d_kz2, kz2);
    if (s == NOVA_OK) {
        s = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ctx->own_stream = (s == NOVA_OK);
    }
    if (s != NOVA_OK) {
        nova_destroy(ctx);
        return s;
    }
    *out = ctx;
    return NOVA_OK;
}

extern "C" nova_status nova_destroy(nova_ctx *ctx)
{
    if (!ctx) return NOVA_E_INVALID;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    prof_collect(ctx);
    for (auto e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->plans) {
        cufftDestroy(ctx->plan_f);
        cufftDestroy(ctx->plan_b);
    }
    if (ctx->dct_plans) {
        cufftDestroy(ctx->dct_f);
        cufftDestroy(ctx->dct_b);
    }
    if (ctx->dct2_plans) {
        cufftDestroy(ctx->dct2_f);
        cufftDestroy(ctx->dct2_b);
    }
    void *ptrs[] = {ctx->d_ia64, ctx->d_corr64, ctx->d_ia32, ctx->d_corr32, ctx->d_kx2, ctx->d_ky2, ctx->d_kz2,
                    ctx->d_spec, ctx->d_rhs, ctx->w64[0], ctx->w64[1], ctx->w64[2], ctx->w32[0], ctx->w32[1],
                    ctx->w32[2], ctx->d_part, ctx->d_scalar, ctx->d_flag, ctx->d_hist, ctx->d_stage, ctx->adj_pool, ctx->d_row, ctx->d_ext, ctx->d_ky2e, ctx->d_spec2, ctx->d_twN, ctx->d_tw256,
                    ctx->d_spec3, ctx->d_t512};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NOVA_OK;
}

extern "C" const char *nova_last_error(const nova_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" nova_status nova_set_stream(nova_ctx *ctx, void *stream)
{
    if (!ctx) return NOVA_E_INVALID;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return NOVA_OK;
}

extern "C" nova_status nova_synchronize(nova_ctx *ctx)
{
    if (!ctx) return NOVA_E_INVALID;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_mesh_local_n(const nova_ctx *ctx, int local_n[3])
{
    if (!ctx || !local_n) return NOVA_E_INVALID;
    for (int a = 0; a < 3; a++) local_n[a] = ctx->local_n[a];
    return NOVA_OK;
}

extern "C" nova_status nova_mesh_metrics(const nova_ctx *ctx, double *dzdxi, double *d2zdxi2)
{
    if (!ctx) return NOVA_E_INVALID;
    if (dzdxi) std::memcpy(dzdxi, ctx->dzdxi.data(), sizeof(double) * ctx->dzdxi.size());
    if (d2zdxi2) std::memcpy(d2zdxi2, ctx->d2zdxi2.data(), sizeof(double) * ctx->d2zdxi2.size());
    return NOVA_OK;
}

// =================================================================== fields ==
extern "C" nova_status nova_field_create(nova_ctx *ctx, int ncomp, int precision, nova_field **out)
{
    if (!ctx || !out || ncomp < 1 || ncomp > 9) return fail(ctx, NOVA_E_INVALID, "nova_field_create: bad arguments");
    if (precision != NOVA_F64 && precision != NOVA_F32SPLIT)
        return fail(ctx, NOVA_E_INVALID, "nova_field_create: unknown precision");
    nova_field *f = new (std::nothrow) nova_field();
    if (!f) return fail(ctx, NOVA_E_OOM, "nova_field_create: host allocation");
    f->nc = ncomp;
    f->prec = precision;
    f->n3 = ctx->g.N3;
    default_bc(ctx, &f->bc);
    const size_t n = (size_t)ncomp * f->n3;
    nova_status s;
    if (precision == NOVA_F64) {
        s = dalloc(ctx, &f->d64, n);
        if (s == NOVA_OK) s = cuda_check(ctx, cudaMemsetAsync(f->d64, 0, sizeof(double) * n, ctx->stream), "memset");
    } else {
        s = dalloc(ctx, &f->hi, n);
        if (s == NOVA_OK) s = dalloc(ctx, &f->lo, n);
        if (s == NOVA_OK) s = cuda_check(ctx, cudaMemsetAsync(f->hi, 0, sizeof(float) * n, ctx->stream), "memset");
        if (s == NOVA_OK) s = cuda_check(ctx, cudaMemsetAsync(f->lo, 0, sizeof(float) * n, ctx->stream), "memset");
    }
    if (s != NOVA_OK) {
        nova_field_destroy(ctx, f);
        return s;
    }
    *out = f;
    return NOVA_OK;
}

extern "C" nova_status nova_field_destroy(nova_ctx *ctx, nova_field *f)
{
    if (!f) return NOVA_E_INVALID;
    if (ctx && ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (f->d64) cudaFree(f->d64);
    if (f->hi) cudaFree(f->hi);
    if (f->lo) cudaFree(f->lo);
    delete f;
    return NOVA_OK;
}

extern "C" nova_status nova_field_set_bc(nova_ctx *ctx, nova_field *f, const nova_bc *bc)
{
    if (!ctx || !f || !bc) return fail(ctx, NOVA_E_INVALID, "nova_field_set_bc: null argument");
    for (int q = 0; q < 6 * (f->nc < 3 ? f->nc : 3); q++) {
        const int face = q % 6;
        const int axis = (face == NOVA_EAST || face == NOVA_WEST) ? 0 : (face == NOVA_TOP || face == NOVA_BOTTOM) ? 2 : 1;
        const int t = bc->type[q];
        if (t != NOVA_BC_PERIODIC && t != NOVA_BC_NEUMANN && t != NOVA_BC_DIRICHLET)
            return fail(ctx, NOVA_E_INVALID, "nova_field_set_bc: unknown BC type");
        const bool wall_axis = ctx->md.walls[axis] != 0;
        if (wall_axis == (t == NOVA_BC_PERIODIC))
            return fail(ctx, NOVA_E_INVALID, "nova_field_set_bc: periodic faces on periodic axes, "
                                             "Neumann/Dirichlet faces on wall axes");
    }
    f->bc = *bc;
    return NOVA_OK;
}

extern "C" nova_status nova_field_get_bc(nova_ctx *ctx, const nova_field *f, nova_bc *bc)
{
    if (!ctx || !f || !bc) return fail(ctx, NOVA_E_INVALID, "nova_field_get_bc: null argument");
    *bc = f->bc;
    return NOVA_OK;
}

static nova_status check_local_n(nova_ctx *ctx, const int local_n[3])
{
    if (!local_n) return fail(ctx, NOVA_E_INVALID, "local_n is null");
    for (int a = 0; a < 3; a++)
        if (local_n[a] != ctx->local_n[a])
            return fail(ctx, NOVA_E_INVALID, "local_n does not match the mesh (expected N+1+m per axis)");
    return NOVA_OK;
}

extern "C" nova_status nova_field_upload(nova_ctx *ctx, nova_field *f, const double *host, const int local_n[3])
{
    if (!ctx || !f || !host) return fail(ctx, NOVA_E_INVALID, "nova_field_upload: null argument");
    if (!on_mesh(ctx, f)) return fail(ctx, NOVA_E_INVALID, "nova_field_upload: field of another mesh");
    nova_status s = check_local_n(ctx, local_n);
    if (s != NOVA_OK) return s;
    const size_t n = (size_t)local_n[0] * local_n[1] * local_n[2] * f->nc;
    if ((s = ensure_stage(ctx, n)) != NOVA_OK) return s;
    CK(cudaMemcpyAsync(ctx->d_stage, host, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    launch_aos_to_soa(ctx->g, ctx->h, ctx->local_n, f->nc, ctx->d_stage, f->d64, f->hi, f->lo, ctx->stream);
    ctx->launches += 1;
    CKL("k_aos_to_soa");
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_field_download(nova_ctx *ctx, const nova_field *f, double *host, const int local_n[3],
                                           const nova_bc *bc)
{
    if (!ctx || !f || !host) return fail(ctx, NOVA_E_INVALID, "nova_field_download: null argument");
    if (!on_mesh(ctx, f)) return fail(ctx, NOVA_E_INVALID, "nova_field_download: field of another mesh");
    nova_status s = check_local_n(ctx, local_n);
    if (s != NOVA_OK) return s;
    nova_field tmp = *f;  // ghosts from the given BCs, or the field's own
    if (bc) {
        nova_field probe = *f;
        if ((s = nova_field_set_bc(ctx, &probe, bc)) != NOVA_OK) return s;
        tmp.bc = *bc;
    }
    const size_t n = (size_t)local_n[0] * local_n[1] * local_n[2] * f->nc;
    if ((s = ensure_stage(ctx, n)) != NOVA_OK) return s;
    launch_soa_to_aos(ctx->g, walls_of<double>(ctx, &tmp), ctx->h, ctx->local_n, f->nc, f->d64, f->hi, f->lo,
                      ctx->d_stage, ctx->stream);
    ctx->launches += 1;
    CKL("k_soa_to_aos");
    CK(cudaMemcpyAsync(host, ctx->d_stage, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

static nova_status soa_in(nova_ctx *ctx, nova_field *f, const double *src, cudaMemcpyKind kind)
{
    if (!on_mesh(ctx, f)) return fail(ctx, NOVA_E_INVALID, "field upload: field of another mesh");
    const size_t n = (size_t)f->nc * f->n3;
    if (f->prec == NOVA_F64) {
        CK(cudaMemcpyAsync(f->d64, src, sizeof(double) * n, kind, ctx->stream));
    } else {
        nova_status s = ensure_stage(ctx, n);
        if (s != NOVA_OK) return s;
        CK(cudaMemcpyAsync(ctx->d_stage, src, sizeof(double) * n, kind, ctx->stream));
        launch_split((long long)n, ctx->d_stage, f->hi, f->lo, ctx->stream);
        ctx->launches += 1;
        CKL("k_split");
    }
    return NOVA_OK;
}

static nova_status soa_out(nova_ctx *ctx, const nova_field *f, double *dst, cudaMemcpyKind kind)
{
    if (!on_mesh(ctx, f)) return fail(ctx, NOVA_E_INVALID, "field download: field of another mesh");
    const size_t n = (size_t)f->nc * f->n3;
    if (f->prec == NOVA_F64) {
        CK(cudaMemcpyAsync(dst, f->d64, sizeof(double) * n, kind, ctx->stream));
    } else {
        nova_status s = ensure_stage(ctx, n);
        if (s != NOVA_OK) return s;
        launch_join((long long)n, f->hi, f->lo, ctx->d_stage, ctx->stream);
        ctx->launches += 1;
        CKL("k_join");
        CK(cudaMemcpyAsync(dst, ctx->d_stage, sizeof(double) * n, kind, ctx->stream));
    }
    return NOVA_OK;
}

extern "C" nova_status nova_field_upload_soa(nova_ctx *ctx, nova_field *f, const double *host)
{
    if (!ctx || !f || !host) return fail(ctx, NOVA_E_INVALID, "nova_field_upload_soa: null argument");
    nova_status s = soa_in(ctx, f, host, cudaMemcpyHostToDevice);
    if (s != NOVA_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_field_download_soa(nova_ctx *ctx, const nova_field *f, double *host)
{
    if (!ctx || !f || !host) return fail(ctx, NOVA_E_INVALID, "nova_field_download_soa: null argument");
    nova_status s = soa_out(ctx, f, host, cudaMemcpyDeviceToHost);
    if (s != NOVA_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_field_copy_from_device(nova_ctx *ctx, nova_field *f, const double *dev)
{
    if (!ctx || !f || !dev) return fail(ctx, NOVA_E_INVALID, "nova_field_copy_from_device: null argument");
    return soa_in(ctx, f, dev, cudaMemcpyDeviceToDevice);
}

extern "C" nova_status nova_field_copy_to_device(nova_ctx *ctx, const nova_field *f, double *dev)
{
    if (!ctx || !f || !dev) return fail(ctx, NOVA_E_INVALID, "nova_field_copy_to_device: null argument");
    return soa_out(ctx, f, dev, cudaMemcpyDeviceToDevice);
}

// ================================================================ operators ==
static nova_status op_common(nova_ctx *ctx, int op, const nova_field *a, const nova_field *b, nova_field *out,
                             int nc_in, int nc_out, double nu)
{
    if (!ctx || !a || !out) return fail(ctx, NOVA_E_INVALID, "operator: null argument");
    if (!on_mesh(ctx, a) || !on_mesh(ctx, out) || (b && !on_mesh(ctx, b)))
        return fail(ctx, NOVA_E_INVALID, "operator: field of another mesh");
    if ((nc_in && a->nc != nc_in) || (nc_out && out->nc != nc_out))
        return fail(ctx, NOVA_E_INVALID, "operator: wrong number of components");
    if (a->prec != NOVA_F64 || out->prec != NOVA_F64 || (b && b->prec != NOVA_F64))
        return fail(ctx, NOVA_E_UNSUPPORTED, "operator: the ex:: entry points take FP64 fields");
    if (a == out || (b && b == out)) return fail(ctx, NOVA_E_INVALID, "operator: output aliases an input");
    launch_op(op, ctx->h, ctx->g, walls_of<double>(ctx, a), walls_of<double>(ctx, b), ctx->co64, ctx->d_ia64,
              ctx->d_corr64, a->d64, b ? b->d64 : nullptr, (op == OP_DIV_VF || op == OP_LAP_F) ? b->nc : a->nc, nu, out->d64,
              ctx->stream);
    ctx->launches += 1;
    CKL("operator kernel");
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_grad_s(nova_ctx *ctx, const nova_field *s, nova_field *out)
{
    return op_common(ctx, OP_GRAD_S, s, nullptr, out, 1, 3, 0.0);
}

extern "C" nova_status nova_grad_v(nova_ctx *ctx, const nova_field *U, nova_field *out)
{
    return op_common(ctx, OP_GRAD_V, U, nullptr, out, 3, 9, 0.0);
}

extern "C" nova_status nova_curl(nova_ctx *ctx, const nova_field *U, nova_field *out)
{
    return op_common(ctx, OP_CURL, U, nullptr, out, 3, 3, 0.0);
}

extern "C" nova_status nova_div_v(nova_ctx *ctx, const nova_field *U, nova_field *out)
{
    return op_common(ctx, OP_DIV_V, U, nullptr, out, 3, 1, 0.0);
}

extern "C" nova_status nova_div_t(nova_ctx *ctx, const nova_field *T, nova_field *out)
{
    if (!ctx || !T) return fail(ctx, NOVA_E_INVALID, "nova_div_t: null argument");
    if (T->nc != 9 && T->nc != 6) return fail(ctx, NOVA_E_INVALID, "nova_div_t: a tensor (9) or symmTensor (6) field");
    return op_common(ctx, OP_DIV_T, T, nullptr, out, 0, 3, 0.0);
}

extern "C" nova_status nova_div_st(nova_ctx *ctx, const nova_field *s, const nova_field *T, nova_field *out)
{
    if (!ctx || !s || !T) return fail(ctx, NOVA_E_INVALID, "nova_div_st: null argument");
    if (T->nc != 9) return fail(ctx, NOVA_E_INVALID, "nova_div_st: T must be a tensor (9) field");
    return op_common(ctx, OP_DIV_ST, s, T, out, 1, 3, 0.0);
}

extern "C" nova_status nova_laplacian_f(nova_ctx *ctx, const nova_field *nu, const nova_field *f, nova_field *out)
{
    if (!ctx || !nu || !f || !out) return fail(ctx, NOVA_E_INVALID, "nova_laplacian_f: null argument");
    if (out->nc != f->nc) return fail(ctx, NOVA_E_INVALID, "nova_laplacian_f: out must have the components of f");
    return op_common(ctx, OP_LAP_F, nu, f, out, 1, 0, 0.0);
}

extern "C" nova_status nova_div_vf(nova_ctx *ctx, const nova_field *U, const nova_field *f, nova_field *out)
{
    if (!ctx || !f) return fail(ctx, NOVA_E_INVALID, "nova_div_vf: null argument");
    if (out && out->nc != f->nc) return fail(ctx, NOVA_E_INVALID, "nova_div_vf: out must match f");
    return op_common(ctx, OP_DIV_VF, U, f, out, 3, 0, 0.0);
}

extern "C" nova_status nova_laplacian(nova_ctx *ctx, double nu, const nova_field *f, nova_field *out)
{
    if (!ctx || !f || !out) return fail(ctx, NOVA_E_INVALID, "nova_laplacian: null argument");
    if (out->nc != f->nc) return fail(ctx, NOVA_E_INVALID, "nova_laplacian: out must match f");
    return op_common(ctx, OP_LAP, f, nullptr, out, 0, 0, nu);
}

extern "C" nova_status nova_poisson_solve(nova_ctx *ctx, const nova_field *rhs, nova_field *p)
{
    if (!ctx || !rhs || !p) return fail(ctx, NOVA_E_INVALID, "nova_poisson_solve: null argument");
    if (!on_mesh(ctx, rhs) || !on_mesh(ctx, p)) return fail(ctx, NOVA_E_INVALID, "nova_poisson_solve: field of another mesh");
    if (rhs->nc != 1 || p->nc != 1 || rhs->prec != NOVA_F64 || p->prec != NOVA_F64)
        return fail(ctx, NOVA_E_INVALID, "nova_poisson_solve: needs FP64 scalar fields");
    nova_status s = ensure_fft(ctx);
    if (s == NOVA_OK) s = ensure_red(ctx);
    if (s != NOVA_OK) return s;
    CK(cudaMemsetAsync(ctx->d_flag + 1, 0, sizeof(int), ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_rhs, rhs->d64, sizeof(double) * ctx->g.N3, cudaMemcpyDeviceToDevice, ctx->stream));
    if ((s = poisson_device(ctx, ctx->d_rhs, p->d64)) != NOVA_OK) return s;
    int perr = 0;
    CK(cudaMemcpyAsync(&perr, ctx->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (perr) return fail(ctx, NOVA_E_CUDA, "nova_poisson_solve: a k_pois_tma pipeline wait timed out");
    return NOVA_OK;
}

extern "C" nova_status nova_field_maxabs(nova_ctx *ctx, const nova_field *f, double *out)
{
    if (!ctx || !f || !out) return fail(ctx, NOVA_E_INVALID, "nova_field_maxabs: null argument");
    if (!on_mesh(ctx, f)) return fail(ctx, NOVA_E_INVALID, "nova_field_maxabs: field of another mesh");
    if (f->nc != 1 || f->prec != NOVA_F64) return fail(ctx, NOVA_E_INVALID, "nova_field_maxabs: FP64 scalar only");
    nova_status s = ensure_red(ctx);
    if (s != NOVA_OK) return s;
    launch_maxabs(ctx->g, f->d64, ctx->d_part, ctx->d_scalar, ctx->stream);
    ctx->launches += 2;
    CKL("maxabs");
    CK(cudaMemcpyAsync(out, ctx->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_field_maxabs_noalloc(nova_ctx *ctx, const nova_field *f, double *out)
{
    if (!ctx || !f || !out) return fail(ctx, NOVA_E_INVALID, "nova_field_maxabs_noalloc: null argument");
    if (!on_mesh(ctx, f)) return fail(ctx, NOVA_E_INVALID, "nova_field_maxabs_noalloc: field of another mesh");
    if (f->nc != 1 || f->prec != NOVA_F64)
        return fail(ctx, NOVA_E_INVALID, "nova_field_maxabs_noalloc: FP64 scalar only");
    const long long n = ctx->g.N3;
    if (n < 1 || n > NOVA_MAXABS_NOALLOC_MAX_NODES)
        return fail(ctx, NOVA_E_INVALID,
                    "nova_field_maxabs_noalloc: " + std::to_string(n) +
                        " stored nodes, more than its static scratch covers (NOVA_MAXABS_NOALLOC_MAX_NODES = " +
                        std::to_string((long long)NOVA_MAXABS_NOALLOC_MAX_NODES) + "); use nova_field_maxabs");
    double *scratch = nullptr;
    CK(maxabs_noalloc_scratch(&scratch));
    launch_maxabs_noalloc(n, f->d64, scratch, ctx->stream);
    ctx->launches += 2;
    CKL("maxabs_noalloc");
    CK(cudaMemcpyAsync(out, scratch + kMaxabsStaticParts, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

// ================================================================== advance ==
namespace {

// app/shearLayer: the RK4 weights used as stage coefficients (shearLayer.cpp:164)
// and settings::RK4c_ (src/settings/settings.cpp:51), the projection's scale per stage
const double kShearW[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
const double kRK4c[4] = {0.5, 0.5, 1.0, 1.0};

// the physical parameters of a history row of a run (epsilon's viscosities,
// tools::CFL's dt and the mesh spacing Mesh::dx_, dy_, dz_)
DiagPhys phys_of(const nova_ctx *ctx, const nova_run_desc *rd)
{
    return DiagPhys{rd->nu, rd->model == NOVA_MODEL_MHD ? rd->eta : 0.0, rd->dt, ctx->md.L[0] / ctx->md.N[0],
                    ctx->md.L[1] / ctx->md.N[1], ctx->md.L[2] / ctx->md.N[2]};
}

DiagPhys phys_of(const DiagFinal &f)
{
    return DiagPhys{f.nu, f.eta, f.dt, f.dx, f.dy, f.dz};
}

nova_status ensure_work(nova_ctx *ctx, int prec)
{
    const size_t n = 3 * (size_t)ctx->g.N3;
    nova_status s = NOVA_OK;
    for (int q = 0; q < 3 && s == NOVA_OK; q++) {
        if (prec == NOVA_F64)
            s = dalloc(ctx, &ctx->w64[q], n);
        else
            s = dalloc(ctx, &ctx->w32[q], n);
    }
    // the FP32-split path's U* (FP64, the projection's input)
    if (s == NOVA_OK && prec != NOVA_F64) s = dalloc(ctx, &ctx->w64[0], n);
    if (s == NOVA_OK) s = ensure_fft(ctx);
    if (s == NOVA_OK) s = ensure_red(ctx);
    return s;
}

// One RK4 (or literal) sweep of an evolved field Y with the frozen field X,
// followed by its projection.  Y is updated in place.  With walls, the
// wall-node overwrites land where the reference calls correctBoundaryConditions:
// on every refreshed stage state (CLASSICAL: U = Ustar; U.correctBC), on U*
// before the projection, on p after the solve and on U after the correction.
// dg: diagnostics of Y as it enters this sweep (the previous step's history
// row), taken by the first stage kernel where it can (FP64 TMA stage), else
// by the diagnostics kernel right after that stage, which leaves Y unchanged.
nova_status evolve(nova_ctx *ctx, const nova_run_desc *rd, int phys, nova_field *Y, const nova_field *X,
                   nova_field *p, double visc, double divisor, double corr_scale, const StageDiag *dg = nullptr)
{
    const Geo &g = ctx->g;
    cudaStream_t st = ctx->stream;
    const bool lit = rd->rk_mode == NOVA_RK_LITERAL;
    const bool str = ctx->md.hyperbolic_z != 0;
    const bool walls = g.wallY != 0;
    const bool dct = walls && rd->poisson == NOVA_POISSON_DCT;
    const WallFix yfix = wall_fix_of(ctx, Y), pfix = wall_fix_of(ctx, p);
    const Walls<double> yw64 = walls_of<double>(ctx, Y), pw64 = walls_of<double>(ctx, p);
    auto fix64 = [&](double *f) {
        if (walls) {
            launch_wall_fix64(g, yfix, f, st);
            ctx->launches += 1;
        }
    };
    const StageExec ex{ctx->stage_impl, ctx->d_flag + 1};
    if (rd->rk_mode == NOVA_RK_SHEARLAYER) {
        // app/shearLayer/UEqn.H:14-38: per stage rk, U* = UOld + RK4[rk] dt F(U),
        // rhs = div(U*)/dt/RK4c[rk], U = U* - RK4c[rk] dt grad(p), with the
        // wall-node overwrites of U*.correctBC, p.correctBC and U.correctBC
        const bool f64 = Y->prec == NOVA_F64;
        if (dg) {
            launch_diag(ctx->h, g, walls_of<double>(ctx, Y), ctx->co64, ctx->d_ia64, Y->d64, Y->hi, Y->lo, nullptr,
                        nullptr, nullptr, 0, dg->part, dg->fin.step, dg->fin.time, dg->row, dg->flag, st,
                        phys_of(dg->fin));
            ctx->launches += 2;
        }
        // the split U* leaves stage 5 in FP64 (as many bytes as the (hi, lo)
        // pair) for the FP64 projection, whose correction writes the pair
        const size_t n3 = 3 * (size_t)g.N3;
        double *Old64 = ctx->w64[2], *Us64 = f64 ? ctx->w64[1] : ctx->w64[0];
        float *Oh = ctx->w32[0], *Ol = ctx->w32[1];
        const Walls<double> sw64 = walls_of<double>(ctx, Y, X);
        const Walls<float> sw32 = walls_of<float>(ctx, Y, X);
        if (walls) {
            if (f64)
                launch_wall_fix64(g, yfix, Y->d64, st);
            else
                launch_wall_fix_split(g, yfix, Y->hi, Y->lo, st);
            ctx->launches += 1;
        }
        if (f64) {
            CK(cudaMemcpyAsync(Old64, Y->d64, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st));
        } else {
            CK(cudaMemcpyAsync(Oh, Y->hi, sizeof(float) * n3, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(Ol, Y->lo, sizeof(float) * n3, cudaMemcpyDeviceToDevice, st));
        }
        for (int rk = 0; rk < 4; rk++) {
            cudaError_t e;
            {
                ProfScope ps(ctx, NOVA_K_STAGE);
                if (f64)
                    e = launch_stage64(phys, 5, str, g, sw64, ctx->co64, ctx->d_ia64, ctx->d_corr64, rd->dt, visc,
                                       StageArgs64{Y->d64, X ? X->d64 : nullptr, Old64, nullptr, Us64, kShearW[rk]},
                                       st, ex);
                else {
                    StageArgs32 a{Y->hi, X ? X->hi : nullptr, Oh, Ol, nullptr, nullptr, nullptr, nullptr,
                                  (float)kShearW[rk]};
                    a.out64 = Us64;
                    e = launch_stage32(phys, 5, str, g, sw32, ctx->co32, ctx->d_ia32, ctx->d_corr32, (float)rd->dt,
                                       (float)visc, a, st, ex);
                }
                ctx->launches += 1;
            }
            if (e != cudaSuccess) return stage_fail(ctx, e);
            if (walls) {
                launch_wall_fix64(g, yfix, Us64, st);
                ctx->launches += 1;
            }
            CKL("stage kernel");
            {
                ProfScope ps(ctx, NOVA_K_DIV);
                e = launch_div_proj(ctx->h, g, yw64, ctx->co64, ctx->d_ia64, Us64, nullptr, nullptr,
                                    divisor * kRK4c[rk], ctx->d_rhs, st, ex);
                if (e != cudaSuccess) return stage_fail(ctx, e);
                ctx->launches += 1;
            }
            CKL("divergence kernel");
            nova_status s =
                dct ? poisson_device_dct(ctx, ctx->d_rhs, p->d64) : poisson_device(ctx, ctx->d_rhs, p->d64);
            if (s != NOVA_OK) return s;
            if (walls && !dct) {
                launch_wall_fix64(g, pfix, p->d64, st);
                ctx->launches += 1;
            }
            {
                ProfScope ps(ctx, NOVA_K_CORRECT);
                e = launch_correct(ctx->h, g, pw64, ctx->co64, ctx->d_ia64, p->d64, kRK4c[rk] * corr_scale, Us64,
                                   f64 ? Y->d64 : nullptr, nullptr, nullptr, f64 ? nullptr : Y->hi,
                                   f64 ? nullptr : Y->lo, st, ex);
                if (e != cudaSuccess) return stage_fail(ctx, e);
                ctx->launches += 1;
            }
            if (walls) {
                if (f64)
                    launch_wall_fix64(g, yfix, Y->d64, st);
                else
                    launch_wall_fix_split(g, yfix, Y->hi, Y->lo, st);
                ctx->launches += 1;
            }
            CKL("correction kernel");
        }
        return NOVA_OK;
    }
    if (Y->prec == NOVA_F64) {
        const Walls<double> sw = walls_of<double>(ctx, Y, X);
        fix64(Y->d64);
        double *Ustar;
        nova_status sst = NOVA_OK;
        auto run64 = [&](int stage, const StageArgs64 &a) {
            ProfScope ps(ctx, NOVA_K_STAGE);
            const bool first = stage == 0 || stage == 4;
            bool taken = false;
            const cudaError_t e = launch_stage64(phys, stage, str, g, sw, ctx->co64, ctx->d_ia64, ctx->d_corr64,
                                                 rd->dt, visc, a, st, StageExec{ctx->stage_impl, ctx->d_flag + 1},
                                                 first ? dg : nullptr, &taken);
            if (e != cudaSuccess && sst == NOVA_OK) sst = stage_fail(ctx, e);
            ctx->launches += taken ? 2 : 1;
            if (first && dg && !taken) {
                launch_diag(ctx->h, g, walls_of<double>(ctx, Y), ctx->co64, ctx->d_ia64, Y->d64, nullptr, nullptr,
                            nullptr, nullptr, nullptr, 0, dg->part, dg->fin.step, dg->fin.time, dg->row, dg->flag, st,
                            phys_of(dg->fin));
                ctx->launches += 2;
            }
        };
        if (lit) {
            run64(4, StageArgs64{Y->d64, X ? X->d64 : nullptr, nullptr, nullptr, ctx->w64[1]});
            Ustar = ctx->w64[1];
        } else {
            double *w0 = ctx->w64[0], *w1 = ctx->w64[1], *A = ctx->w64[2];
            const double *Xp = X ? X->d64 : nullptr;
            run64(0, StageArgs64{Y->d64, Xp, nullptr, A, w0});
            fix64(w0);
            run64(1, StageArgs64{w0, Xp, Y->d64, A, w1});
            fix64(w1);
            run64(2, StageArgs64{w1, Xp, Y->d64, A, w0});
            fix64(w0);
            run64(3, StageArgs64{w0, Xp, nullptr, A, Y->d64});
            Ustar = Y->d64;
        }
        fix64(Ustar);
        if (sst != NOVA_OK) return sst;
        CKL("stage kernel");
        {
            ProfScope ps(ctx, NOVA_K_DIV);
            const cudaError_t e = launch_div_proj(ctx->h, g, yw64, ctx->co64, ctx->d_ia64, Ustar, nullptr, nullptr,
                                                  divisor, ctx->d_rhs, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
            if (e != cudaSuccess) return stage_fail(ctx, e);
            ctx->launches += 1;
        }
        CKL("k_div_tiled");
        nova_status s = dct ? poisson_device_dct(ctx, ctx->d_rhs, p->d64) : poisson_device(ctx, ctx->d_rhs, p->d64);
        if (s != NOVA_OK) return s;
        if (walls && !dct) {
            launch_wall_fix64(g, pfix, p->d64, st);
            ctx->launches += 1;
        }
        {
            ProfScope ps(ctx, NOVA_K_CORRECT);
            const cudaError_t e = launch_correct(ctx->h, g, pw64, ctx->co64, ctx->d_ia64, p->d64, corr_scale, Ustar,
                                                 Y->d64, nullptr, nullptr, nullptr, nullptr, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
            if (e != cudaSuccess) return stage_fail(ctx, e);
            ctx->launches += 1;
        }
        fix64(Y->d64);
        CKL("k_correct_tiled");
    } else {
        const Walls<float> sw = walls_of<float>(ctx, Y, X);
        auto fix32 = [&](float *f) {
            if (walls) {
                launch_wall_fix32(g, yfix, f, st);
                ctx->launches += 1;
            }
        };
        auto fixpair = [&](float *hi, float *lo) {
            if (walls) {
                launch_wall_fix_split(g, yfix, hi, lo, st);
                ctx->launches += 1;
            }
        };
        fixpair(Y->hi, Y->lo);
        if (dg) {
            launch_diag(ctx->h, g, walls_of<double>(ctx, Y), ctx->co64, ctx->d_ia64, nullptr, Y->hi, Y->lo, nullptr,
                        nullptr, nullptr, 0, dg->part, dg->fin.step, dg->fin.time, dg->row, dg->flag, st,
                        phys_of(dg->fin));
            ctx->launches += 2;
        }
        nova_status sst = NOVA_OK;
        auto run32 = [&](int stage, const StageArgs32 &a) {
            ProfScope ps(ctx, NOVA_K_STAGE);
            const cudaError_t e = launch_stage32(phys, stage, str, g, sw, ctx->co32, ctx->d_ia32, ctx->d_corr32,
                                                 (float)rd->dt, (float)visc, a, st,
                                                 StageExec{ctx->stage_impl, ctx->d_flag + 1});
            if (e != cudaSuccess && sst == NOVA_OK) sst = stage_fail(ctx, e);
            ctx->launches += 1;
        };
        const float *Xp = X ? X->hi : nullptr;
        // U* leaves the last stage in FP64 (as many bytes as the (hi, lo) pair)
        // for the FP64 projection, which reads it as the FP64 path does
        double *Us64 = ctx->w64[0];
        if (lit) {
            StageArgs32 a{Y->hi, Xp, nullptr, Y->lo, nullptr, nullptr, nullptr, nullptr};
            a.out64 = Us64;
            run32(4, a);
        } else {
            float *w0 = ctx->w32[0], *w1 = ctx->w32[1], *A = ctx->w32[2];
            run32(0, StageArgs32{Y->hi, Xp, nullptr, nullptr, A, w0, nullptr, nullptr});
            fix32(w0);
            run32(1, StageArgs32{w0, Xp, Y->hi, nullptr, A, w1, nullptr, nullptr});
            fix32(w1);
            run32(2, StageArgs32{w1, Xp, Y->hi, nullptr, A, w0, nullptr, nullptr});
            fix32(w0);
            StageArgs32 a{w0, Xp, Y->hi, Y->lo, A, nullptr, nullptr, nullptr};
            a.out64 = Us64;
            run32(3, a);
        }
        if (walls) {
            launch_wall_fix64(g, yfix, Us64, st);
            ctx->launches += 1;
        }
        if (sst != NOVA_OK) return sst;
        CKL("stage kernel");
        {
            ProfScope ps(ctx, NOVA_K_DIV);
            const cudaError_t e = launch_div_proj(ctx->h, g, yw64, ctx->co64, ctx->d_ia64, Us64, nullptr, nullptr,
                                                  divisor, ctx->d_rhs, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
            if (e != cudaSuccess) return stage_fail(ctx, e);
            ctx->launches += 1;
        }
        CKL("k_div_tiled");
        nova_status s = dct ? poisson_device_dct(ctx, ctx->d_rhs, p->d64) : poisson_device(ctx, ctx->d_rhs, p->d64);
        if (s != NOVA_OK) return s;
        if (walls && !dct) {
            launch_wall_fix64(g, pfix, p->d64, st);
            ctx->launches += 1;
        }
        {
            ProfScope ps(ctx, NOVA_K_CORRECT);
            const cudaError_t e = launch_correct(ctx->h, g, pw64, ctx->co64, ctx->d_ia64, p->d64, corr_scale, Us64,
                                                 nullptr, nullptr, nullptr, Y->hi, Y->lo, st,
                                                 StageExec{ctx->stage_impl, ctx->d_flag + 1});
            if (e != cudaSuccess) return stage_fail(ctx, e);
            ctx->launches += 1;
        }
        fixpair(Y->hi, Y->lo);
        CKL("k_correct_tiled");
    }
    return NOVA_OK;
}

}  // namespace

extern "C" nova_status nova_advance(nova_ctx *ctx, const nova_run_desc *rd, nova_state *st, int nsteps, double *hist)
{
    if (!ctx || !rd || !st || nsteps < 0) return fail(ctx, NOVA_E_INVALID, "nova_advance: bad arguments");
    const bool mhd = rd->model == NOVA_MODEL_MHD;
    if (rd->model != NOVA_MODEL_NS && !mhd) return fail(ctx, NOVA_E_INVALID, "nova_advance: unknown model");
    if (rd->rk_mode != NOVA_RK_LITERAL && rd->rk_mode != NOVA_RK_CLASSICAL && rd->rk_mode != NOVA_RK_SHEARLAYER)
        return fail(ctx, NOVA_E_INVALID, "nova_advance: unknown rk_mode");
    const bool shear = rd->rk_mode == NOVA_RK_SHEARLAYER;
    if (ctx->h != 3) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_advance: the fused kernels are built for m = 6");
    if (mhd && ctx->g.wallY) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_advance: MHD is built for periodic meshes");
    if (rd->poisson != NOVA_POISSON_FFT && rd->poisson != NOVA_POISSON_DCT)
        return fail(ctx, NOVA_E_INVALID, "nova_advance: unknown poisson mode");
    if (ctx->g.wallY && rd->poisson == NOVA_POISSON_DCT && st->p)
        for (int face : {NOVA_NORTH, NOVA_SOUTH})
            if (st->p->bc.type[face] != NOVA_BC_NEUMANN || st->p->bc.val[face] != 0.0)
                return fail(ctx, NOVA_E_INVALID, "nova_advance: the DCT wall Poisson needs Neumann-0 pressure walls");
    if (!valid_field(ctx, st->U, 3) || !valid_field(ctx, st->p, 1) || st->p->prec != NOVA_F64 || st->U->prec != rd->precision)
        return fail(ctx, NOVA_E_INVALID, "nova_advance: U (3 comps, run precision) and p (FP64 scalar) required");
    if (mhd && (!valid_field(ctx, st->B, 3) || !valid_field(ctx, st->pB, 1) || st->pB->prec != NOVA_F64 ||
                st->B->prec != rd->precision))
        return fail(ctx, NOVA_E_INVALID, "nova_advance: MHD needs B (3 comps) and pB (FP64 scalar)");
    if (!(rd->dt > 0.0)) return fail(ctx, NOVA_E_INVALID, "nova_advance: dt must be positive");
    nova_status s = ensure_work(ctx, rd->precision);
    if (s != NOVA_OK) return s;
    if (hist && rd->diag_every > 0) {
        if (ctx->hist_cap < (long long)nsteps * NOVA_HIST_COLS) {
            if (ctx->d_hist) cudaFree(ctx->d_hist);
            ctx->d_hist = nullptr;
            ctx->hist_cap = 0;
            if ((s = dalloc(ctx, &ctx->d_hist, (size_t)nsteps * NOVA_HIST_COLS)) != NOVA_OK) return s;
            ctx->hist_cap = (long long)nsteps * NOVA_HIST_COLS;
        }
        CK(cudaMemsetAsync(ctx->d_hist, 0, sizeof(double) * nsteps * NOVA_HIST_COLS, ctx->stream));
    }
    CK(cudaMemsetAsync(ctx->d_flag, 0, 2 * sizeof(int), ctx->stream));
    // FP64 Navier-Stokes on a uniform periodic mesh: the history row of a step
    // is taken by the first stage kernel of the next step, which reads the same
    // state with its halos and forms its divergence anyway (the last step's row
    // by the diagnostics kernel)
    const bool defer_diag = hist && rd->diag_every > 0 && !mhd && !shear && rd->precision == NOVA_F64 && !ctx->g.wallY &&
                            !ctx->md.hyperbolic_z && ctx->h == 3 && ctx->stage_impl != STAGE_MARCH &&
                            stage_tma_fits(ctx->g, true);
    StageDiag pend{};
    bool have = false;
    for (int n = 0; n < nsteps; n++) {
        // app/TG_Piosson/RKLoop.H (NS) or app/OT_Poisson/UEqn.H then BEqn.H (MHD)
        s = evolve(ctx, rd, mhd ? PHYS_MHD_U : PHYS_NS, st->U, mhd ? st->B : nullptr, st->p, rd->nu, rd->dt, rd->dt,
                   have ? &pend : nullptr);
        have = false;
        if (s != NOVA_OK) return s;
        if (mhd && !shear) {
            // B loop is always the refreshed RK4 (BEqn.H:86-87); B cleaning has no 1/dt (BEqn.H:91-94)
            nova_run_desc rb = *rd;
            rb.rk_mode = NOVA_RK_CLASSICAL;
            s = evolve(ctx, &rb, PHYS_MHD_B, st->B, st->U, st->pB, rd->eta, 1.0, 1.0);
            if (s != NOVA_OK) return s;
        }
        if (hist && rd->diag_every > 0 && ((n + 1) % rd->diag_every == 0 || n + 1 == nsteps) && defer_diag &&
            n + 1 < nsteps) {
            pend = StageDiag{ctx->d_part, diag_blocks(ctx->g), ctx->d_hist + (long long)n * NOVA_HIST_COLS,
                             ctx->d_flag,
                             diag_final_of(ctx->g, phys_of(ctx, rd), (double)(n + 1), rd->t0 + (n + 1) * rd->dt,
                                           st->U->d64, nullptr, nullptr)};
            have = true;
        } else if (hist && rd->diag_every > 0 && ((n + 1) % rd->diag_every == 0 || n + 1 == nsteps)) {
            ProfScope ps(ctx, NOVA_K_DIAG);
            const nova_field *U = st->U, *B = mhd ? st->B : nullptr;
            launch_diag(ctx->h, ctx->g, walls_of<double>(ctx, U, B), ctx->co64, ctx->d_ia64, U->d64, U->hi, U->lo,
                        B ? B->d64 : nullptr,
                        B ? B->hi : nullptr, B ? B->lo : nullptr, mhd ? 1 : 0, ctx->d_part, (double)(n + 1),
                        rd->t0 + (n + 1) * rd->dt, ctx->d_hist + (long long)n * NOVA_HIST_COLS, ctx->d_flag,
                        ctx->stream, phys_of(ctx, rd));
            ctx->launches += 2;
            CKL("k_diag");
        }
    }
    if (hist && rd->diag_every > 0)
        CK(cudaMemcpyAsync(hist, ctx->d_hist, sizeof(double) * nsteps * NOVA_HIST_COLS, cudaMemcpyDeviceToHost,
                           ctx->stream));
    int flag[2] = {0, 0};
    CK(cudaMemcpyAsync(flag, ctx->d_flag, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (flag[1]) return fail(ctx, NOVA_E_TIMEOUT, "nova_advance: a stage kernel pipeline wait timed out");
    if (flag[0]) return fail(ctx, NOVA_E_NONFINITE, "nova_advance: non-finite value in the diagnostics");
    return NOVA_OK;
}

// ================================================================== adjoint ==
namespace {

// One classical RK4 loop of the evolved FP64 field Yin with the frozen field X
// (physics phys, viscosity visc), stage states into S2, S3, S4 (S4 may alias
// S2); with `full` the stage-3 result and its projection (rhs divisor and
// correction scale `div`) into out (may alias Yin).  Without `full` only the
// stage states are produced.
nova_status rk_loop64(nova_ctx *ctx, const nova_run_desc *rd, int phys, double visc, double div, const double *Yin,
                      const double *X, double *S2, double *S3, double *S4, double *out, bool full)
{
    const Geo &g = ctx->g;
    cudaStream_t st = ctx->stream;
    double *A = ctx->w64[2];
    const bool str = ctx->md.hyperbolic_z != 0;
    nova_status sst = NOVA_OK;
    auto run = [&](int stage, const StageArgs64 &a) {
        ProfScope ps(ctx, NOVA_K_STAGE);
        const cudaError_t e = launch_stage64(phys, stage, str, g, Walls<double>{}, ctx->co64, ctx->d_ia64,
                                             ctx->d_corr64, rd->dt, visc, a, st,
                                             StageExec{ctx->stage_impl, ctx->d_flag + 1});
        if (e != cudaSuccess && sst == NOVA_OK) sst = stage_fail(ctx, e);
        ctx->launches += 1;
    };
    run(0, StageArgs64{Yin, X, nullptr, A, S2});
    run(1, StageArgs64{S2, X, Yin, A, S3});
    run(2, StageArgs64{S3, X, Yin, A, S4});
    if (!full) {
        if (sst != NOVA_OK) return sst;
        CKL("stage kernel");
        return NOVA_OK;
    }
    run(3, StageArgs64{S4, X, nullptr, A, out});
    if (sst != NOVA_OK) return sst;
    CKL("stage kernel");
    cudaError_t e = launch_div_proj(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, out, nullptr, nullptr, div,
                                    ctx->d_rhs, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
    if (e != cudaSuccess) return stage_fail(ctx, e);
    ctx->launches += 1;
    CKL("k_div_tiled");
    nova_status s = poisson_device(ctx, ctx->d_rhs, ctx->w64[1]);
    if (s != NOVA_OK) return s;
    e = launch_correct(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, ctx->w64[1], div, out, out, nullptr,
                       nullptr, nullptr, nullptr, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
    if (e != cudaSuccess) return stage_fail(ctx, e);
    ctx->launches += 1;
    CKL("k_correct_tiled");
    return NOVA_OK;
}

// One classical RK4 loop + projection of an FP32-split state (physics phys,
// viscosity visc, frozen field X given by its hi part, rhs divisor and
// correction scale div), the launches of the split path of nova_advance:
// (hi, lo) -> (ohi, olo) (may alias), FP32 stage states into S2, S3, S4 (S4
// may alias S2), the pressure into pbuf (FP64).  Without `full` only the
// stage states are produced.
nova_status rk_loop32(nova_ctx *ctx, const nova_run_desc *rd, int phys, double visc, double div, const float *hi,
                      const float *lo, const float *X, float *S2, float *S3, float *S4, float *ohi, float *olo,
                      double *pbuf, bool full)
{
    const Geo &g = ctx->g;
    cudaStream_t st = ctx->stream;
    float *A = ctx->w32[2];
    const bool str = ctx->md.hyperbolic_z != 0;
    nova_status sst = NOVA_OK;
    auto run = [&](int stage, const StageArgs32 &a) {
        ProfScope ps(ctx, NOVA_K_STAGE);
        const cudaError_t e = launch_stage32(phys, stage, str, g, Walls<float>{}, ctx->co32, ctx->d_ia32,
                                             ctx->d_corr32, (float)rd->dt, (float)visc, a, st,
                                             StageExec{ctx->stage_impl, ctx->d_flag + 1});
        if (e != cudaSuccess && sst == NOVA_OK) sst = stage_fail(ctx, e);
        ctx->launches += 1;
    };
    run(0, StageArgs32{hi, X, nullptr, nullptr, A, S2, nullptr, nullptr});
    run(1, StageArgs32{S2, X, hi, nullptr, A, S3, nullptr, nullptr});
    run(2, StageArgs32{S3, X, hi, nullptr, A, S4, nullptr, nullptr});
    double *Us64 = ctx->w64[0];  // U* in FP64, as nova_advance's split path keeps it
    if (full) {
        StageArgs32 a{S4, X, hi, lo, A, nullptr, nullptr, nullptr};
        a.out64 = Us64;
        run(3, a);
    }
    if (sst != NOVA_OK) return sst;
    CKL("stage kernel");
    if (!full) return NOVA_OK;
    cudaError_t e = launch_div_proj(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, Us64, nullptr, nullptr, div,
                                    ctx->d_rhs, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
    if (e != cudaSuccess) return stage_fail(ctx, e);
    ctx->launches += 1;
    CKL("k_div_tiled");
    nova_status s = poisson_device(ctx, ctx->d_rhs, pbuf);
    if (s != NOVA_OK) return s;
    e = launch_correct(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, pbuf, div, Us64, nullptr, nullptr, nullptr,
                       ohi, olo, st, StageExec{ctx->stage_impl, ctx->d_flag + 1});
    if (e != cudaSuccess) return stage_fail(ctx, e);
    ctx->launches += 1;
    CKL("k_correct_tiled");
    return NOVA_OK;
}

// One classical RK4 step + projection of an FP64 Navier-Stokes state:
// Uin -> Uout (may alias), stage states into Y2, Y3, Y4 (Y4 may alias Y2).
// Without `full` only the stage states are produced.
nova_status fwd_step64(nova_ctx *ctx, const nova_run_desc *rd, const double *Uin, double *Y2, double *Y3, double *Y4,
                       double *Uout, bool full)
{
    return rk_loop64(ctx, rd, PHYS_NS, rd->nu, rd->dt, Uin, nullptr, Y2, Y3, Y4, Uout, full);
}

// out = P in = in - G L^-1 D in (the projection is symmetric: its own adjoint)
nova_status project64(nova_ctx *ctx, const double *in, double *out, double *pbuf)
{
    const Geo &g = ctx->g;
    cudaError_t e = launch_div_proj(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, in, nullptr, nullptr, 1.0,
                                    ctx->d_rhs, ctx->stream, StageExec{ctx->stage_impl, ctx->d_flag + 1});
    if (e != cudaSuccess) return stage_fail(ctx, e);
    ctx->launches += 1;
    CKL("k_div_tiled");
    nova_status s = poisson_device(ctx, ctx->d_rhs, pbuf);
    if (s != NOVA_OK) return s;
    e = launch_correct(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, pbuf, 1.0, in, out, nullptr, nullptr,
                       nullptr, nullptr, ctx->stream, StageExec{ctx->stage_impl, ctx->d_flag + 1});
    if (e != cudaSuccess) return stage_fail(ctx, e);
    ctx->launches += 1;
    CKL("k_correct_tiled");
    return NOVA_OK;
}

// the adjoint's device pool: `need` doubles, grown on demand
nova_status adj_pool(nova_ctx *ctx, size_t need)
{
    if (ctx->adj_cap >= need) return NOVA_OK;
    if (ctx->adj_pool) cudaFree(ctx->adj_pool);
    ctx->adj_pool = nullptr;
    ctx->adj_cap = 0;
    const nova_status s = dalloc(ctx, &ctx->adj_pool, need);
    if (s == NOVA_OK) ctx->adj_cap = need;
    return s;
}

nova_status adjoint_mhd(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init, nova_field *gradU,
                        nova_field *gradB, double *objective);
nova_status adjoint_split(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init, nova_field *gradU,
                          double *objective);
nova_status adjoint_mhd_split(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init, nova_field *gradU,
                              nova_field *gradB, double *objective);

}  // namespace

extern "C" nova_status nova_adjoint_grad(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init,
                                         nova_field *gradU, nova_field *gradB, double *objective)
{
    if (!ctx || !ad || !init || !gradU) return fail(ctx, NOVA_E_INVALID, "nova_adjoint_grad: null argument");
    const nova_run_desc *rd = &ad->run;
    const bool mhd = rd->model == NOVA_MODEL_MHD;
    const bool split = rd->precision == NOVA_F32SPLIT;
    if ((rd->model != NOVA_MODEL_NS && !mhd) || rd->rk_mode != NOVA_RK_CLASSICAL ||
        (rd->precision != NOVA_F64 && !split))
        return fail(ctx, NOVA_E_UNSUPPORTED,
                    "nova_adjoint_grad: built for classical RK4 Navier-Stokes and MHD, FP64 or FP32-split");
    const bool window = ad->objective == NOVA_OBJ_DISSIPATION_WINDOW;
    const bool linear = ad->objective == NOVA_OBJ_LINEAR_FINAL;
    if (ad->objective != NOVA_OBJ_EKIN_FINAL && !window && !(mhd && ad->objective == NOVA_OBJ_ETOT_FINAL) &&
        !(linear && !mhd && !split))
        return fail(ctx, NOVA_E_UNSUPPORTED, "nova_adjoint_grad: unknown objective for this model and precision");
    if (linear && (!valid_field(ctx, ad->weight, 3) || ad->weight->prec != NOVA_F64))
        return fail(ctx, NOVA_E_INVALID, "nova_adjoint_grad: the linear objective needs a 3-component FP64 weight");
    if (window && (ad->window_start < 0 || ad->window_start >= ad->nsteps))
        return fail(ctx, NOVA_E_INVALID, "nova_adjoint_grad: window_start must lie in [0, nsteps)");
    if (ctx->h != 3) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_adjoint_grad: the fused kernels are built for m = 6");
    if (ctx->g.wallY || ctx->md.hyperbolic_z)
        return fail(ctx, NOVA_E_UNSUPPORTED, "nova_adjoint_grad: periodic uniform meshes only");
    if (ad->nsteps < 1 || ad->checkpoint_every < 1 || !(rd->dt > 0.0))
        return fail(ctx, NOVA_E_INVALID, "nova_adjoint_grad: nsteps, checkpoint_every and dt must be positive");
    if (!valid_field(ctx, init->U, 3) || init->U->prec != rd->precision || !valid_field(ctx, gradU, 3) ||
        gradU->prec != NOVA_F64)
        return fail(ctx, NOVA_E_INVALID,
                    "nova_adjoint_grad: U (3 comps, run precision) and gradU (3 comps, FP64) required");
    if (mhd) {
        if (!valid_field(ctx, init->B, 3) || init->B->prec != rd->precision || !gradB || !valid_field(ctx, gradB, 3) ||
            gradB->prec != NOVA_F64)
            return fail(ctx, NOVA_E_INVALID,
                        "nova_adjoint_grad: MHD needs B (3 comps, run precision) and gradB (3 comps, FP64)");
        return split ? adjoint_mhd_split(ctx, ad, init, gradU, gradB, objective)
                     : adjoint_mhd(ctx, ad, init, gradU, gradB, objective);
    }
    if (gradB) return fail(ctx, NOVA_E_INVALID, "nova_adjoint_grad: gradB is for MHD runs (pass NULL)");
    if (split) return adjoint_split(ctx, ad, init, gradU, objective);
    nova_status s = ensure_work(ctx, NOVA_F64);
    if (s != NOVA_OK) return s;
    CK(cudaMemsetAsync(ctx->d_flag + 1, 0, sizeof(int), ctx->stream));
    const int N = ad->nsteps, K = ad->checkpoint_every;
    const int nck = (N + K - 1) / K;
    const int mmax = K < N ? K : N;
    const size_t V = 3 * (size_t)ctx->g.N3;
    // layout: nck checkpoints | 4*mmax segment fields | lam, mu, gA, gB, Lam
    const size_t need = V * ((size_t)nck + 4 * (size_t)mmax + 5);
    if ((s = adj_pool(ctx, need)) != NOVA_OK) return s;
    double *ck = ctx->adj_pool;
    double *seg = ck + V * nck;
    double *lam = seg + V * 4 * mmax, *mu = lam + V, *gA = mu + V, *gB = gA + V, *Lam = gB + V;
    auto St = [&](int t) { return seg + V * (4 * (size_t)t + 0); };
    auto Y2 = [&](int t) { return seg + V * (4 * (size_t)t + 1); };
    auto Y3 = [&](int t) { return seg + V * (4 * (size_t)t + 2); };
    auto Y4 = [&](int t) { return seg + V * (4 * (size_t)t + 3); };
    cudaStream_t st = ctx->stream;

    // forward pass, keeping every K-th state (the running state lives in mu);
    // the last segment keeps its states and stage states as it goes, so the
    // reverse sweep does not recompute it
    const int c_last = nck - 1, n_last = c_last * K, m_last = N - n_last;
    CK(cudaMemcpyAsync(ck, init->U->d64, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
    if ((s = dalloc(ctx, &ctx->d_row, 2 * NOVA_HIST_COLS)) != NOVA_OK) return s;
    const int n0w = window ? ad->window_start : -1;
    auto ekin = [&](const double *u, double *row_dev) {  // diagnostics row of the state u
        launch_diag(ctx->h, ctx->g, Walls<double>{}, ctx->co64, ctx->d_ia64, u, nullptr, nullptr, nullptr, nullptr,
                    nullptr, 0, ctx->d_part, 0.0, 0.0, row_dev, ctx->d_flag, st);
        ctx->launches += 2;
    };
    for (int n = 0; n < N; n++) {
        if (n == n0w)  // Ek(n0) of the window: the state before step n0
            ekin(n >= n_last ? (n == n_last ? ck + V * c_last : St(n - n_last)) : (n % K == 0 ? ck + V * (n / K) : mu),
                 ctx->d_row + NOVA_HIST_COLS);
        if (n >= n_last) {
            const int t = n - n_last;
            if (t == 0) CK(cudaMemcpyAsync(St(0), ck + V * c_last, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
            double *out = (t + 1 < m_last) ? St(t + 1) : mu;
            if ((s = fwd_step64(ctx, rd, St(t), Y2(t), Y3(t), Y4(t), out, true)) != NOVA_OK) return s;
            continue;
        }
        const double *src = (n % K == 0) ? ck + V * (n / K) : mu;
        if ((s = fwd_step64(ctx, rd, src, ctx->w64[0], ctx->w64[1], ctx->w64[0], mu, true)) != NOVA_OK) return s;
        if ((n + 1) % K == 0 && n + 1 < N)
            CK(cudaMemcpyAsync(ck + V * ((n + 1) / K), mu, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
    }
    // Ek(N); lambda_N = dJ/dU_N = +-U_N / N^3 (the unique nodes are the N^3 entries)
    ekin(mu, ctx->d_row);
    double row[2 * NOVA_HIST_COLS];
    CK(cudaMemcpyAsync(row, ctx->d_row, sizeof(row), cudaMemcpyDeviceToHost, st));
    if (linear) {  // J = <w, U_N> / N^3, lambda_N = w / N^3
        launch_dot((long long)V, ad->weight->d64, mu, 1.0 / (double)ctx->g.N3, ctx->d_part, 592, ctx->d_scalar, st);
        launch_scale_copy((long long)V, 1.0 / (double)ctx->g.N3, ad->weight->d64, lam, st);
        ctx->launches += 3;
        CK(cudaMemcpyAsync(row + 2, ctx->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
        launch_scale_copy((long long)V, (window ? -1.0 : 1.0) / (double)ctx->g.N3, mu, lam, st);
        ctx->launches += 1;
    }
    CKL("adjoint seed");

    // reverse sweep, segment by segment
    cudaError_t aerr = cudaSuccess;
    for (int c = nck - 1; c >= 0; c--) {
        const int n0 = c * K;
        const int m = (N - n0) < K ? (N - n0) : K;
        if (c != c_last) {
            CK(cudaMemcpyAsync(St(0), ck + V * c, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
            for (int t = 0; t < m; t++) {
                const bool full = t + 1 < m;
                if ((s = fwd_step64(ctx, rd, St(t), Y2(t), Y3(t), Y4(t), full ? St(t + 1) : nullptr, full)) !=
                    NOVA_OK)
                    return s;
            }
        }
        for (int t = m - 1; t >= 0; t--) {
            {
                ProfScope ps(ctx, NOVA_K_DIV);
                if ((s = project64(ctx, lam, mu, gB)) != NOVA_OK) return s;
            }
            const double dt = rd->dt, nu = rd->nu;
            auto adj = [&](int stage, const AdjArgs &a) {
                ProfScope ps(ctx, NOVA_K_ADJ);
                const cudaError_t e = launch_adj_stage64(stage, ctx->g, ctx->co64, ctx->d_ia64, dt, nu, a, st,
                                                         ctx->stage_impl != STAGE_MARCH ? ctx->d_flag + 1 : nullptr);
                if (e != cudaSuccess && aerr == cudaSuccess) aerr = e;
                ctx->launches += 1;
            };
            adj(4, AdjArgs{Y4(t), mu, mu, nullptr, gA, Lam});
            adj(3, AdjArgs{Y3(t), gA, mu, Lam, gB, Lam});
            adj(2, AdjArgs{Y2(t), gB, mu, Lam, gA, Lam});
            adj(1, AdjArgs{St(t), gA, mu, Lam, lam, nullptr});
            CKL("k_adj_stage");
            if (n0 + t == n0w) {  // lambda is dJ/dU_n0: add dEk(n0)/dU_n0
                launch_axpy((long long)V, 1.0 / (double)ctx->g.N3, St(t), lam, st);
                ctx->launches += 1;
            }
        }
    }
    if (aerr != cudaSuccess) return stage_fail(ctx, aerr);
    CK(cudaMemcpyAsync(gradU->d64, lam, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
    int perr = 0;
    CK(cudaMemcpyAsync(&perr, ctx->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (perr) return fail(ctx, NOVA_E_TIMEOUT, "nova_adjoint_grad: a stage kernel pipeline wait timed out");
    const double J = window ? row[NOVA_HIST_COLS + 2] - row[2] : row[2];
    if (objective) *objective = J;
    if (!std::isfinite(J)) return fail(ctx, NOVA_E_NONFINITE, "nova_adjoint_grad: non-finite objective");
    return NOVA_OK;
}

namespace {

// Discrete adjoint of the MHD step of nova_advance (app/OT_Poisson: UEqn.H then
// BEqn.H): U^{n+1} = P Phi_U(U^n; B^n), then B^{n+1} = P Phi_B(B^n; U^{n+1}),
// Phi the classical RK4 loops, P the projection.  Reverse of one step, given
// lamU = dJ/dU^{n+1}, lamB = dJ/dB^{n+1}:
//   B loop: mu = P lamB; stages S = 4..1 of Phi_B (frozen U^{n+1}, stage states
//           Z_S): the recursion of k_adj_stage with xi = dt dF_B/dB^T g_S gives
//           lamB <- dJ/dB^n through the B loop, and lamU += dt dF_B/dU^T g_S;
//   U loop: mu = P lamU; stages S = 4..1 of Phi_U (frozen B^n, stage states
//           Y_S): the Navier-Stokes recursion gives lamU <- dJ/dU^n, and
//           lamB += dt dF_U/dB^T g_S.
nova_status adjoint_mhd(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init, nova_field *gradU,
                        nova_field *gradB, double *objective)
{
    const nova_run_desc *rd = &ad->run;
    const bool window = ad->objective == NOVA_OBJ_DISSIPATION_WINDOW;
    const bool etot = window || ad->objective == NOVA_OBJ_ETOT_FINAL;
    nova_status s = ensure_work(ctx, NOVA_F64);
    if (s != NOVA_OK) return s;
    CK(cudaMemsetAsync(ctx->d_flag + 1, 0, sizeof(int), ctx->stream));
    const int N = ad->nsteps, K = ad->checkpoint_every;
    const int nck = (N + K - 1) / K;
    const int mmax = K < N ? K : N;
    const size_t V = 3 * (size_t)ctx->g.N3;
    // layout: nck U and nck B checkpoints | 8*mmax + 1 segment fields | lamU, lamB, mu, gA, gB, Lam
    if ((s = adj_pool(ctx, V * (2 * (size_t)nck + 8 * (size_t)mmax + 1 + 6))) != NOVA_OK) return s;
    double *ckU = ctx->adj_pool, *ckB = ckU + V * nck;
    double *seg = ckB + V * nck;
    double *lamU = seg + V * (8 * (size_t)mmax + 1), *lamB = lamU + V, *mu = lamB + V, *gA = mu + V, *gB = gA + V,
           *Lam = gB + V;
    // per step t of a segment: U^n, Y2, Y3, Y4 (U loop), B^n, Z2, Z3, Z4 (B loop); U^{n+1} is slot t + 1
    auto slot = [&](int t, int f) { return seg + V * (8 * (size_t)t + f); };
    auto St = [&](int t) { return slot(t, 0); };
    auto SB = [&](int t) { return slot(t, 4); };
    cudaStream_t st = ctx->stream;
    double *w0 = ctx->w64[0], *w1 = ctx->w64[1];
    double *runU = mu, *runB = Lam;  // running state of the forward pass

    // one step; the B loop is projected only when bout is set
    auto step = [&](const double *u, const double *b, double *y2, double *y3, double *y4, double *uout, double *z2,
                    double *z3, double *z4, double *bout) {
        nova_status r = rk_loop64(ctx, rd, PHYS_MHD_U, rd->nu, rd->dt, u, b, y2, y3, y4, uout, true);
        if (r != NOVA_OK) return r;
        return rk_loop64(ctx, rd, PHYS_MHD_B, rd->eta, 1.0, b, uout, z2, z3, z4, bout, bout != nullptr);
    };
    auto seg_step = [&](int t, int m, double *blast) {
        return step(St(t), SB(t), slot(t, 1), slot(t, 2), slot(t, 3), St(t + 1), slot(t, 5), slot(t, 6), slot(t, 7),
                    t + 1 < m ? SB(t + 1) : blast);
    };
    auto energy = [&](const double *u, const double *b, double *row_dev) {  // diagnostics row of (u, b)
        launch_diag(ctx->h, ctx->g, Walls<double>{}, ctx->co64, ctx->d_ia64, u, nullptr, nullptr, b, nullptr,
                    nullptr, 1, ctx->d_part, 0.0, 0.0, row_dev, ctx->d_flag, st);
        ctx->launches += 2;
    };
    auto copy = [&](double *dst, const double *src) {
        return cudaMemcpyAsync(dst, src, sizeof(double) * V, cudaMemcpyDeviceToDevice, st);
    };

    // forward pass, keeping (U, B) every K steps; the last segment keeps its
    // states and stage states as it goes
    const int c_last = nck - 1, n_last = c_last * K, m_last = N - n_last;
    CK(copy(ckU, init->U->d64));
    CK(copy(ckB, init->B->d64));
    if ((s = dalloc(ctx, &ctx->d_row, 2 * NOVA_HIST_COLS)) != NOVA_OK) return s;
    const int n0w = window ? ad->window_start : -1;
    for (int n = 0; n < N; n++) {
        if (n == n0w) {  // E(n0) of the window: the state before step n0
            const bool ck = n == n_last || (n < n_last && n % K == 0);
            const double *u = ck ? ckU + V * (n / K) : (n > n_last ? St(n - n_last) : runU);
            const double *b = ck ? ckB + V * (n / K) : (n > n_last ? SB(n - n_last) : runB);
            energy(u, b, ctx->d_row + NOVA_HIST_COLS);
        }
        if (n >= n_last) {
            const int t = n - n_last;
            if (t == 0) {
                CK(copy(St(0), ckU + V * c_last));
                CK(copy(SB(0), ckB + V * c_last));
            }
            if ((s = seg_step(t, m_last, runB)) != NOVA_OK) return s;
            continue;
        }
        const bool ck = n % K == 0;
        if ((s = step(ck ? ckU + V * (n / K) : runU, ck ? ckB + V * (n / K) : runB, w0, w1, w0, runU, w0, w1, w0,
                      runB)) != NOVA_OK)
            return s;
        if ((n + 1) % K == 0 && n + 1 < N) {
            CK(copy(ckU + V * ((n + 1) / K), runU));
            CK(copy(ckB + V * ((n + 1) / K), runB));
        }
    }
    // E(N); lamU = dJ/dU_N = +-U_N / N^3, lamB = +-B_N / N^3 (or 0 for Ek alone)
    const double *UN = St(m_last);
    energy(UN, runB, ctx->d_row);
    double row[2 * NOVA_HIST_COLS];
    CK(cudaMemcpyAsync(row, ctx->d_row, sizeof(row), cudaMemcpyDeviceToHost, st));
    const double seed = (window ? -1.0 : 1.0) / (double)ctx->g.N3;
    launch_scale_copy((long long)V, seed, UN, lamU, st);
    ctx->launches += 1;
    if (etot) {
        launch_scale_copy((long long)V, seed, runB, lamB, st);
        ctx->launches += 1;
    } else {
        CK(cudaMemsetAsync(lamB, 0, sizeof(double) * V, st));
    }
    CKL("adjoint seed");

    const double dt = rd->dt;
    cudaError_t aerr = cudaSuccess;
    auto adj_u = [&](int stage, const AdjArgs &a) {
        ProfScope ps(ctx, NOVA_K_ADJ);
        const cudaError_t e = launch_adj_stage64(stage, ctx->g, ctx->co64, ctx->d_ia64, dt, rd->nu, a, st,
                                                 ctx->stage_impl != STAGE_MARCH ? ctx->d_flag + 1 : nullptr);
        if (e != cudaSuccess && aerr == cudaSuccess) aerr = e;
        ctx->launches += 1;
    };
    auto adj_mhd = [&](int kind, int stage, const AdjArgs &a, double *acc) {
        ProfScope ps(ctx, NOVA_K_ADJ);
        const cudaError_t e = launch_adj_mhd(kind, stage, ctx->g, ctx->co64, ctx->d_ia64, dt, rd->eta, a, acc, st,
                                             ctx->stage_impl != STAGE_MARCH ? ctx->d_flag + 1 : nullptr);
        if (e != cudaSuccess && aerr == cudaSuccess) aerr = e;
        ctx->launches += 1;
    };
    auto proj = [&](const double *in) {
        ProfScope ps(ctx, NOVA_K_DIV);
        return project64(ctx, in, mu, gB);
    };
    enum { UB = 0, BU = 1, BB = 2 };
    for (int c = nck - 1; c >= 0; c--) {
        const int n0 = c * K;
        const int m = (N - n0) < K ? (N - n0) : K;
        if (c != c_last) {
            CK(copy(St(0), ckU + V * c));
            CK(copy(SB(0), ckB + V * c));
            for (int t = 0; t < m; t++)
                if ((s = seg_step(t, m, nullptr)) != NOVA_OK) return s;
        }
        for (int t = m - 1; t >= 0; t--) {
            // B loop: frozen U^{n+1} = St(t + 1), stage states Z_S
            if ((s = proj(lamB)) != NOVA_OK) return s;
            const double *Up = St(t + 1);
            adj_mhd(BB, 4, AdjArgs{Up, mu, mu, nullptr, gA, Lam}, nullptr);
            adj_mhd(BU, 4, AdjArgs{slot(t, 7), mu, mu, nullptr, nullptr, nullptr}, lamU);
            adj_mhd(BB, 3, AdjArgs{Up, gA, mu, Lam, gB, Lam}, nullptr);
            adj_mhd(BU, 3, AdjArgs{slot(t, 6), gA, nullptr, nullptr, nullptr, nullptr}, lamU);
            adj_mhd(BB, 2, AdjArgs{Up, gB, mu, Lam, gA, Lam}, nullptr);
            adj_mhd(BU, 2, AdjArgs{slot(t, 5), gB, nullptr, nullptr, nullptr, nullptr}, lamU);
            adj_mhd(BB, 1, AdjArgs{Up, gA, mu, Lam, lamB, nullptr}, nullptr);
            adj_mhd(BU, 1, AdjArgs{SB(t), gA, nullptr, nullptr, nullptr, nullptr}, lamU);
            // U loop: frozen B^n = SB(t), stage states Y_S
            if ((s = proj(lamU)) != NOVA_OK) return s;
            adj_u(4, AdjArgs{slot(t, 3), mu, mu, nullptr, gA, Lam});
            adj_mhd(UB, 4, AdjArgs{SB(t), mu, mu, nullptr, nullptr, nullptr}, lamB);
            adj_u(3, AdjArgs{slot(t, 2), gA, mu, Lam, gB, Lam});
            adj_mhd(UB, 3, AdjArgs{SB(t), gA, nullptr, nullptr, nullptr, nullptr}, lamB);
            adj_u(2, AdjArgs{slot(t, 1), gB, mu, Lam, gA, Lam});
            adj_mhd(UB, 2, AdjArgs{SB(t), gB, nullptr, nullptr, nullptr, nullptr}, lamB);
            adj_u(1, AdjArgs{St(t), gA, mu, Lam, lamU, nullptr});
            adj_mhd(UB, 1, AdjArgs{SB(t), gA, nullptr, nullptr, nullptr, nullptr}, lamB);
            CKL("k_adj_mhd");
            if (n0 + t == n0w) {  // add dE(n0)/d(U, B)_n0
                launch_axpy((long long)V, 1.0 / (double)ctx->g.N3, St(t), lamU, st);
                launch_axpy((long long)V, 1.0 / (double)ctx->g.N3, SB(t), lamB, st);
                ctx->launches += 2;
            }
        }
    }
    if (aerr != cudaSuccess) return stage_fail(ctx, aerr);
    CK(copy(gradU->d64, lamU));
    CK(copy(gradB->d64, lamB));
    int perr = 0;
    CK(cudaMemcpyAsync(&perr, ctx->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (perr) return fail(ctx, NOVA_E_TIMEOUT, "nova_adjoint_grad: a stage kernel pipeline wait timed out");
    const double E = row[2] + (etot ? row[3] : 0.0);
    const double J = window ? (row[NOVA_HIST_COLS + 2] + row[NOVA_HIST_COLS + 3]) - E : E;
    if (objective) *objective = J;
    if (!std::isfinite(J)) return fail(ctx, NOVA_E_NONFINITE, "nova_adjoint_grad: non-finite objective");
    return NOVA_OK;
}

}  // namespace

namespace {

// FP32-split adjoint: the trajectory of the split path of nova_advance (FP32
// stage states, (hi, lo) state, FP64 projection) and the adjoint stage
// kernels in FP32 (stage states, directions g, running sum Lam); the adjoint
// lam = dJ/dU between steps and its projection mu = P lam stay FP64, and the
// last reverse stage forms lam = mu + (Lam + xi) in FP64.  Checkpoints keep
// the (hi, lo) pairs, so the recomputed segments repeat the forward pass bit
// for bit.
nova_status adjoint_split(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init, nova_field *gradU,
                          double *objective)
{
    const nova_run_desc *rd = &ad->run;
    const bool window = ad->objective == NOVA_OBJ_DISSIPATION_WINDOW;
    nova_status s = ensure_work(ctx, NOVA_F32SPLIT);
    if (s != NOVA_OK) return s;
    CK(cudaMemsetAsync(ctx->d_flag + 1, 0, sizeof(int), ctx->stream));
    const int N = ad->nsteps, K = ad->checkpoint_every;
    const int nck = (N + K - 1) / K;
    const int mmax = K < N ? K : N;
    const size_t V = 3 * (size_t)ctx->g.N3;
    const size_t Vf = (V + 63) / 64 * 64;  // float field stride (256-byte aligned starts)
    // layout: FP64 lam, mu, pbuf | FP32: nck (hi, lo) checkpoints, mmax + 1 step states (hi),
    // 3 mmax stage states, lo_run, lo_n0, gA, gB, Lam
    const size_t nf = 2 * (size_t)nck + (mmax + 1) + 3 * (size_t)mmax + 5;
    if ((s = adj_pool(ctx, 3 * V + (nf * Vf + 1) / 2)) != NOVA_OK) return s;
    double *lam = ctx->adj_pool, *mu = lam + V, *pbuf = mu + V;
    float *fl = reinterpret_cast<float *>(pbuf + V);
    auto F = [&](size_t i) { return fl + Vf * i; };
    auto ckhi = [&](int c) { return F(2 * (size_t)c); };
    auto cklo = [&](int c) { return F(2 * (size_t)c + 1); };
    const size_t b1 = 2 * (size_t)nck, b2 = b1 + mmax + 1, b3 = b2 + 3 * (size_t)mmax;
    auto Y1 = [&](int t) { return F(b1 + t); };
    auto Ys = [&](int t, int st) { return F(b2 + 3 * (size_t)t + (st - 2)); };  // stage states 2, 3, 4
    float *lo_run = F(b3), *lo_n0 = F(b3 + 1), *gA = F(b3 + 2), *gB = F(b3 + 3), *Lam = F(b3 + 4);
    float *runhi = gA, *runlo = gB;  // running state of the forward pass outside the kept segment
    float *w0 = ctx->w32[0], *w1 = ctx->w32[1];
    cudaStream_t st = ctx->stream;
    auto copyf = [&](float *dst, const float *src) {
        return cudaMemcpyAsync(dst, src, sizeof(float) * V, cudaMemcpyDeviceToDevice, st);
    };
    auto energy = [&](const float *hi, const float *lo, double *row_dev) {
        launch_diag(ctx->h, ctx->g, Walls<double>{}, ctx->co64, ctx->d_ia64, nullptr, hi, lo, nullptr, nullptr,
                    nullptr, 0, ctx->d_part, 0.0, 0.0, row_dev, ctx->d_flag, st);
        ctx->launches += 2;
    };

    const int c_last = nck - 1, n_last = c_last * K, m_last = N - n_last;
    CK(copyf(ckhi(0), init->U->hi));
    CK(copyf(cklo(0), init->U->lo));
    if ((s = dalloc(ctx, &ctx->d_row, 2 * NOVA_HIST_COLS)) != NOVA_OK) return s;
    const int n0w = window ? ad->window_start : -1;
    for (int n = 0; n < N; n++) {
        const bool kept = n >= n_last;
        const int t = n - n_last;
        if (kept && t == 0) {
            CK(copyf(Y1(0), ckhi(c_last)));
            CK(copyf(lo_run, cklo(c_last)));
        }
        const bool ck = !kept && n % K == 0;
        const float *hi = kept ? Y1(t) : (ck ? ckhi(n / K) : runhi);
        const float *lo = kept ? lo_run : (ck ? cklo(n / K) : runlo);
        if (n == n0w) {  // E(n0) of the window: the state before step n0
            energy(hi, lo, ctx->d_row + NOVA_HIST_COLS);
            CK(copyf(lo_n0, lo));
        }
        if (kept) {
            if ((s = rk_loop32(ctx, rd, PHYS_NS, rd->nu, rd->dt, Y1(t), lo_run, nullptr, Ys(t, 2), Ys(t, 3),
                               Ys(t, 4), Y1(t + 1), lo_run, pbuf, true)) != NOVA_OK)
                return s;
            continue;
        }
        if ((s = rk_loop32(ctx, rd, PHYS_NS, rd->nu, rd->dt, hi, lo, nullptr, w0, w1, w0, runhi, runlo, pbuf,
                           true)) != NOVA_OK)
            return s;
        if ((n + 1) % K == 0 && n + 1 < N) {
            CK(copyf(ckhi((n + 1) / K), runhi));
            CK(copyf(cklo((n + 1) / K), runlo));
        }
    }
    // E(N); lam_N = +-U_N / N^3 with U_N = hi + lo
    energy(Y1(m_last), lo_run, ctx->d_row);
    double row[2 * NOVA_HIST_COLS];
    CK(cudaMemcpyAsync(row, ctx->d_row, sizeof(row), cudaMemcpyDeviceToHost, st));
    launch_join((long long)V, Y1(m_last), lo_run, lam, st);
    launch_scale_copy((long long)V, (window ? -1.0 : 1.0) / (double)ctx->g.N3, lam, lam, st);
    ctx->launches += 2;
    CKL("adjoint seed");

    const float dt = (float)rd->dt, nu = (float)rd->nu;
    auto adj = [&](int stage, const AdjArgs32 &a) {
        ProfScope ps(ctx, NOVA_K_ADJ);
        launch_adj_stage32(stage, ctx->g, ctx->co32, ctx->d_ia32, dt, nu, a, st);
        ctx->launches += 1;
    };
    for (int c = nck - 1; c >= 0; c--) {
        const int n0 = c * K;
        const int m = (N - n0) < K ? (N - n0) : K;
        if (c != c_last) {
            CK(copyf(Y1(0), ckhi(c)));
            CK(copyf(lo_run, cklo(c)));
            for (int t = 0; t < m; t++) {
                if (n0 + t == n0w) CK(copyf(lo_n0, lo_run));
                if ((s = rk_loop32(ctx, rd, PHYS_NS, rd->nu, rd->dt, Y1(t), lo_run, nullptr, Ys(t, 2), Ys(t, 3),
                                   Ys(t, 4), Y1(t + 1), lo_run, pbuf, t + 1 < m)) != NOVA_OK)
                    return s;
            }
        }
        for (int t = m - 1; t >= 0; t--) {
            {
                ProfScope ps(ctx, NOVA_K_DIV);
                if ((s = project64(ctx, lam, mu, pbuf)) != NOVA_OK) return s;
            }
            adj(4, AdjArgs32{Ys(t, 4), nullptr, mu, nullptr, gA, Lam, nullptr});
            adj(3, AdjArgs32{Ys(t, 3), gA, mu, Lam, gB, Lam, nullptr});
            adj(2, AdjArgs32{Ys(t, 2), gB, mu, Lam, gA, Lam, nullptr});
            adj(1, AdjArgs32{Y1(t), gA, mu, Lam, nullptr, nullptr, lam});
            CKL("k_adj_stage");
            if (n0 + t == n0w) {  // lam is dJ/dU_n0: add dEk(n0)/dU_n0 = U_n0 / N^3
                launch_join((long long)V, Y1(t), lo_n0, pbuf, st);
                launch_axpy((long long)V, 1.0 / (double)ctx->g.N3, pbuf, lam, st);
                ctx->launches += 2;
            }
        }
    }
    CK(cudaMemcpyAsync(gradU->d64, lam, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
    int perr = 0;
    CK(cudaMemcpyAsync(&perr, ctx->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (perr) return fail(ctx, NOVA_E_TIMEOUT, "nova_adjoint_grad: a stage kernel pipeline wait timed out");
    const double J = window ? row[NOVA_HIST_COLS + 2] - row[2] : row[2];
    if (objective) *objective = J;
    if (!std::isfinite(J)) return fail(ctx, NOVA_E_NONFINITE, "nova_adjoint_grad: non-finite objective");
    return NOVA_OK;
}

}  // namespace

namespace {

// FP32-split MHD adjoint: the split MHD step of nova_advance (U loop with B's
// hi part frozen, then the B loop with the new U's hi part frozen, FP64
// projections), (hi, lo) checkpoints and FP32 stage states; the stage
// recursions and the coupling transposes in FP32; lamU, lamB and both
// projections in FP64.  The reverse of a step is that of adjoint_mhd.
nova_status adjoint_mhd_split(nova_ctx *ctx, const nova_adj_desc *ad, const nova_state *init, nova_field *gradU,
                              nova_field *gradB, double *objective)
{
    const nova_run_desc *rd = &ad->run;
    const bool window = ad->objective == NOVA_OBJ_DISSIPATION_WINDOW;
    const bool etot = window || ad->objective == NOVA_OBJ_ETOT_FINAL;
    nova_status s = ensure_work(ctx, NOVA_F32SPLIT);
    if (s != NOVA_OK) return s;
    CK(cudaMemsetAsync(ctx->d_flag + 1, 0, sizeof(int), ctx->stream));
    const int N = ad->nsteps, K = ad->checkpoint_every;
    const int nck = (N + K - 1) / K;
    const int mmax = K < N ? K : N;
    const size_t V = 3 * (size_t)ctx->g.N3;
    const size_t Vf = (V + 63) / 64 * 64;
    // layout: FP64 lamU, lamB, mu, pbuf | FP32: nck (U hi, U lo, B hi, B lo) checkpoints,
    // per step t: U hi, Y2, Y3, Y4, B hi, Z2, Z3, Z4, then U hi of step mmax,
    // loU, loB, loU0, loB0, gA, gB, Lam, one more running field
    const size_t nf = 4 * (size_t)nck + 8 * (size_t)mmax + 1 + 8;
    if ((s = adj_pool(ctx, 4 * V + (nf * Vf + 1) / 2)) != NOVA_OK) return s;
    double *lamU = ctx->adj_pool, *lamB = lamU + V, *mu = lamB + V, *pbuf = mu + V;
    float *fl = reinterpret_cast<float *>(pbuf + V);
    auto F = [&](size_t i) { return fl + Vf * i; };
    auto ck = [&](int c, int f) { return F(4 * (size_t)c + f); };  // f: 0 U hi, 1 U lo, 2 B hi, 3 B lo
    const size_t b1 = 4 * (size_t)nck, b2 = b1 + 8 * (size_t)mmax + 1;
    auto slot = [&](int t, int f) { return F(b1 + 8 * (size_t)t + f); };
    auto Uh = [&](int t) { return slot(t, 0); };
    auto Bh = [&](int t) { return slot(t, 4); };
    float *loU = F(b2), *loB = F(b2 + 1), *loU0 = F(b2 + 2), *loB0 = F(b2 + 3), *gA = F(b2 + 4), *gB = F(b2 + 5),
          *Lam = F(b2 + 6), *extra = F(b2 + 7);
    float *rUh = gA, *rUl = gB, *rBh = Lam, *rBl = extra;  // running state of the forward pass
    float *w0 = ctx->w32[0], *w1 = ctx->w32[1];
    cudaStream_t st = ctx->stream;
    auto copyf = [&](float *dst, const float *src) {
        return cudaMemcpyAsync(dst, src, sizeof(float) * V, cudaMemcpyDeviceToDevice, st);
    };
    auto energy = [&](const float *uh, const float *ul, const float *bh, const float *bl, double *row_dev) {
        launch_diag(ctx->h, ctx->g, Walls<double>{}, ctx->co64, ctx->d_ia64, nullptr, uh, ul, nullptr, bh, bl, 1,
                    ctx->d_part, 0.0, 0.0, row_dev, ctx->d_flag, st);
        ctx->launches += 2;
    };
    // one step of the kept or recomputed segment; the B loop is projected
    // (into bhi, lo in place) unless this is a recomputed segment's last step
    auto seg_step = [&](int t, int m, float *blast) {
        nova_status r = rk_loop32(ctx, rd, PHYS_MHD_U, rd->nu, rd->dt, Uh(t), loU, Bh(t), slot(t, 1), slot(t, 2),
                                  slot(t, 3), Uh(t + 1), loU, pbuf, true);
        if (r != NOVA_OK) return r;
        float *bh = t + 1 < m ? Bh(t + 1) : blast;
        return rk_loop32(ctx, rd, PHYS_MHD_B, rd->eta, 1.0, Bh(t), loB, Uh(t + 1), slot(t, 5), slot(t, 6),
                         slot(t, 7), bh, loB, pbuf, bh != nullptr);
    };

    const int c_last = nck - 1, n_last = c_last * K, m_last = N - n_last;
    CK(copyf(ck(0, 0), init->U->hi));
    CK(copyf(ck(0, 1), init->U->lo));
    CK(copyf(ck(0, 2), init->B->hi));
    CK(copyf(ck(0, 3), init->B->lo));
    if ((s = dalloc(ctx, &ctx->d_row, 2 * NOVA_HIST_COLS)) != NOVA_OK) return s;
    const int n0w = window ? ad->window_start : -1;
    for (int n = 0; n < N; n++) {
        const bool kept = n >= n_last;
        const int t = n - n_last;
        if (kept && t == 0) {
            CK(copyf(Uh(0), ck(c_last, 0)));
            CK(copyf(loU, ck(c_last, 1)));
            CK(copyf(Bh(0), ck(c_last, 2)));
            CK(copyf(loB, ck(c_last, 3)));
        }
        const bool isck = !kept && n % K == 0;
        const float *uh = kept ? Uh(t) : (isck ? ck(n / K, 0) : rUh);
        const float *ul = kept ? loU : (isck ? ck(n / K, 1) : rUl);
        const float *bh = kept ? Bh(t) : (isck ? ck(n / K, 2) : rBh);
        const float *bl = kept ? loB : (isck ? ck(n / K, 3) : rBl);
        if (n == n0w) {  // E(n0) of the window: the state before step n0
            energy(uh, ul, bh, bl, ctx->d_row + NOVA_HIST_COLS);
            CK(copyf(loU0, ul));
            CK(copyf(loB0, bl));
        }
        if (kept) {
            if ((s = seg_step(t, m_last, rBh)) != NOVA_OK) return s;
            continue;
        }
        if ((s = rk_loop32(ctx, rd, PHYS_MHD_U, rd->nu, rd->dt, uh, ul, bh, w0, w1, w0, rUh, rUl, pbuf, true)) !=
            NOVA_OK)
            return s;
        if ((s = rk_loop32(ctx, rd, PHYS_MHD_B, rd->eta, 1.0, bh, bl, rUh, w0, w1, w0, rBh, rBl, pbuf, true)) !=
            NOVA_OK)
            return s;
        if ((n + 1) % K == 0 && n + 1 < N) {
            CK(copyf(ck((n + 1) / K, 0), rUh));
            CK(copyf(ck((n + 1) / K, 1), rUl));
            CK(copyf(ck((n + 1) / K, 2), rBh));
            CK(copyf(ck((n + 1) / K, 3), rBl));
        }
    }
    // E(N); lamU = +-U_N / N^3, lamB = +-B_N / N^3 (or 0 for Ek alone); U_N = (Uh(m_last), loU), B_N = (rBh, loB)
    energy(Uh(m_last), loU, rBh, loB, ctx->d_row);
    double row[2 * NOVA_HIST_COLS];
    CK(cudaMemcpyAsync(row, ctx->d_row, sizeof(row), cudaMemcpyDeviceToHost, st));
    const double seed = (window ? -1.0 : 1.0) / (double)ctx->g.N3;
    launch_join((long long)V, Uh(m_last), loU, lamU, st);
    launch_scale_copy((long long)V, seed, lamU, lamU, st);
    ctx->launches += 2;
    if (etot) {
        launch_join((long long)V, rBh, loB, lamB, st);
        launch_scale_copy((long long)V, seed, lamB, lamB, st);
        ctx->launches += 2;
    } else {
        CK(cudaMemsetAsync(lamB, 0, sizeof(double) * V, st));
    }
    CKL("adjoint seed");

    const float dt = (float)rd->dt;
    auto adj_u = [&](int stage, const AdjArgs32 &a) {
        ProfScope ps(ctx, NOVA_K_ADJ);
        launch_adj_stage32(stage, ctx->g, ctx->co32, ctx->d_ia32, dt, (float)rd->nu, a, st);
        ctx->launches += 1;
    };
    auto adj_mhd = [&](int kind, int stage, const AdjArgs32 &a, double *acc) {
        ProfScope ps(ctx, NOVA_K_ADJ);
        launch_adj_mhd32(kind, stage, ctx->g, ctx->co32, ctx->d_ia32, dt, (float)rd->eta, a, acc, st);
        ctx->launches += 1;
    };
    auto proj = [&](const double *in) {
        ProfScope ps(ctx, NOVA_K_DIV);
        return project64(ctx, in, mu, pbuf);
    };
    enum { UB = 0, BU = 1, BB = 2 };
    for (int c = nck - 1; c >= 0; c--) {
        const int n0 = c * K;
        const int m = (N - n0) < K ? (N - n0) : K;
        if (c != c_last) {
            CK(copyf(Uh(0), ck(c, 0)));
            CK(copyf(loU, ck(c, 1)));
            CK(copyf(Bh(0), ck(c, 2)));
            CK(copyf(loB, ck(c, 3)));
            for (int t = 0; t < m; t++) {
                if (n0 + t == n0w) {
                    CK(copyf(loU0, loU));
                    CK(copyf(loB0, loB));
                }
                if ((s = seg_step(t, m, nullptr)) != NOVA_OK) return s;
            }
        }
        for (int t = m - 1; t >= 0; t--) {
            // B loop: frozen U^{n+1} (its hi part, Uh(t + 1)), stage states Z_S
            if ((s = proj(lamB)) != NOVA_OK) return s;
            const float *Up = Uh(t + 1);
            adj_mhd(BB, 4, AdjArgs32{Up, nullptr, mu, nullptr, gA, Lam, nullptr}, nullptr);
            adj_mhd(BU, 4, AdjArgs32{slot(t, 7), nullptr, mu, nullptr, nullptr, nullptr, nullptr}, lamU);
            adj_mhd(BB, 3, AdjArgs32{Up, gA, mu, Lam, gB, Lam, nullptr}, nullptr);
            adj_mhd(BU, 3, AdjArgs32{slot(t, 6), gA, mu, nullptr, nullptr, nullptr, nullptr}, lamU);
            adj_mhd(BB, 2, AdjArgs32{Up, gB, mu, Lam, gA, Lam, nullptr}, nullptr);
            adj_mhd(BU, 2, AdjArgs32{slot(t, 5), gB, mu, nullptr, nullptr, nullptr, nullptr}, lamU);
            adj_mhd(BB, 1, AdjArgs32{Up, gA, mu, Lam, nullptr, nullptr, lamB}, nullptr);
            adj_mhd(BU, 1, AdjArgs32{Bh(t), gA, mu, nullptr, nullptr, nullptr, nullptr}, lamU);
            // U loop: frozen B^n (its hi part, Bh(t)), stage states Y_S
            if ((s = proj(lamU)) != NOVA_OK) return s;
            adj_u(4, AdjArgs32{slot(t, 3), nullptr, mu, nullptr, gA, Lam, nullptr});
            adj_mhd(UB, 4, AdjArgs32{Bh(t), nullptr, mu, nullptr, nullptr, nullptr, nullptr}, lamB);
            adj_u(3, AdjArgs32{slot(t, 2), gA, mu, Lam, gB, Lam, nullptr});
            adj_mhd(UB, 3, AdjArgs32{Bh(t), gA, mu, nullptr, nullptr, nullptr, nullptr}, lamB);
            adj_u(2, AdjArgs32{slot(t, 1), gB, mu, Lam, gA, Lam, nullptr});
            adj_mhd(UB, 2, AdjArgs32{Bh(t), gB, mu, nullptr, nullptr, nullptr, nullptr}, lamB);
            adj_u(1, AdjArgs32{Uh(t), gA, mu, Lam, nullptr, nullptr, lamU});
            adj_mhd(UB, 1, AdjArgs32{Bh(t), gA, mu, nullptr, nullptr, nullptr, nullptr}, lamB);
            CKL("k_adj_mhd");
            if (n0 + t == n0w) {  // add dE(n0)/d(U, B)_n0 = (U, B)_n0 / N^3
                launch_join((long long)V, Uh(t), loU0, pbuf, st);
                launch_axpy((long long)V, 1.0 / (double)ctx->g.N3, pbuf, lamU, st);
                launch_join((long long)V, Bh(t), loB0, pbuf, st);
                launch_axpy((long long)V, 1.0 / (double)ctx->g.N3, pbuf, lamB, st);
                ctx->launches += 4;
            }
        }
    }
    CK(cudaMemcpyAsync(gradU->d64, lamU, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(gradB->d64, lamB, sizeof(double) * V, cudaMemcpyDeviceToDevice, st));
    int perr = 0;
    CK(cudaMemcpyAsync(&perr, ctx->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (perr) return fail(ctx, NOVA_E_TIMEOUT, "nova_adjoint_grad: a stage kernel pipeline wait timed out");
    const double E = row[2] + (etot ? row[3] : 0.0);
    const double J = window ? (row[NOVA_HIST_COLS + 2] + row[NOVA_HIST_COLS + 3]) - E : E;
    if (objective) *objective = J;
    if (!std::isfinite(J)) return fail(ctx, NOVA_E_NONFINITE, "nova_adjoint_grad: non-finite objective");
    return NOVA_OK;
}

}  // namespace

// ======================================================= implicit operators ==
// fdMatrix<scalar> of src/im (kernels in nova_im.cu): coef = [al0..al5 | ap | b]
struct nova_fdm {
    nova_ctx *ctx = nullptr;
    nova_field *x = nullptr;     // the transported field (not owned)
    double *coef = nullptr;      // 8 x N3
    double *scratch = nullptr;   // the solve's second x buffer (N3)
    double *fac = nullptr;       // line factors along i, j, k: 3 x 4 N3, then the per-line scalars
    bool factored = false;       // fac matches the coefficients (the source does not enter it)
};

namespace {

nova_status fdm_check(nova_ctx *ctx, const nova_fdm *a, const char *what)
{
    if (!ctx || !a || a->ctx != ctx || !a->coef) return fail(ctx, NOVA_E_INVALID, what);
    return NOVA_OK;
}

bool fdm_mesh_ok(const nova_ctx *ctx) { return !ctx->g.wallY && !ctx->md.hyperbolic_z; }

}  // namespace

extern "C" nova_status nova_im_laplacian(nova_ctx *ctx, double mu, nova_field *x, nova_fdm **out)
{
    if (!ctx || !x || !out) return fail(ctx, NOVA_E_INVALID, "nova_im_laplacian: null argument");
    *out = nullptr;
    if (!valid_field(ctx, x, 1) || x->prec != NOVA_F64)
        return fail(ctx, NOVA_E_INVALID, "nova_im_laplacian: x must be an FP64 scalar field");
    if (!fdm_mesh_ok(ctx)) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_im_laplacian: periodic uniform meshes only");
    const Geo &g = ctx->g;
    if (g.N0 < 3 || g.N1 < 3 || g.N2 < 3)
        return fail(ctx, NOVA_E_UNSUPPORTED, "nova_im_laplacian: at least 3 nodes per direction");
    nova_fdm *a = new (std::nothrow) nova_fdm;
    if (!a) return fail(ctx, NOVA_E_OOM, "nova_im_laplacian: out of host memory");
    a->ctx = ctx;
    a->x = x;
    nova_status s = dalloc(ctx, &a->coef, 8 * (size_t)g.N3);
    if (s != NOVA_OK) {
        delete a;
        return s;
    }
    const double dx = ctx->md.L[0] / ctx->md.N[0], dy = ctx->md.L[1] / ctx->md.N[1],
                 dz = ctx->md.L[2] / ctx->md.N[2];
    // the deferred correction's ex::laplacian goes through the source slot (read, then overwritten per node)
    launch_fdm_laplacian(g, ctx->co64, ctx->d_ia64, ctx->d_corr64, ctx->h, mu, dx, dy, dz, x->d64,
                         a->coef + 7 * (size_t)g.N3, a->coef, ctx->stream);
    ctx->launches += 3;
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(a->coef);
        delete a;
        return cuda_check(ctx, e, "nova_im_laplacian");
    }
    *out = a;
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_add(nova_ctx *ctx, nova_fdm *a, double alpha, const nova_fdm *b)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_add: bad matrix")) != NOVA_OK) return s;
    if ((s = fdm_check(ctx, b, "nova_fdm_add: bad matrix")) != NOVA_OK) return s;
    a->factored = false;
    launch_fdm_algebra(ctx->g, 0, alpha, a->coef, b->coef, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_mul(nova_ctx *ctx, nova_fdm *a, const nova_fdm *b)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_mul: bad matrix")) != NOVA_OK) return s;
    if ((s = fdm_check(ctx, b, "nova_fdm_mul: bad matrix")) != NOVA_OK) return s;
    a->factored = false;
    launch_fdm_algebra(ctx->g, 1, 0.0, a->coef, b->coef, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_scale(nova_ctx *ctx, nova_fdm *a, double sc)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_scale: bad matrix")) != NOVA_OK) return s;
    a->factored = false;
    launch_fdm_algebra(ctx->g, 2, sc, a->coef, nullptr, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_add_source(nova_ctx *ctx, nova_fdm *a, double alpha, const nova_field *f)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_add_source: bad matrix")) != NOVA_OK) return s;
    if (!valid_field(ctx, f, 1) || f->prec != NOVA_F64)
        return fail(ctx, NOVA_E_INVALID, "nova_fdm_add_source: f must be an FP64 scalar field");
    launch_fdm_point(ctx->g, 0, alpha, a->coef, f->d64, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_add_diagonal(nova_ctx *ctx, nova_fdm *a, double d)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_add_diagonal: bad matrix")) != NOVA_OK) return s;
    a->factored = false;
    launch_fdm_point(ctx->g, 1, d, a->coef, nullptr, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_relax(nova_ctx *ctx, nova_fdm *a, double urf)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_relax: bad matrix")) != NOVA_OK) return s;
    if (!(urf > 0.0)) return fail(ctx, NOVA_E_INVALID, "nova_fdm_relax: urf must be positive");
    a->factored = false;
    launch_fdm_point(ctx->g, 2, urf, a->coef, a->x->d64, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_set_reference(nova_ctx *ctx, nova_fdm *a, int i, int j, int k, double val)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_set_reference: bad matrix")) != NOVA_OK) return s;
    const Geo &g = ctx->g;
    if (i < 0 || i >= g.N0 || j < 0 || j >= g.N1 || k < 0 || k >= g.N2)
        return fail(ctx, NOVA_E_INVALID, "nova_fdm_set_reference: node outside the mesh");
    a->factored = false;
    launch_fdm_setref(g, a->coef, ((long long)i * g.N1 + j) * g.N2 + k, val, ctx->stream);
    ctx->launches += 1;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

namespace {

nova_status fdm_res(nova_ctx *ctx, const nova_fdm *a, const double *x, double *res)
{
    nova_status s = ensure_red(ctx);
    if (s != NOVA_OK) return s;
    const int nb = 592;  // 4 blocks per SM (k_fdm_res launch bounds); <= the partials reserved (diag_blocks(g) * 4)
    launch_fdm_residual(ctx->g, a->coef, x, ctx->d_part, nb, ctx->d_scalar, ctx->stream);
    ctx->launches += 2;
    CK(cudaMemcpyAsync(res, ctx->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

}  // namespace

extern "C" nova_status nova_fdm_residual(nova_ctx *ctx, const nova_fdm *a, double *res)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_residual: bad matrix")) != NOVA_OK) return s;
    if (!res) return fail(ctx, NOVA_E_INVALID, "nova_fdm_residual: null argument");
    return fdm_res(ctx, a, a->x->d64, res);
}

extern "C" nova_status nova_fdm_solve(nova_ctx *ctx, nova_fdm *a, double tol, int max_its, int *its, double *res)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_solve: bad matrix")) != NOVA_OK) return s;
    if (max_its < 0) return fail(ctx, NOVA_E_INVALID, "nova_fdm_solve: max_its must not be negative");
    if (max_its == 0) {  // no iteration: only the residual of x, and nothing to allocate
        double r = 0.0;
        if ((s = fdm_res(ctx, a, a->x->d64, &r)) != NOVA_OK) return s;
        if (its) *its = 0;
        if (res) *res = r;
        return NOVA_OK;
    }
    const Geo &g = ctx->g;
    if ((s = dalloc(ctx, &a->scratch, (size_t)g.N3)) != NOVA_OK) return s;
    // factors of the three line directions (4 N3 each) and their per-line scalars (2 per line)
    const size_t lines[3] = {(size_t)g.N1 * g.N2, (size_t)g.N0 * g.N2, (size_t)g.N0 * g.N1};
    if ((s = dalloc(ctx, &a->fac, 12 * (size_t)g.N3 + 2 * (lines[0] + lines[1] + lines[2]))) != NOVA_OK) return s;
    double *fac[3], *ls[3];
    {
        double *q = a->fac + 12 * (size_t)g.N3;
        for (int ax = 0; ax < 3; ax++) {
            fac[ax] = a->fac + 4 * (size_t)ax * g.N3;
            ls[ax] = q;
            q += 2 * lines[ax];
        }
    }
    if (!a->factored) {
        for (int ax = 0; ax < 3; ax++) launch_fdm_factor(ax, g, a->coef, fac[ax], ls[ax], ctx->stream);
        ctx->launches += 3;
        CKL("k_fdm_factor");
        a->factored = true;
    }
    // x and the second buffer swap roles every sweep; cur holds the iterate
    double *cur = a->x->d64, *other = a->scratch;
    double r = 0.0;
    int n = 0;
    while (n < max_its) {
        // the residual checked before each iteration, as the reference reports it
        if ((s = fdm_res(ctx, a, cur, &r)) != NOVA_OK) return s;
        if (!(r > tol)) break;
        n++;
        for (const int ax : {1, 0, 2}) {  // j lines, i lines, k lines
            launch_fdm_line(ax, g, a->coef, fac[ax], ls[ax], cur, other, ctx->stream);
            std::swap(cur, other);
        }
        ctx->launches += 3;
        CKL("k_fdm_line");
    }
    if (cur != a->x->d64) {
        CK(cudaMemcpyAsync(a->x->d64, cur, sizeof(double) * g.N3, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (its) *its = n;
    if (res) *res = r;
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_download(nova_ctx *ctx, const nova_fdm *a, double *host)
{
    nova_status s;
    if ((s = fdm_check(ctx, a, "nova_fdm_download: bad matrix")) != NOVA_OK) return s;
    if (!host) return fail(ctx, NOVA_E_INVALID, "nova_fdm_download: null argument");
    CK(cudaMemcpyAsync(host, a->coef, sizeof(double) * 8 * ctx->g.N3, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

extern "C" nova_status nova_fdm_destroy(nova_fdm *a)
{
    if (!a) return NOVA_OK;
    if (a->coef) cudaFree(a->coef);
    if (a->scratch) cudaFree(a->scratch);
    if (a->fac) cudaFree(a->fac);
    delete a;
    return NOVA_OK;
}

// ========================================================= weakly compressible ==
extern "C" nova_status nova_advance_wc(nova_ctx *ctx, const nova_wc_desc *wd, nova_wc_state *st, int nsteps,
                                       double *hist)
{
    if (!ctx || !wd || !st || nsteps < 0) return fail(ctx, NOVA_E_INVALID, "nova_advance_wc: bad arguments");
    const bool shear = wd->wc_case == NOVA_WC_SHEAR;
    if (wd->wc_case != NOVA_WC_TG && !shear) return fail(ctx, NOVA_E_INVALID, "nova_advance_wc: unknown case");
    auto f64 = [ctx](const nova_field *f, int nc) { return valid_field(ctx, f, nc) && f->prec == NOVA_F64; };
    if (!f64(st->U, 3) || !f64(st->rho, 1) || !f64(st->p, 1) || (shear && !f64(st->T, 1)))
        return fail(ctx, NOVA_E_INVALID, "nova_advance_wc: U, rho, p (and T for the shear case) must be FP64 fields");
    if (ctx->g.wallY) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_advance_wc: periodic meshes only");
    if (ctx->h != 3) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_advance_wc: the fused kernels are built for m = 6");
    nova_status s = ensure_work(ctx, NOVA_F64);
    if (s != NOVA_OK) return s;
    if (hist && wd->diag_every > 0) {
        if (ctx->hist_cap < (long long)nsteps * NOVA_HIST_COLS) {
            if (ctx->d_hist) cudaFree(ctx->d_hist);
            ctx->d_hist = nullptr;
            ctx->hist_cap = 0;
            if ((s = dalloc(ctx, &ctx->d_hist, (size_t)nsteps * NOVA_HIST_COLS)) != NOVA_OK) return s;
            ctx->hist_cap = (long long)nsteps * NOVA_HIST_COLS;
        }
        CK(cudaMemsetAsync(ctx->d_hist, 0, sizeof(double) * nsteps * NOVA_HIST_COLS, ctx->stream));
    }
    CK(cudaMemsetAsync(ctx->d_flag, 0, 2 * sizeof(int), ctx->stream));
    const Geo &g = ctx->g;
    const bool str = ctx->md.hyperbolic_z != 0;
    double *w0 = ctx->w64[0], *w1 = ctx->w64[1], *acc = ctx->w64[2];
    // one RK loop of the quantity q (stored in qf): stage states alternate w0/w1, the last stage writes qf
    auto loop = [&](int which, double *qf, double visc) {
        WcArgs a{};
        a.U = st->U->d64;
        a.rho = st->rho->d64;
        a.T = st->T ? st->T->d64 : nullptr;
        a.p = st->p->d64;
        a.Q0 = qf;
        a.acc = acc;
        a.dt = wd->dt;
        a.visc = visc;
        a.eos_k = wd->eos_k;
        for (int c = 0; c < 3; c++) a.g[c] = wd->g[c];
        const double *ys[4] = {qf, w0, w1, w0};
        double *yn[4] = {w0, w1, w0, qf};
        for (int stage = 0; stage < 4; stage++) {
            ProfScope ps(ctx, NOVA_K_STAGE);
            a.Y = ys[stage];
            a.Ynext = yn[stage];
            launch_wc_stage(which, stage, wd->wc_case, str, g, ctx->co64, ctx->d_ia64, ctx->d_corr64, a, ctx->stream);
            ctx->launches += 1;
        }
    };
    for (int n = 0; n < nsteps; n++) {
        if (shear) {
            loop(WC_LOOP_U, st->U->d64, wd->mu);
            loop(WC_LOOP_RHO, st->rho->d64, 0.0);
            loop(WC_LOOP_T, st->T->d64, wd->ka);
        } else {
            loop(WC_LOOP_RHO, st->rho->d64, 0.0);
            loop(WC_LOOP_U, st->U->d64, wd->mu);
        }
        CKL("weakly-compressible stage kernels");
        if (hist && wd->diag_every > 0 && ((n + 1) % wd->diag_every == 0 || n + 1 == nsteps)) {
            ProfScope ps(ctx, NOVA_K_DIAG);
            launch_diag(ctx->h, g, Walls<double>{}, ctx->co64, ctx->d_ia64, st->U->d64, nullptr, nullptr, nullptr,
                        nullptr, nullptr, 0, ctx->d_part, (double)(n + 1), wd->t0 + (n + 1) * wd->dt,
                        ctx->d_hist + (long long)n * NOVA_HIST_COLS, ctx->d_flag, ctx->stream,
                        DiagPhys{wd->mu, 0.0, wd->dt, ctx->md.L[0] / ctx->md.N[0], ctx->md.L[1] / ctx->md.N[1],
                                 ctx->md.L[2] / ctx->md.N[2]});
            ctx->launches += 2;
            CKL("k_diag");
        }
    }
    if (hist && wd->diag_every > 0)
        CK(cudaMemcpyAsync(hist, ctx->d_hist, sizeof(double) * nsteps * NOVA_HIST_COLS, cudaMemcpyDeviceToHost,
                           ctx->stream));
    int flag[2] = {0, 0};
    CK(cudaMemcpyAsync(flag, ctx->d_flag, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (flag[0]) return fail(ctx, NOVA_E_NONFINITE, "nova_advance_wc: non-finite value in the diagnostics");
    return NOVA_OK;
}

extern "C" nova_status nova_wc_hydrostatic(nova_ctx *ctx, const nova_wc_desc *wd, double rho0, const nova_field *T,
                                           nova_field *p, nova_field *rho)
{
    if (!ctx || !wd || !T || !p || !rho) return fail(ctx, NOVA_E_INVALID, "nova_wc_hydrostatic: null argument");
    auto f64 = [ctx](const nova_field *f) { return valid_field(ctx, f, 1) && f->prec == NOVA_F64; };
    if (!f64(T) || !f64(p) || !f64(rho))
        return fail(ctx, NOVA_E_INVALID, "nova_wc_hydrostatic: T, p, rho must be FP64 scalar fields");
    if (ctx->g.wallY) return fail(ctx, NOVA_E_UNSUPPORTED, "nova_wc_hydrostatic: periodic meshes only");
    if (!(wd->eos_k > 0.0)) return fail(ctx, NOVA_E_INVALID, "nova_wc_hydrostatic: eos_k must be positive");
    launch_wc_hydrostatic(ctx->g, ctx->md.L[2] / ctx->md.N[2], wd->g[2], rho0, wd->eos_k, T->d64, p->d64, rho->d64,
                          ctx->stream);
    ctx->launches += 1;
    CKL("k_wc_hydrostatic");
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

// =============================================================== checkpoints ==
namespace {

const char kCkptMagic[8] = {'N', 'O', 'V', 'A', 'C', 'K', 'P', '1'};

struct CkptFile {
    std::FILE *fp = nullptr;
    bool ok = true;
    ~CkptFile()
    {
        if (fp) std::fclose(fp);
    }
    void put(const void *p, size_t n) { ok = ok && std::fwrite(p, 1, n, fp) == n; }
    void get(void *p, size_t n) { ok = ok && std::fread(p, 1, n, fp) == n; }
};

struct CkptMesh {
    int32_t N[3], m, walls[3], hyperbolic_z;
    double L[3], origin[3], s1, s2;
};

CkptMesh ckpt_mesh(const nova_mesh_desc &md)
{
    CkptMesh c{};
    for (int a = 0; a < 3; a++) {
        c.N[a] = md.N[a];
        c.walls[a] = md.walls[a];
        c.L[a] = md.L[a];
        c.origin[a] = md.origin[a];
    }
    c.m = md.m;
    c.hyperbolic_z = md.hyperbolic_z;
    c.s1 = md.hyperbolic_z ? md.s1 : 0.0;
    c.s2 = md.hyperbolic_z ? md.s2 : 0.0;
    return c;
}

void put_mesh(CkptFile &f, const CkptMesh &c)
{
    f.put(c.N, sizeof c.N), f.put(&c.m, 4), f.put(c.walls, sizeof c.walls), f.put(&c.hyperbolic_z, 4);
    f.put(c.L, sizeof c.L), f.put(c.origin, sizeof c.origin), f.put(&c.s1, 8), f.put(&c.s2, 8);
}

void get_mesh(CkptFile &f, CkptMesh &c)
{
    f.get(c.N, sizeof c.N), f.get(&c.m, 4), f.get(c.walls, sizeof c.walls), f.get(&c.hyperbolic_z, 4);
    f.get(c.L, sizeof c.L), f.get(c.origin, sizeof c.origin), f.get(&c.s1, 8), f.get(&c.s2, 8);
}

bool same_mesh(const CkptMesh &a, const CkptMesh &b)
{
    bool same = a.m == b.m && a.hyperbolic_z == b.hyperbolic_z && a.s1 == b.s1 && a.s2 == b.s2;
    for (int d = 0; d < 3; d++)
        same = same && a.N[d] == b.N[d] && a.walls[d] == b.walls[d] && a.L[d] == b.L[d] && a.origin[d] == b.origin[d];
    return same;
}

const int kCkptComps[4] = {3, 1, 3, 1};  // U, p, B, pB

}  // namespace

extern "C" nova_status nova_checkpoint_write(nova_ctx *ctx, const char *path, const nova_state *st, double t,
                                             long long step)
{
    if (!ctx || !path || !st) return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_write: null argument");
    const nova_field *fs[4] = {st->U, st->p, st->B, st->pB};
    int32_t nf = 0;
    for (int q = 0; q < 4; q++) {
        if (!fs[q]) continue;
        if (!valid_field(ctx, fs[q], kCkptComps[q]))
            return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_write: state field " + std::to_string(q) +
                                                 " has the wrong component count");
        nf++;
    }
    CkptFile f;
    f.fp = std::fopen(path, "wb");
    if (!f.fp) return fail(ctx, NOVA_E_INVALID, std::string("nova_checkpoint_write: cannot open ") + path);
    f.put(kCkptMagic, 8);
    put_mesh(f, ckpt_mesh(ctx->md));
    const int64_t st64 = step;
    const int32_t zero = 0;
    f.put(&t, 8), f.put(&st64, 8), f.put(&nf, 4), f.put(&zero, 4);
    std::vector<double> host;
    for (int q = 0; q < 4 && f.ok; q++) {
        const nova_field *fl = fs[q];
        if (!fl) continue;
        const int32_t hdr[4] = {q, fl->nc, fl->prec, 0};
        f.put(hdr, sizeof hdr);
        int32_t types[18];
        for (int i = 0; i < 18; i++) types[i] = fl->bc.type[i];
        f.put(types, sizeof types), f.put(fl->bc.val, sizeof fl->bc.val);
        host.resize((size_t)fl->nc * ctx->g.N3);
        nova_status s = soa_out(ctx, fl, host.data(), cudaMemcpyDeviceToHost);
        if (s != NOVA_OK) return s;
        CK(cudaStreamSynchronize(ctx->stream));
        f.put(host.data(), sizeof(double) * host.size());
    }
    const bool closed = std::fclose(f.fp) == 0;
    f.fp = nullptr;
    if (!f.ok || !closed) return fail(ctx, NOVA_E_INVALID, std::string("nova_checkpoint_write: write failed: ") + path);
    return NOVA_OK;
}

extern "C" nova_status nova_checkpoint_read(nova_ctx *ctx, const char *path, nova_state *st, double *t,
                                            long long *step)
{
    if (!ctx || !path || !st) return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_read: null argument");
    nova_field *fs[4] = {st->U, st->p, st->B, st->pB};
    for (int q = 0; q < 4; q++)
        if (fs[q] && !valid_field(ctx, fs[q], kCkptComps[q]))
            return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_read: state field " + std::to_string(q) +
                                                 " has the wrong component count");
    CkptFile f;
    f.fp = std::fopen(path, "rb");
    if (!f.fp) return fail(ctx, NOVA_E_INVALID, std::string("nova_checkpoint_read: cannot open ") + path);
    char magic[8];
    f.get(magic, 8);
    if (!f.ok || std::memcmp(magic, kCkptMagic, 8) != 0)
        return fail(ctx, NOVA_E_INVALID, std::string("nova_checkpoint_read: not a checkpoint file: ") + path);
    CkptMesh cm{};
    get_mesh(f, cm);
    if (!f.ok || !same_mesh(cm, ckpt_mesh(ctx->md)))
        return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_read: the file holds another mesh");
    double tt = 0.0;
    int64_t st64 = 0;
    int32_t nf = 0, reserved = 0;
    f.get(&tt, 8), f.get(&st64, 8), f.get(&nf, 4), f.get(&reserved, 4);
    if (!f.ok || nf < 0 || nf > 4) return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_read: corrupt header");
    std::vector<double> host;
    for (int i = 0; i < nf; i++) {
        int32_t hdr[4];
        f.get(hdr, sizeof hdr);
        if (!f.ok || hdr[0] < 0 || hdr[0] > 3 || hdr[1] != kCkptComps[hdr[0]])
            return fail(ctx, NOVA_E_INVALID, "nova_checkpoint_read: corrupt field record");
        int32_t types[18];
        nova_bc bc;
        f.get(types, sizeof types), f.get(bc.val, sizeof bc.val);
        for (int k = 0; k < 18; k++) bc.type[k] = types[k];
        host.resize((size_t)hdr[1] * ctx->g.N3);
        f.get(host.data(), sizeof(double) * host.size());
        if (!f.ok) return fail(ctx, NOVA_E_INVALID, std::string("nova_checkpoint_read: truncated file: ") + path);
        nova_field *fl = fs[hdr[0]];
        if (!fl) continue;
        nova_status s = nova_field_set_bc(ctx, fl, &bc);
        if (s != NOVA_OK) return s;
        if ((s = soa_in(ctx, fl, host.data(), cudaMemcpyHostToDevice)) != NOVA_OK) return s;
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (t) *t = tt;
    if (step) *step = st64;
    return NOVA_OK;
}

// =================================================================== EnSight ==
extern "C" nova_status nova_ensight_write_field(nova_ctx *ctx, const nova_field *f, const char *dir, const char *name,
                                                int num)
{
    if (!ctx || !f || !dir || !name) return fail(ctx, NOVA_E_INVALID, "nova_ensight_write_field: null argument");
    std::vector<double> host((size_t)f->nc * ctx->g.N3);
    nova_status s = soa_out(ctx, f, host.data(), cudaMemcpyDeviceToHost);
    if (s != NOVA_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream));
    if (nova_ensight_write_host(&ctx->md, host.data(), f->nc, dir, name, num) != NOVA_OK)
        return fail(ctx, NOVA_E_INVALID, std::string("nova_ensight_write_field: cannot write ") + dir + "/" + name);
    return NOVA_OK;
}

extern "C" nova_status nova_ensight_read_field(nova_ctx *ctx, nova_field *f, const char *dir, const char *name, int num)
{
    if (!ctx || !f || !dir || !name) return fail(ctx, NOVA_E_INVALID, "nova_ensight_read_field: null argument");
    std::vector<double> host((size_t)f->nc * ctx->g.N3);
    if (nova_ensight_read_host(&ctx->md, host.data(), f->nc, dir, name, num) != NOVA_OK)
        return fail(ctx, NOVA_E_INVALID, std::string("nova_ensight_read_field: cannot read ") + dir + "/" + name);
    nova_status s = soa_in(ctx, f, host.data(), cudaMemcpyHostToDevice);
    if (s != NOVA_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream));
    return NOVA_OK;
}

// ========================================================== instrumentation ==
extern "C" nova_status nova_profile_enable(nova_ctx *ctx, int on)
{
    if (!ctx) return NOVA_E_INVALID;
    prof_collect(ctx);
    ctx->prof = on != 0;
    return NOVA_OK;
}

extern "C" nova_status nova_profile_read(nova_ctx *ctx, int cls, double *total_ms, long *launches, int reset)
{
    if (!ctx || cls < 0 || cls >= NOVA_K_COUNT) return NOVA_E_INVALID;
    prof_collect(ctx);
    if (total_ms) *total_ms = ctx->prof_ms[cls];
    if (launches) *launches = ctx->prof_n[cls];
    if (reset) {
        ctx->prof_ms[cls] = 0.0;
        ctx->prof_n[cls] = 0;
    }
    return NOVA_OK;
}

extern "C" nova_status nova_launch_count(nova_ctx *ctx, long *launches, int reset)
{
    if (!ctx || !launches) return NOVA_E_INVALID;
    *launches = ctx->launches;
    if (reset) ctx->launches = 0;
    return NOVA_OK;
}
