// The implicit operators of src/im on the GPU: fdMatrix<scalar>
// (src/im/fdMatrix/fdMatrix.h:33-77, fdMatrix.hxx) as eight per-node FP64
// fields, coef = [al0..al5 | ap | b], the coefficients of the neighbours
// j+1, j-1, i+1, i-1, k+1, k-1 (N, S, E, W, T, B), the centre and the source,
// over the unique nodes of a periodic mesh; (A x)_n = ap x_n + sum_l al_l x_{n+l}.
//
//   im::laplacian (src/im/laplacian/laplacian.hxx:24-58): al = mu/d^2,
//     ap = -2 mu sum 1/d^2, b = -ex::laplacian(mu, x) + A x (the deferred
//     correction, fdMatrix.hxx:201-225, summed in the reference's order);
//   residual (fdMatrix.hxx:249-290): RMS of b - A x over the nodes the
//     reference counts, (N0+1)(N1+1)(N2+1) with the duplicate periodic nodes;
//   solve (fdMatrix.hxx:59-198): line sweeps along j, i, k per iteration.
//     The reference sweeps the lines of a direction one after another
//     (Gauss-Seidel across lines) and holds the duplicate node of each line
//     at its value from the last ghost refresh; here every line of a sweep is
//     solved at once, the neighbours off the line taken at the sweep's start,
//     as an exactly periodic tridiagonal system (Thomas' algorithm with the
//     Sherman-Morrison correction for the two corner entries).  Both are
//     iterations with the same fixed point, A x = b with periodic wrap.
#include "nova_internal.cuh"
#include "nova_ops.cuh"

namespace nova {

namespace {

__device__ __forceinline__ long long nidx(const Geo &g, int i, int j, int k)
{
    return ((long long)i * g.N1 + j) * g.N2 + k;
}

__global__ void k_fdm_fill(Geo g, double *coef, double cx, double cy, double cz, double apv)
{
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.N3) return;
    coef[0 * g.N3 + n] = cy;
    coef[1 * g.N3 + n] = cy;
    coef[2 * g.N3 + n] = cx;
    coef[3 * g.N3 + n] = cx;
    coef[4 * g.N3 + n] = cz;
    coef[5 * g.N3 + n] = cz;
    coef[6 * g.N3 + n] = apv;
}

// b = -hoa + al0 x(j+1) + al1 x(j-1) + al2 x(i+1) + al3 x(i-1) + al4 x(k+1) + al5 x(k-1) + ap x
__global__ void k_fdm_defcorr(Geo g, double *coef, const double *__restrict__ hoa, const double *__restrict__ x)
{
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.N3) return;
    const int k = (int)(n % g.N2), j = (int)((n / g.N2) % g.N1), i = (int)(n / g.N12);
    const long long N3 = g.N3;
    const double *al = coef;
    // unfused products and sums, as the reference evaluates the expression
    double v = -hoa[n];
    v = __dadd_rn(v, __dmul_rn(al[0 * N3 + n], x[nidx(g, i, wrapi(j + 1, g.N1), k)]));
    v = __dadd_rn(v, __dmul_rn(al[1 * N3 + n], x[nidx(g, i, wrapi(j - 1, g.N1), k)]));
    v = __dadd_rn(v, __dmul_rn(al[2 * N3 + n], x[nidx(g, wrapi(i + 1, g.N0), j, k)]));
    v = __dadd_rn(v, __dmul_rn(al[3 * N3 + n], x[nidx(g, wrapi(i - 1, g.N0), j, k)]));
    v = __dadd_rn(v, __dmul_rn(al[4 * N3 + n], x[nidx(g, i, j, wrapi(k + 1, g.N2))]));
    v = __dadd_rn(v, __dmul_rn(al[5 * N3 + n], x[nidx(g, i, j, wrapi(k - 1, g.N2))]));
    v = __dadd_rn(v, __dmul_rn(al[6 * N3 + n], x[n]));
    coef[7 * N3 + n] = __dadd_rn(0.0, v);  // the source starts at zero (fdMatrix.hxx:40-43)
}

// a = a + alpha b (mode 0), a = a * b (mode 1), a = s a (mode 2) over all eight fields
__global__ void k_fdm_axpy(long long n8, int mode, double alpha, double *a, const double *__restrict__ b)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n8) return;
    if (mode == 0)
        a[t] = a[t] + alpha * b[t];
    else if (mode == 1)
        a[t] = a[t] * b[t];
    else
        a[t] = a[t] * alpha;
}

// b += alpha f (mode 0), ap += d (mode 1), relax: b += (1-urf)/urf ap x, ap /= urf (mode 2)
__global__ void k_fdm_point(Geo g, int mode, double v, double *coef, const double *__restrict__ f)
{
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.N3) return;
    double *ap = coef + 6 * g.N3, *b = coef + 7 * g.N3;
    if (mode == 0) {
        b[n] = b[n] + v * f[n];
    } else if (mode == 1) {
        ap[n] = ap[n] + v;
    } else {
        b[n] = b[n] + (1.0 - v) / v * (ap[n] * f[n]);
        ap[n] = ap[n] / v;
    }
}

__global__ void k_fdm_setref(double *ap, double *b, long long n, double val)
{
    b[n] = b[n] + 1e15 * val;
    ap[n] = ap[n] * 1e15;
}

// partial sums of (b - A x)^2 over the (N0+1)(N1+1)(N2+1) nodes (indices wrap)
__global__ void k_fdm_res(Geo g, const double *__restrict__ coef, const double *__restrict__ x, double *part)
{
    __shared__ double sh[32];
    const long long tot = (long long)(g.N0 + 1) * (g.N1 + 1) * (g.N2 + 1);
    const long long N3 = g.N3;
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % (g.N2 + 1)) % g.N2, j = (int)((t / (g.N2 + 1)) % (g.N1 + 1)) % g.N1;
        const int i = (int)(t / ((long long)(g.N1 + 1) * (g.N2 + 1))) % g.N0;
        const long long n = nidx(g, i, j, k);
        double r = coef[7 * N3 + n];
        r = __dsub_rn(r, __dmul_rn(coef[0 * N3 + n], x[nidx(g, i, wrapi(j + 1, g.N1), k)]));
        r = __dsub_rn(r, __dmul_rn(coef[1 * N3 + n], x[nidx(g, i, wrapi(j - 1, g.N1), k)]));
        r = __dsub_rn(r, __dmul_rn(coef[2 * N3 + n], x[nidx(g, wrapi(i + 1, g.N0), j, k)]));
        r = __dsub_rn(r, __dmul_rn(coef[3 * N3 + n], x[nidx(g, wrapi(i - 1, g.N0), j, k)]));
        r = __dsub_rn(r, __dmul_rn(coef[4 * N3 + n], x[nidx(g, i, j, wrapi(k + 1, g.N2))]));
        r = __dsub_rn(r, __dmul_rn(coef[5 * N3 + n], x[nidx(g, i, j, wrapi(k - 1, g.N2))]));
        r = __dsub_rn(r, __dmul_rn(coef[6 * N3 + n], x[n]));
        acc = __dadd_rn(acc, __dmul_rn(r, r));
    }
    acc = block_reduce_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void k_fdm_res_final(const double *__restrict__ part, int nb, double count, double *out)
{
    __shared__ double sh[32];
    double a = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) a += part[q];
    a = block_reduce_sum(a, sh);
    if (threadIdx.x == 0) out[0] = sqrt(a / count);
}

// One line per thread along AXIS (0: i, 1: j, 2: k): a_t x_{t-1} + b_t x_t +
// c_t x_{t+1} = d_t with periodic wrap, the off-line neighbours from xin.
// Scratch: cp, yv, zv (one element per node of the line).
template <int AXIS>
__global__ void k_fdm_sweep(Geo g, const double *__restrict__ coef, const double *__restrict__ xin, double *xout,
                            double *cp, double *yv, double *zv)
{
    const long long N3 = g.N3;
    const int n = AXIS == 0 ? g.N0 : (AXIS == 1 ? g.N1 : g.N2);
    const long long lines = N3 / n;
    const long long line = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (line >= lines) return;
    // the line's fixed indices: i-lines by (j, k), j-lines by (i, k), k-lines by (i, j), the fastest last
    int i0 = 0, j0 = 0, k0 = 0;
    if (AXIS == 0) {
        j0 = (int)(line / g.N2);
        k0 = (int)(line % g.N2);
    } else if (AXIS == 1) {
        i0 = (int)(line / g.N2);
        k0 = (int)(line % g.N2);
    } else {
        i0 = (int)(line / g.N1);
        j0 = (int)(line % g.N1);
    }
    auto node = [&](int t) -> long long {
        return AXIS == 0 ? nidx(g, t, j0, k0) : (AXIS == 1 ? nidx(g, i0, t, k0) : nidx(g, i0, j0, t));
    };
    // sub/super-diagonal coefficients and the off-line neighbours (fdMatrix.hxx:99-108, 134-143, 169-178)
    constexpr int LO = AXIS == 0 ? 3 : (AXIS == 1 ? 1 : 5), HI = AXIS == 0 ? 2 : (AXIS == 1 ? 0 : 4);
    auto rhs = [&](int t, long long o) -> double {
        const int i = AXIS == 0 ? t : i0, j = AXIS == 1 ? t : j0, k = AXIS == 2 ? t : k0;
        double d = coef[7 * N3 + o];
        if (AXIS != 1) {
            d = d - coef[0 * N3 + o] * xin[nidx(g, i, wrapi(j + 1, g.N1), k)];
            d = d - coef[1 * N3 + o] * xin[nidx(g, i, wrapi(j - 1, g.N1), k)];
        }
        if (AXIS != 0) {
            d = d - coef[2 * N3 + o] * xin[nidx(g, wrapi(i + 1, g.N0), j, k)];
            d = d - coef[3 * N3 + o] * xin[nidx(g, wrapi(i - 1, g.N0), j, k)];
        }
        if (AXIS != 2) {
            d = d - coef[4 * N3 + o] * xin[nidx(g, i, j, wrapi(k + 1, g.N2))];
            d = d - coef[5 * N3 + o] * xin[nidx(g, i, j, wrapi(k - 1, g.N2))];
        }
        return d;
    };
    // Sherman-Morrison: T' = T - u v^T with the corners folded into the
    // diagonal, gamma = -b_0, u = (gamma, 0.., c_{n-1}), v = (1, 0.., a_0/gamma)
    const long long o0 = node(0), on = node(n - 1);
    const double a0 = coef[LO * N3 + o0], cn = coef[HI * N3 + on];
    const double gam = -coef[6 * N3 + o0];
    double cprev = 0.0, yprev = 0.0, zprev = 0.0;
    for (int t = 0; t < n; t++) {
        const long long o = node(t);
        const double a = t == 0 ? 0.0 : coef[LO * N3 + o];
        const double c = t == n - 1 ? 0.0 : coef[HI * N3 + o];
        double b = coef[6 * N3 + o];
        if (t == 0) b -= gam;
        if (t == n - 1) b -= cn * a0 / gam;
        const double u = t == 0 ? gam : (t == n - 1 ? cn : 0.0);
        const double den = b - a * cprev;
        const double cc = c / den;
        const double yy = (rhs(t, o) - a * yprev) / den;
        const double zz = (u - a * zprev) / den;
        cp[o] = cc;
        yv[o] = yy;
        zv[o] = zz;
        cprev = cc;
        yprev = yy;
        zprev = zz;
    }
    // back substitution (y and z), then x = y - z (v.y)/(1 + v.z)
    double ynext = 0.0, znext = 0.0, y0 = 0.0, z0 = 0.0, yn = 0.0, zn = 0.0;
    for (int t = n - 1; t >= 0; t--) {
        const long long o = node(t);
        const double yy = t == n - 1 ? yv[o] : yv[o] - cp[o] * ynext;
        const double zz = t == n - 1 ? zv[o] : zv[o] - cp[o] * znext;
        yv[o] = yy;
        zv[o] = zz;
        ynext = yy;
        znext = zz;
        if (t == n - 1) {
            yn = yy;
            zn = zz;
        }
        if (t == 0) {
            y0 = yy;
            z0 = zz;
        }
    }
    const double vy = y0 + a0 / gam * yn, vz = z0 + a0 / gam * zn;
    const double f = vy / (1.0 + vz);
    for (int t = 0; t < n; t++) {
        const long long o = node(t);
        xout[o] = yv[o] - f * zv[o];
    }
}

unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

void launch_fdm_laplacian(const Geo &g, const Coef<double> &co, const double *ia, const double *corr2, int h,
                          double mu, double dx, double dy, double dz, const double *x, double *hoa, double *coef,
                          cudaStream_t st)
{
    // mu / pow(d, 2) and -2 mu / dx^2 - 2 mu / dy^2 - 2 mu / dz^2 as laplacian.hxx:37-48 evaluates them
    const double cx = mu / (dx * dx), cy = mu / (dy * dy), cz = mu / (dz * dz);
    const double apv = -2.0 * mu / (dx * dx) - 2.0 * mu / (dy * dy) - 2.0 * mu / (dz * dz);
    k_fdm_fill<<<blocks_for(g.N3, 256), 256, 0, st>>>(g, coef, cx, cy, cz, apv);
    launch_op(OP_LAP, h, g, Walls<double>{}, Walls<double>{}, co, ia, corr2, x, nullptr, 1, mu, hoa, st);
    k_fdm_defcorr<<<blocks_for(g.N3, 256), 256, 0, st>>>(g, coef, hoa, x);
}

void launch_fdm_algebra(const Geo &g, int mode, double alpha, double *a, const double *b, cudaStream_t st)
{
    k_fdm_axpy<<<blocks_for(8 * g.N3, 256), 256, 0, st>>>(8 * g.N3, mode, alpha, a, b);
}

void launch_fdm_point(const Geo &g, int mode, double v, double *coef, const double *f, cudaStream_t st)
{
    k_fdm_point<<<blocks_for(g.N3, 256), 256, 0, st>>>(g, mode, v, coef, f);
}

void launch_fdm_setref(const Geo &g, double *coef, long long n, double val, cudaStream_t st)
{
    k_fdm_setref<<<1, 1, 0, st>>>(coef + 6 * g.N3, coef + 7 * g.N3, n, val);
}

void launch_fdm_residual(const Geo &g, const double *coef, const double *x, double *part, int nb, double *out,
                         cudaStream_t st)
{
    k_fdm_res<<<nb, 256, 0, st>>>(g, coef, x, part);
    const double count = (double)(g.N0 + 1) * (double)(g.N1 + 1) * (double)(g.N2 + 1);
    k_fdm_res_final<<<1, 256, 0, st>>>(part, nb, count, out);
}

void launch_fdm_sweep(int axis, const Geo &g, const double *coef, const double *xin, double *xout, double *scratch,
                      cudaStream_t st)
{
    double *cp = scratch, *yv = scratch + g.N3, *zv = scratch + 2 * g.N3;
    const int n = axis == 0 ? g.N0 : (axis == 1 ? g.N1 : g.N2);
    const unsigned nb = blocks_for(g.N3 / n, 128);
    if (axis == 0)
        k_fdm_sweep<0><<<nb, 128, 0, st>>>(g, coef, xin, xout, cp, yv, zv);
    else if (axis == 1)
        k_fdm_sweep<1><<<nb, 128, 0, st>>>(g, coef, xin, xout, cp, yv, zv);
    else
        k_fdm_sweep<2><<<nb, 128, 0, st>>>(g, coef, xin, xout, cp, yv, zv);
}

}  // namespace nova
