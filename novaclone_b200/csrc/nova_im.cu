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
//     (Gauss-Seidel across lines) and holds the ghost and duplicate end
//     nodes of each line at their values from the last ghost refresh; here
//     every line of a sweep is solved at once, the neighbours off the line
//     taken at the sweep's start, as an exactly periodic tridiagonal system
//     (Thomas' algorithm with the Sherman-Morrison correction for the two
//     corner entries).  Both are iterations with the same fixed point,
//     A x = b with periodic wrap.
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

// partial sums of (b - A x)^2 over the (N0+1)(N1+1)(N2+1) nodes the reference
// loops over: its duplicate periodic node N of each direction is node 0 here,
// so node 0 of a direction counts twice.  A block takes whole (i, j) rows, two
// at a time so that both rows' loads are in flight together, its threads
// along k.
__device__ __forceinline__ double fdm_res_node(const Geo &g, const double *__restrict__ coef,
                                               const double *__restrict__ x, int row, int k)
{
    const long long N3 = g.N3;
    const int i = row / g.N1, j = row - i * g.N1;
    const long long base = (long long)row * g.N2, n = base + k;
    double r = coef[7 * N3 + n];
    r = __dsub_rn(r, __dmul_rn(coef[0 * N3 + n], x[nidx(g, i, wrapi(j + 1, g.N1), k)]));
    r = __dsub_rn(r, __dmul_rn(coef[1 * N3 + n], x[nidx(g, i, wrapi(j - 1, g.N1), k)]));
    r = __dsub_rn(r, __dmul_rn(coef[2 * N3 + n], x[nidx(g, wrapi(i + 1, g.N0), j, k)]));
    r = __dsub_rn(r, __dmul_rn(coef[3 * N3 + n], x[nidx(g, wrapi(i - 1, g.N0), j, k)]));
    r = __dsub_rn(r, __dmul_rn(coef[4 * N3 + n], x[base + wrapi(k + 1, g.N2)]));
    r = __dsub_rn(r, __dmul_rn(coef[5 * N3 + n], x[base + wrapi(k - 1, g.N2)]));
    r = __dsub_rn(r, __dmul_rn(coef[6 * N3 + n], x[n]));
    const double w = (i == 0 ? 2.0 : 1.0) * (j == 0 ? 2.0 : 1.0) * (k == 0 ? 2.0 : 1.0);
    return __dmul_rn(w, __dmul_rn(r, r));
}

__global__ void __launch_bounds__(256, 4) k_fdm_res(Geo g, const double *__restrict__ coef,
                                                    const double *__restrict__ x, double *part)
{
    __shared__ double sh[32];
    const int rows = g.N0 * g.N1;
    double acc = 0.0;
    for (int row = blockIdx.x; row < rows; row += 2 * gridDim.x) {
        const int row2 = row + gridDim.x;
        for (int k = threadIdx.x; k < g.N2; k += blockDim.x) {
            const double a = fdm_res_node(g, coef, x, row, k);
            const double b = row2 < rows ? fdm_res_node(g, coef, x, row2, k) : 0.0;
            acc = __dadd_rn(acc, __dadd_rn(a, b));
        }
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

// Lines along AXIS (0: i, 1: j, 2: k) and their numbering: i-lines by (j, k),
// j-lines by (i, k), k-lines by (i, j), the fastest coordinate last; LO and HI
// are the coefficients below and above the diagonal along AXIS
// (fdMatrix.hxx:99-101, 134-136, 169-171).
template <int AXIS>
struct LineGeo {
    static constexpr int LO = AXIS == 0 ? 3 : (AXIS == 1 ? 1 : 5), HI = AXIS == 0 ? 2 : (AXIS == 1 ? 0 : 4);
    static __device__ __forceinline__ int len(const Geo &g) { return AXIS == 0 ? g.N0 : (AXIS == 1 ? g.N1 : g.N2); }
    // (i, j, k) of node t on line (slow, fast): the line's two fixed coordinates,
    // slowest first (j, k for i-lines; i, k for j-lines; i, j for k-lines)
    static __device__ __forceinline__ void coords(int slow, int fast, int t, int &i, int &j, int &k)
    {
        if (AXIS == 0) {
            i = t;
            j = slow;
            k = fast;
        } else if (AXIS == 1) {
            i = slow;
            j = t;
            k = fast;
        } else {
            i = slow;
            j = fast;
            k = t;
        }
    }
    // the extent of the fastest fixed coordinate: line number = slow * nfast(g) + fast
    static __device__ __forceinline__ int nfast(const Geo &g) { return AXIS == 2 ? g.N1 : g.N2; }
};

// Factors of the periodic tridiagonal system of every line along AXIS.  The
// line's rows a_t x_{t-1} + b_t x_t + c_t x_{t+1} = d_t wrap around
// (x_{-1} = x_{n-1}, x_n = x_0).  Folding the two corner entries into the
// diagonal with gamma = -b_0 gives the open tridiagonal T' with
// T = T' + u v^T, u = (gamma, 0.., c_{n-1}), v = (1, 0.., a_0/gamma), so
// (Sherman-Morrison) x = y - z (v.y)/(1 + v.z) with T' y = d, T' z = u.
// Stored per node (fac = [w | cp | P | z], 4 N3 per axis): the inverse Thomas
// pivots w_t, the eliminated super-diagonal cp_t, z, and
// P_t = prod_{s<t} (-cp_s), so that the back-substituted y_0 is the sum of
// P_t yhat_t over the forward-eliminated yhat; per line (ls = [q | h]):
// q = a_0/gamma, h = 1/(1 + v.z).  The coefficients do not change while a
// solve runs, so this runs once per solve, and again only after they change.
// Blocks, tiles and warp 0's recurrences are those of k_fdm_line below: the
// forward pass turns a chunk's (a, b, c) into (w, cp, P, zhat) in place, the
// backward pass zhat into z.
constexpr int FDM_LT = 32, FDM_TT = 16, FDM_LINE_THREADS = 256;
constexpr int FDM_PER = FDM_LT * FDM_TT / FDM_LINE_THREADS;  // tile elements per thread
static_assert(FDM_LT * FDM_TT % FDM_LINE_THREADS == 0, "tile elements split evenly over the threads");

template <int AXIS>
__global__ void __launch_bounds__(FDM_LINE_THREADS, 4) k_fdm_factor(Geo g, const double *__restrict__ coef,
                                                                     double *fac, double *ls)
{
    using LG = LineGeo<AXIS>;
    constexpr int LO = LG::LO, HI = LG::HI, LT = FDM_LT, TT = FDM_TT;
    __shared__ double sm[4][LT][TT + 1];
    const long long N3 = g.N3;
    const int n = LG::len(g), nf = LG::nfast(g);
    const long long lines = N3 / n;
    const int groups = (nf + LT - 1) / LT;
    const int slow = (int)(blockIdx.x / groups), f0 = (int)(blockIdx.x % groups) * LT;
    const int nl = min(LT, nf - f0);
    const long long line0 = (long long)slow * nf + f0;
    double *W = fac, *CP = fac + N3, *P = fac + 2 * N3, *Z = fac + 3 * N3;
    const int tid = threadIdx.x;
    auto elem = [&](int e, int &l, int &tt) {
        if (AXIS == 2) {
            l = e / TT;
            tt = e % TT;
        } else {
            l = e % LT;
            tt = e / LT;
        }
    };
    auto node = [&](int l, int t) {
        int i, j, k;
        LG::coords(slow, f0 + l, t, i, j, k);
        return nidx(g, i, j, k);
    };
    const int nch = (n + TT - 1) / TT;
    // warp 0, lane l: line l's corner entries and running values
    double a0 = 0.0, cn = 0.0, gam = 1.0, cprev = 0.0, zprev = 0.0, pprev = 1.0;
    if (tid < nl) {
        a0 = coef[LO * N3 + node(tid, 0)];
        cn = coef[HI * N3 + node(tid, n - 1)];
        gam = -coef[6 * N3 + node(tid, 0)];
    }

    // forward elimination: slots (a, b, c) in, (w, cp, P, zhat) out
    for (int c = 0; c < nch; c++) {
        const int t0 = c * TT, nt = min(TT, n - t0);
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            if (c > 0 && l < nl) {  // the previous (full) chunk's factors
                const long long o = node(l, t0 - TT + tt);
                W[o] = sm[0][l][tt];
                CP[o] = sm[1][l][tt];
                P[o] = sm[2][l][tt];
                Z[o] = sm[3][l][tt];
            }
            const bool in = l < nl && tt < nt;
            const int t = in ? t0 + tt : t0;
            const long long o = node(in ? l : 0, t);
            const double av = t == 0 ? 0.0 : coef[LO * N3 + o], bv = coef[6 * N3 + o],
                         cv = t == n - 1 ? 0.0 : coef[HI * N3 + o];
            if (in) {
                sm[0][l][tt] = av;
                sm[1][l][tt] = bv;
                sm[2][l][tt] = cv;
            }
        }
        __syncthreads();
        if (tid < nl) {
            const int l = tid;
            for (int tt = 0; tt < nt; tt++) {
                const int t = t0 + tt;
                const double a = sm[0][l][tt], cc = sm[2][l][tt];
                double bb = sm[1][l][tt];
                if (t == 0) bb -= gam;
                if (t == n - 1) bb -= cn * a0 / gam;
                const double u = t == 0 ? gam : (t == n - 1 ? cn : 0.0);
                const double w = 1.0 / (bb - a * cprev);
                const double p = t == 0 ? 1.0 : pprev * -cprev;
                const double cpv = cc * w;
                const double zz = (u - a * zprev) * w;
                sm[0][l][tt] = w;
                sm[1][l][tt] = cpv;
                sm[2][l][tt] = p;
                sm[3][l][tt] = zz;
                cprev = cpv;
                zprev = zz;
                pprev = p;
            }
        }
        __syncthreads();
    }
    {  // the last chunk's factors
        const int t0 = (nch - 1) * TT, nt = n - t0;
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            if (l >= nl || tt >= nt) continue;
            const long long o = node(l, t0 + tt);
            W[o] = sm[0][l][tt];
            CP[o] = sm[1][l][tt];
            P[o] = sm[2][l][tt];
            Z[o] = sm[3][l][tt];
        }
    }
    __syncthreads();

    // z = zhat back-substituted, from the last chunk to the first
    double znext = 0.0, z0 = 0.0, zn = 0.0;
    for (int c = nch - 1; c >= 0; c--) {
        const int t0 = c * TT, nt = min(TT, n - t0);
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            const bool in = l < nl && tt < nt;
            const long long o = in ? node(l, t0 + tt) : node(0, t0);
            const double cpv = CP[o], zh = Z[o];
            if (in) {
                sm[1][l][tt] = cpv;
                sm[3][l][tt] = zh;
            }
        }
        __syncthreads();
        if (tid < nl) {
            const int l = tid;
            for (int tt = nt - 1; tt >= 0; tt--) {
                const double zz = sm[3][l][tt] - sm[1][l][tt] * znext;
                sm[3][l][tt] = zz;
                znext = zz;
                if (t0 + tt == n - 1) zn = zz;
                if (t0 + tt == 0) z0 = zz;
            }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            if (l >= nl || tt >= nt) continue;
            Z[node(l, t0 + tt)] = sm[3][l][tt];
        }
        __syncthreads();
    }
    if (tid < nl) {
        const double q = a0 / gam;
        ls[line0 + tid] = q;
        ls[lines + line0 + tid] = 1.0 / (1.0 + z0 + q * zn);
    }
}

// One sweep along AXIS with the factors of k_fdm_factor: every line solved at
// once, the neighbours off the line read from xin, the result in xout.  A
// block takes FDM_LT lines with consecutive values of the fastest fixed
// coordinate, in chunks of FDM_TT nodes along them.  Each chunk's tiles pass
// through shared memory so that every global access is coalesced: across the
// lines for i- and j-lines (consecutive k), along the line for k-lines.
// Warp 0 runs the recurrences, lane l on line l:
//   forward   yhat_t = (d_t - a_t yhat_{t-1}) w_t,  Y0 += P_t yhat_t   (yhat into xout)
//   f = (Y0 + q yhat_{n-1}) h                                            (= (v.y)/(1 + v.z))
//   backward  y_t = yhat_t - cp_t y_{t+1},  x_t = y_t - f z_t           (xout in place)
// Every thread loads its tile elements of the next chunk into registers
// before the block waits for warp 0, so those loads are in flight during the
// recurrences and the barriers.
template <int AXIS>
__global__ void __launch_bounds__(FDM_LINE_THREADS, 3) k_fdm_line(Geo g, const double *__restrict__ coef,
                                                                const double *__restrict__ fac,
                                                                const double *__restrict__ ls,
                                                                const double *__restrict__ xin, double *xout)
{
    using LG = LineGeo<AXIS>;
    constexpr int LO = LG::LO, LT = FDM_LT, TT = FDM_TT;
    __shared__ double sm[4][LT][TT + 1];
    const long long N3 = g.N3;
    const int n = LG::len(g), nf = LG::nfast(g);
    const long long lines = N3 / n;
    const int groups = (nf + LT - 1) / LT;
    const int slow = (int)(blockIdx.x / groups), f0 = (int)(blockIdx.x % groups) * LT;
    const int nl = min(LT, nf - f0);
    const long long line0 = (long long)slow * nf + f0;
    const double *W = fac, *CP = fac + N3, *P = fac + 2 * N3, *Z = fac + 3 * N3;
    const int tid = threadIdx.x;
    // element e of a tile, (line l, node tt of the chunk): consecutive threads on consecutive addresses
    auto elem = [&](int e, int &l, int &tt) {
        if (AXIS == 2) {
            l = e / TT;
            tt = e % TT;
        } else {
            l = e % LT;
            tt = e / LT;
        }
    };
    auto node = [&](int l, int t) {
        int i, j, k;
        LG::coords(slow, f0 + l, t, i, j, k);
        return nidx(g, i, j, k);
    };
    const int nch = (n + TT - 1) / TT;

    // a thread's forward operands of one tile element, as loaded: the source,
    // the four coefficients off the line and their neighbours (in the order
    // they are subtracted), the coefficient below the diagonal, w and P;
    // elements past the lines' or the chunk's end load node (0, t0)
    struct Fwd {
        double b, c[4], x[4], lo, w, p;
    };
    Fwd R[FDM_PER];
    auto load_fwd = [&](int c) {
        const int t0 = c * TT, nt = min(TT, n - t0);
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            const bool in = l < nl && tt < nt;
            const int t = in ? t0 + tt : t0;
            int i, j, k;
            LG::coords(slow, f0 + (in ? l : 0), t, i, j, k);
            const long long o = nidx(g, i, j, k);
            R[m].b = coef[7 * N3 + o];
            int q = 0;
            if (AXIS != 1) {
                R[m].c[q] = coef[0 * N3 + o];
                R[m].x[q++] = xin[nidx(g, i, wrapi(j + 1, g.N1), k)];
                R[m].c[q] = coef[1 * N3 + o];
                R[m].x[q++] = xin[nidx(g, i, wrapi(j - 1, g.N1), k)];
            }
            if (AXIS != 0) {
                R[m].c[q] = coef[2 * N3 + o];
                R[m].x[q++] = xin[nidx(g, wrapi(i + 1, g.N0), j, k)];
                R[m].c[q] = coef[3 * N3 + o];
                R[m].x[q++] = xin[nidx(g, wrapi(i - 1, g.N0), j, k)];
            }
            if (AXIS != 2) {
                R[m].c[q] = coef[4 * N3 + o];
                R[m].x[q++] = xin[nidx(g, i, j, wrapi(k + 1, g.N2))];
                R[m].c[q] = coef[5 * N3 + o];
                R[m].x[q++] = xin[nidx(g, i, j, wrapi(k - 1, g.N2))];
            }
            R[m].lo = t == 0 ? 0.0 : coef[LO * N3 + o];
            R[m].w = W[o];
            R[m].p = P[o];
        }
    };
    double yh = 0.0, Y0 = 0.0;  // warp 0, lane l: line l's last yhat and the sum for y_0

    // forward elimination; a thread stores the previous chunk's yhat of its own
    // tile elements before it puts the next chunk's operands into them
    load_fwd(0);
    for (int c = 0; c < nch; c++) {
        const int t0 = c * TT, nt = min(TT, n - t0);
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            if (c > 0 && l < nl) xout[node(l, t0 - TT + tt)] = sm[0][l][tt];  // chunks before the last are full
            if (l < nl && tt < nt) {
                double d = R[m].b;
#pragma unroll
                for (int q = 0; q < 4; q++) d -= R[m].c[q] * R[m].x[q];
                sm[0][l][tt] = d;
                sm[1][l][tt] = R[m].lo;
                sm[2][l][tt] = R[m].w;
                sm[3][l][tt] = R[m].p;
            }
        }
        if (c + 1 < nch) load_fwd(c + 1);
        __syncthreads();
        if (tid < nl) {
            const int l = tid;
#pragma unroll 8
            for (int tt = 0; tt < nt; tt++) {
                yh = (sm[0][l][tt] - sm[1][l][tt] * yh) * sm[2][l][tt];
                Y0 += sm[3][l][tt] * yh;
                sm[0][l][tt] = yh;
            }
        }
        __syncthreads();
    }

    // a thread's backward operands of one tile element: yhat, cp, z
    struct Bwd {
        double y, cp, z;
    };
    Bwd S[FDM_PER];
    auto load_bwd = [&](int c) {
        const int t0 = c * TT, nt = min(TT, n - t0);
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            const bool in = l < nl && tt < nt;
            const long long o = in ? node(l, t0 + tt) : node(0, t0);
            S[m].y = xout[o];
            S[m].cp = CP[o];
            S[m].z = Z[o];
        }
    };
    {  // the last chunk's yhat, then the backward operands of that chunk
        const int t0 = (nch - 1) * TT, nt = n - t0;
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            if (l < nl && tt < nt) xout[node(l, t0 + tt)] = sm[0][l][tt];
        }
        load_bwd(nch - 1);
    }
    double f = 0.0, ynext = 0.0;
    if (tid < nl) f = (Y0 + ls[line0 + tid] * yh) * ls[lines + line0 + tid];

    // back substitution and the correction, from the last chunk to the first;
    // a thread stores the previous chunk's x of its own tile elements before it
    // puts the next chunk's operands into them
    for (int c = nch - 1; c >= 0; c--) {
        const int t0 = c * TT, nt = min(TT, n - t0);
#pragma unroll
        for (int m = 0; m < FDM_PER; m++) {
            int l, tt;
            elem(tid + m * FDM_LINE_THREADS, l, tt);
            if (c + 1 < nch && l < nl && t0 + TT + tt < n) xout[node(l, t0 + TT + tt)] = sm[0][l][tt];
            if (l < nl && tt < nt) {
                sm[0][l][tt] = S[m].y;
                sm[1][l][tt] = S[m].cp;
                sm[2][l][tt] = S[m].z;
            }
        }
        if (c > 0) load_bwd(c - 1);
        __syncthreads();
        if (tid < nl) {
            const int l = tid;
#pragma unroll 8
            for (int tt = nt - 1; tt >= 0; tt--) {
                const double y = sm[0][l][tt] - sm[1][l][tt] * ynext;
                sm[0][l][tt] = y - f * sm[2][l][tt];
                ynext = y;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < FDM_PER; m++) {  // chunk 0's x
        int l, tt;
        elem(tid + m * FDM_LINE_THREADS, l, tt);
        if (l < nl && tt < min(TT, n)) xout[node(l, tt)] = sm[0][l][tt];
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

void launch_fdm_factor(int axis, const Geo &g, const double *coef, double *fac, double *ls, cudaStream_t st)
{
    // the blocks of k_fdm_line
    const int fast = axis == 2 ? g.N1 : g.N2, slow = axis == 0 ? g.N1 : g.N0;
    const unsigned nb = (unsigned)slow * (unsigned)((fast + FDM_LT - 1) / FDM_LT);
    if (axis == 0)
        k_fdm_factor<0><<<nb, FDM_LINE_THREADS, 0, st>>>(g, coef, fac, ls);
    else if (axis == 1)
        k_fdm_factor<1><<<nb, FDM_LINE_THREADS, 0, st>>>(g, coef, fac, ls);
    else
        k_fdm_factor<2><<<nb, FDM_LINE_THREADS, 0, st>>>(g, coef, fac, ls);
}

void launch_fdm_line(int axis, const Geo &g, const double *coef, const double *fac, const double *ls,
                     const double *xin, double *xout, cudaStream_t st)
{
    // one block per FDM_LT consecutive values of the fastest fixed coordinate
    const int fast = axis == 2 ? g.N1 : g.N2, slow = axis == 0 ? g.N1 : g.N0;
    const unsigned nb = (unsigned)slow * (unsigned)((fast + FDM_LT - 1) / FDM_LT);
    if (axis == 0)
        k_fdm_line<0><<<nb, FDM_LINE_THREADS, 0, st>>>(g, coef, fac, ls, xin, xout);
    else if (axis == 1)
        k_fdm_line<1><<<nb, FDM_LINE_THREADS, 0, st>>>(g, coef, fac, ls, xin, xout);
    else
        k_fdm_line<2><<<nb, FDM_LINE_THREADS, 0, st>>>(g, coef, fac, ls, xin, xout);
}

}  // namespace nova
