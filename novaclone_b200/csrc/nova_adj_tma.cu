// Adjoint stage kernels (FP64) fed by a TMA pipeline, the data movement of
// the forward stage kernel (nova_stage_tma.cu) for six halo'd components: a
// field P (the forward stage state Y of the Navier-Stokes stage, or the field
// frozen in or evolved by an MHD loop) and the adjoint direction g, with the
// building blocks of nova_adj_math.cuh combined per kind:
//   ADJ_NS: xi = dt [ Sx - 1/2 At - 1/2 g divP - nu bsum g ]     (reverse RK4 recursion)
//   ADJ_BB: xi = dt [ Sx + 1/2 At - 1/2 g divP - eta bsum g ]    (B loop, dF_B/dB; recursion)
//   ADJ_UB: acc += dt [ 1/2 g divP - Sx + 1/2 At + P divG ]      (dF_U/dB, P = B^n)
//   ADJ_BU: acc += dt [ 1/2 g divP - Sx - 1/2 At ]               (dF_B/dU, P = the B stage state)
// (Sx with the Laplacian weight nu for NS, eta for BB, none for UB and BU);
// the MHD right-hand sides are app/OT_Poisson/UEqn.H:16-23 and BEqn.H:72-78.
//
// A block owns a kTK(k) x 8(j) column and walks it along i: one producer warp
// (lane 0) loads, per plane, each of the two 3-component fields as its halo'd
// rows (box 32 x 3 x 14, [row][c][k]; a j-boundary tile as two boxes) and its
// 4-wide k halos (box 4 x 8 x 3) into a 7-slot ring, and the epilogue
// operands (mu and Lam, or the accumulated adjoint) into a 3-slot ring.
// Eight consumer warps, one per tile row, keep the i stencil of the six
// components in a register queue; the loop is unrolled by the queue period
// 7 = 2H + 1 = ring size, so the queue rotates by register renaming.  At
// s = 4 the g field is mu itself: every combination is linear in g, so the
// kernel works on mu and scales the result by 1/6, and the centre mu of the
// recursion comes from the queue.
//
// Every mbarrier wait is bounded (nova_tma.cuh); a wait that gives up raises
// the error word, and the producer drains its loads in flight, bounded, before
// the block exits.
#include "nova_adj_math.cuh"
#include "nova_internal.cuh"
#include "nova_tma.cuh"

#include <cstring>
#include <type_traits>

namespace nova {

namespace {

constexpr int kH = 3;
constexpr int TJ = 8;                        // tile rows: one consumer warp per row
constexpr int kWarps = TJ;
constexpr int kThreads = kTK * (TJ + 1);     // plus the producer warp
constexpr int kRing = 7;
constexpr int kERing = 3;
constexpr int kLRB = 8;                      // rows of the k-halo box
constexpr int kRowE = 3 * kTK;               // one halo'd row of a 3-component field
constexpr int kTcbE = (TJ + 2 * kH) * kRowE;
constexpr int kLRE = 3 * TJ * 4;             // one side's k-halo box
constexpr int kFieldE = kTcbE + 2 * kLRE;    // one field in a slot
constexpr int kSlotE = 2 * kFieldE;          // Y, then g
constexpr int kEpiE = TJ * kRowE;            // one epilogue field
static_assert(kRing == 2 * kH + 1, "queue rotation and ring slots share one period");
static_assert(TJ == kLRB && kLRB * 4 == kTK, "one k-halo box per side, component stride kTK");

// epilogue fields: mu, Lam (recursion kinds below s = 4) or the accumulated adjoint
template <int KIND, int S> __host__ __device__ constexpr int adj_epi()
{
    return (KIND == ADJ_NS || KIND == ADJ_BB) ? (S == 4 ? 0 : 2) : 1;
}

template <int NE> constexpr size_t adj_smem_bytes()
{
    return ((size_t)kRing * kSlotE + (size_t)kERing * NE * kEpiE) * sizeof(double) + 8 * (2 * kRing + 2 * kERing);
}

struct AdjMaps {
    CUtensorMap f[2][4];  // per field: rows TJ+6, 3, TJ+3, k halos
    CUtensorMap e[2];     // mu, Lam (or the accumulated adjoint)
};

template <int KIND, int S>
__global__ void __launch_bounds__(kThreads, 1)
    k_adj_tma(Geo g, Coef<double> co, const double *__restrict__ ia, double dt, double nu, AdjArgs args,
              double *__restrict__ acc, const __grid_constant__ AdjMaps maps, int ichunk, int *err)
{
    constexpr int H = kH, NE = adj_epi<KIND, S>();
    constexpr bool kRec = KIND == ADJ_NS || KIND == ADJ_BB;  // reverse RK4 recursion kinds
    constexpr uint32_t kSlotBytes = kSlotE * 8, kRowBytes = kRowE * 8, kEpiBytes = kEpiE * 8;
    constexpr uint32_t kFieldBytes = kFieldE * 8, kLRBytes = kLRE * 8;
    extern __shared__ __align__(128) unsigned char smraw[];
    const double *ring = reinterpret_cast<const double *>(smraw);
    const double *ering = ring + kRing * kSlotE;
    const uint32_t s0 = smem_addr(smraw);
    const uint32_t e0addr = s0 + kRing * kSlotBytes;
    const uint32_t bar0 = e0addr + kERing * NE * kEpiBytes;
    auto full = [&](int r) { return bar0 + 8u * r; };
    auto empty = [&](int r) { return bar0 + 8u * (kRing + r); };
    auto efull = [&](int r) { return bar0 + 8u * (2 * kRing + r); };
    auto eempty = [&](int r) { return bar0 + 8u * (2 * kRing + kERing + r); };

    const int tx = threadIdx.x, ty = threadIdx.y, lane = tx;
    const int k0 = blockIdx.x * kTK, j0 = blockIdx.y * TJ;
    const int ib = blockIdx.z * ichunk, ie = min(ib + ichunk, g.N0);
    const int nout = ie - ib, nld = nout + 2 * H;

    if (ty == TJ && lane == 0) {
        for (int r = 0; r < kRing; r++) {
            mbar_init(full(r), 1);
            mbar_init(empty(r), kWarps);
        }
        for (int r = 0; r < kERing; r++) {
            mbar_init(efull(r), 1);
            mbar_init(eempty(r), kWarps);
        }
        mbar_init_fence();
    }
    __syncthreads();

    // ---- producer warp: lane 0 issues every load of the block ----
    if (ty == TJ) {
        if (lane != 0) return;
        const bool jlo = j0 < H, jhi = j0 + TJ + H > g.N1;
        const int kl = (k0 == 0 ? g.N2 : k0) - 4, kr = (k0 + kTK == g.N2) ? 0 : k0 + kTK;
        auto issue_s = [&](int n) -> bool {  // stencil load n: plane ib - H + n
            const int r = n % kRing;
            if (n >= kRing && !mbar_wait(empty(r), ((n / kRing) + 1) & 1, err)) return false;
            const uint32_t bar = full(r);
            mbar_expect_tx(bar, kSlotBytes);
            const int plane = wrapi(ib - H + n, g.N0);
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const uint32_t dst = s0 + r * kSlotBytes + f * kFieldBytes;
                const CUtensorMap *m = maps.f[f];
                if (jlo) {
                    tma_load_4d(dst, &m[1], bar, k0, 0, g.N1 - H, plane);
                    tma_load_4d(dst + H * kRowBytes, &m[2], bar, k0, 0, 0, plane);
                } else if (jhi) {
                    tma_load_4d(dst, &m[2], bar, k0, 0, j0 - H, plane);
                    tma_load_4d(dst + (TJ + H) * kRowBytes, &m[1], bar, k0, 0, 0, plane);
                } else {
                    tma_load_4d(dst, &m[0], bar, k0, 0, j0 - H, plane);
                }
                tma_load_4d(dst + kTcbE * 8, &m[3], bar, kl, j0, 0, plane);
                tma_load_4d(dst + kTcbE * 8 + kLRBytes, &m[3], bar, kr, j0, 0, plane);
            }
            return true;
        };
        auto issue_e = [&](int n) -> bool {  // epilogue load n: plane ib + n
            const int r = n % kERing;
            if (n >= kERing && !mbar_wait(eempty(r), ((n / kERing) + 1) & 1, err)) return false;
            const uint32_t dst = e0addr + r * NE * kEpiBytes, bar = efull(r);
            mbar_expect_tx(bar, NE * kEpiBytes);
#pragma unroll
            for (int f = 0; f < NE; f++) tma_load_4d(dst + f * kEpiBytes, &maps.e[f], bar, k0, 0, j0, ib + n);
            return true;
        };
        int iss = 0, ise = 0;
        bool ok = true;
        for (int t = -2 * H; t < nout && ok; t++) {
            if ((ok = issue_s(t + 2 * H))) iss++;
            if (NE > 0 && ok && t >= 0 && (ok = issue_e(t))) ise++;
        }
        if (!ok) {
            // the consumers may have left: wait, bounded, for the loads still landing in shared memory
            for (int n = max(0, iss - kRing); n < iss; n++) mbar_wait(full(n % kRing), (n / kRing) & 1, err, true);
            for (int n = max(0, ise - kERing); n < ise; n++)
                mbar_wait(efull(n % kERing), (n / kERing) & 1, err, true);
        }
        return;
    }

    // ---- consumer warps ----
    auto release = [&](uint32_t bar) {
        __syncwarp();
        if (lane == 0) mbar_arrive(bar);
    };
    const int kw = k0 + tx;
    double az[H], bz[H], bsum;
    adj_zweights<double, H>(co, ia[kw], az, bz, bsum);

    // slot offsets within a field: centre, and the k neighbour at s (row box
    // or the left/right halo boxes, [c][8 rows][4]); component stride kTK in both
    const int cen = (H + ty) * kRowE + tx;
    auto zoff = [&](int s) -> int {
        const int x = tx + s;
        return x < 0 ? kTcbE + ty * 4 + 4 + x : (x >= kTK ? kTcbE + kLRE + ty * 4 + (x - kTK) : cen + s);
    };
    auto fo = [](int c) { return (c / 3) * kFieldE + (c % 3) * kTK; };  // field and component offset

    // i-stencil queue: plane ib - H + x lives in q[x % 7]
    double q[2 * H + 1][6];
    bool ok = true;
    for (int n = 0; n < 2 * H; n++) {  // queue: planes ib-3 .. ib+2
        ok = mbar_wait(full(n % kRing), (n / kRing) & 1, err);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        const double *sl = ring + (n % kRing) * kSlotE;
#pragma unroll
        for (int c = 0; c < 6; c++) q[n][c] = sl[fo(c) + cen];
        if (n < H || n >= H + nout) release(empty(n % kRing));  // queue-only plane
    }

    int es = 0, eph = 0;  // epilogue ring slot and phase of step p
    // step p = 7 m + R: queue head plane p + 2H (slot (R + 6) % 7), centre
    // plane p + H (slot (R + 3) % 7)
    auto step = [&](auto Rc, int m, int p) -> bool {
        constexpr int R = decltype(Rc)::value;
        constexpr int sHd = (R + 2 * H) % kRing, sCur = (R + H) % kRing;
        const int hd = p + 2 * H;
        if (!__all_sync(0xffffffffu, mbar_wait(full(sHd), (m + (R + 2 * H) / kRing) & 1, err))) return false;
        {
            constexpr int kQ = (R + 2 * H) % (2 * H + 1);
            const double *sh = ring + sHd * kSlotE;
#pragma unroll
            for (int c = 0; c < 6; c++) q[kQ][c] = sh[fo(c) + cen];
            if (hd >= H + nout) release(empty(sHd));
        }
        const double *sl = ring + sCur * kSlotE;
        auto vx = [&](int c, int s) -> double { return q[(R + H + s + 2 * H + 1) % (2 * H + 1)][c]; };
        auto vy = [&](int c, int s) -> double { return sl[fo(c) + cen + s * kRowE]; };
        auto vz = [&](int c, int s) -> double { return sl[fo(c) + zoff(s)]; };
        constexpr int kC = (R + H) % (2 * H + 1);
        const double p0[3] = {q[kC][0], q[kC][1], q[kC][2]};
        const double g0[3] = {q[kC][3], q[kC][4], q[kC][5]};
        double Sx[3], At[3], divP, divG;
        adj_terms<double, H, KIND == ADJ_UB>(vx, vy, vz, p0, g0, co, az, bz, kRec ? nu : 0.0, Sx, At, divP, divG);
        release(empty(sCur));  // the slot's values are in registers
        constexpr double gs = S == 4 ? 1.0 / 6.0 : 1.0;  // g4 = mu / 6
        double r[3];
#pragma unroll
        for (int e = 0; e < 3; e++) {
            if constexpr (KIND == ADJ_NS)
                r[e] = dt * (Sx[e] - 0.5 * fma(g0[e], divP, At[e]) - nu * bsum * g0[e]);
            else if constexpr (KIND == ADJ_BB)
                r[e] = dt * (Sx[e] + 0.5 * fma(-g0[e], divP, At[e]) - nu * bsum * g0[e]);
            else if constexpr (KIND == ADJ_UB)
                r[e] = dt * (fma(0.5 * g0[e], divP, -Sx[e]) + fma(0.5, At[e], p0[e] * divG));
            else
                r[e] = dt * (fma(0.5 * g0[e], divP, -Sx[e]) - 0.5 * At[e]);
            if constexpr (S == 4) r[e] *= gs;
        }

        double e0[3], e1[3] = {0, 0, 0};
        if constexpr (NE > 0) {
            if (!__all_sync(0xffffffffu, mbar_wait(efull(es), eph, err))) return false;
            const double *se = ering + es * NE * kEpiE + ty * kRowE + tx;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                e0[c] = se[c * kTK];
                if constexpr (NE > 1) e1[c] = se[kEpiE + c * kTK];
            }
            release(eempty(es));
            if (++es == kERing) {
                es = 0;
                eph ^= 1;
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) e0[c] = g0[c];  // mu: the g field at s = 4
        }
        const long long idx = (long long)(ib + p) * g.N12 + (long long)(j0 + ty) * g.N2 + kw;
#pragma unroll
        for (int e = 0; e < 3; e++) {
            const long long o = (long long)e * g.N3 + idx;
            if constexpr (kRec)
                adj_store<double, S>(args, o, e0[e], e1[e], r[e]);
            else
                acc[o] = e0[e] + r[e];
        }
        return true;
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using I3 = std::integral_constant<int, 3>;
    using I4 = std::integral_constant<int, 4>;
    using I5 = std::integral_constant<int, 5>;
    using I6 = std::integral_constant<int, 6>;
    for (int m = 0, p = 0; ok && p < nout; m++, p += kRing) {
        ok = step(I0{}, m, p) && (p + 1 >= nout || (step(I1{}, m, p + 1) && (p + 2 >= nout ||
             (step(I2{}, m, p + 2) && (p + 3 >= nout || (step(I3{}, m, p + 3) && (p + 4 >= nout ||
             (step(I4{}, m, p + 4) && (p + 5 >= nout || (step(I5{}, m, p + 5) && (p + 6 >= nout ||
             step(I6{}, m, p + 6))))))))))));
    }
}

// i-chunk: >= ~4 waves of the one resident block per SM
int adj_ichunk(const Geo &g)
{
    const long long tiles = (long long)(g.N2 / kTK) * (g.N1 / TJ);
    int ch = g.N0;
    while (ch > 16 && tiles * ((g.N0 + ch - 1) / ch) < 148LL * 4) ch /= 2;
    return ch;
}

template <int KIND, int S>
cudaError_t launch_adj_s(const Geo &g, const Coef<double> &co, const double *ia, double dt, double nu,
                         const AdjArgs &a, double *acc, int *err, cudaStream_t st)
{
    constexpr int NE = adj_epi<KIND, S>();
    AdjMaps maps;
    memset(&maps, 0, sizeof maps);
    const double *fld[2] = {a.Y, a.G};  // at s = 4 the drivers pass mu as g
    bool ok = true;
    for (int f = 0; f < 2; f++)
        ok = ok && tma_encode_field(&maps.f[f][0], fld[f], g, TJ + 2 * kH) &&
             tma_encode_field(&maps.f[f][1], fld[f], g, kH) && tma_encode_field(&maps.f[f][2], fld[f], g, TJ + kH) &&
             tma_encode_field(&maps.f[f][3], fld[f], g, 0);
    if (KIND == ADJ_NS || KIND == ADJ_BB) {
        if (NE > 0) ok = ok && tma_encode_field(&maps.e[0], a.mu, g, TJ) && tma_encode_field(&maps.e[1], a.Lam, g, TJ);
    } else {
        ok = ok && tma_encode_field(&maps.e[0], acc, g, TJ);
    }
    if (!ok) return cudaErrorInvalidValue;
    constexpr size_t smem = adj_smem_bytes<NE>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_adj_tma<KIND, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int ch = adj_ichunk(g);
    const dim3 grid(g.N2 / kTK, g.N1 / TJ, (g.N0 + ch - 1) / ch);
    k_adj_tma<KIND, S><<<grid, dim3(kTK, TJ + 1), smem, st>>>(g, co, ia, dt, nu, a, acc, maps, ch, err);
    return cudaGetLastError();
}

template <int KIND>
cudaError_t launch_adj_k(int s, const Geo &g, const Coef<double> &co, const double *ia, double dt, double nu,
                         const AdjArgs &a, double *acc, int *err, cudaStream_t st)
{
    switch (s) {
    case 4: return launch_adj_s<KIND, 4>(g, co, ia, dt, nu, a, acc, err, st);
    case 3: return launch_adj_s<KIND, 3>(g, co, ia, dt, nu, a, acc, err, st);
    case 2: return launch_adj_s<KIND, 2>(g, co, ia, dt, nu, a, acc, err, st);
    default: return launch_adj_s<KIND, 1>(g, co, ia, dt, nu, a, acc, err, st);
    }
}

}  // namespace

bool adj_tma_fits(const Geo &g) { return !g.wallY && g.N2 % kTK == 0 && g.N1 % TJ == 0 && g.N1 >= 2 * TJ; }

cudaError_t launch_adj_tma64(int kind, int s, const Geo &g, const Coef<double> &co, const double *ia, double dt,
                             double nu, const AdjArgs &a, double *acc, int *err, cudaStream_t st)
{
    switch (kind) {
    case ADJ_UB: return launch_adj_k<ADJ_UB>(s, g, co, ia, dt, nu, a, acc, err, st);
    case ADJ_BU: return launch_adj_k<ADJ_BU>(s, g, co, ia, dt, nu, a, acc, err, st);
    case ADJ_BB: return launch_adj_k<ADJ_BB>(s, g, co, ia, dt, nu, a, acc, err, st);
    default: return launch_adj_k<ADJ_NS>(s, g, co, ia, dt, nu, a, acc, err, st);
    }
}

}  // namespace nova
