// Navier-Stokes stage kernel fed by a TMA pipeline (sm_100a).
//
// Same arithmetic and stage update as the register-queue march of
// nova_stage.cu (nova_stage_math.cuh), different data movement.  A block owns
// a kTK(k) x TJ(j) column of the grid and walks it along i.  A producer warp
// issues, for every plane, bulk tensor loads of
//   TCB: the tile's rows plus H halo rows on either side, all three
//        components, laid out [row][c][k] (box 32 x 3 x (TJ + 6)), and
//   L/R: the H-wide k halos left and right of the tile (boxes 4 x 8 x 3,
//        [c][j][k], 4 wide to keep the 16-byte TMA alignment),
// into a ring of kRing shared-memory slots, each completed by an mbarrier
// transaction count, and the pointwise epilogue operands of the plane (RK base
// and accumulator, box 32 x 3 x TJ) into a second ring.  Periodic wrap needs
// no ghost storage: in k the halo boxes start at the wrapped column (the tile
// width divides N2), in j a boundary tile's rows arrive as two boxes (3 and
// TJ + 3 rows) that land back to back in the slot.
//
// The consumer warps keep the i stencil in a register queue (the centre of
// each arriving plane), read the j and k stencils from the slot of the plane
// they are computing, and hand slots back through per-warp arrivals on the
// slot's `empty` barrier; the producer refills a slot as soon as every warp
// has released it, which keeps kRing - 2H - 1 planes in flight ahead of the
// queue head.
//
// Every mbarrier wait is bounded (nova_tma.cuh); a wait that gives up raises
// the error word and the block leaves its pipeline, the producer after waiting,
// again bounded, for the loads it still has in flight.
#include "nova_diag.cuh"
#include "nova_internal.cuh"
#include "nova_ops.cuh"
#include "nova_stage_math.cuh"
#include "nova_tile.cuh"
#include "nova_tma.cuh"

#include <cudaTypedefs.h>

#include <cstring>
#include <type_traits>

namespace nova {

namespace {

constexpr int kH = 3;
constexpr int kRowE = 3 * kTK;  // one halo'd row, three components
constexpr int kLRB = 8;         // rows of one k-halo box

// Tile and ring configuration per precision.  FP64: a 32 x 16 tile, one block
// per SM, one consumer warp per tile row.  FP32: a 32 x 8 tile, three blocks
// per SM, one consumer warp per two tile rows (a half-warp per row, each lane
// two adjacent k nodes in the paired f32x2 arithmetic).  Each block also has
// one producer warp, whose elected lane issues the loads in the order the
// consumers need them and blocks on the ring's `empty` barriers alone, so it
// never delays the arithmetic.
template <typename T> struct TmaCfg {
    static constexpr int TJ = sizeof(T) == 8 ? 16 : 8;
    static constexpr int kWarps = sizeof(T) == 8 ? TJ : TJ / 2;  // consumer warps
    static constexpr int kThreads = kTK * (kWarps + 1);          // plus the producer warp
    static constexpr int kBlocksPerSM = sizeof(T) == 8 ? 1 : 3;
    static constexpr int kRing = 7;   // stencil slots: the queue head runs kRing - 2H - 1 planes behind the loads
    static constexpr int kERing = 3;  // epilogue slots
    static constexpr int kTcbE = (TJ + 2 * kH) * kRowE;
    static constexpr int kLRE = 3 * TJ * 4;           // the k-halo boxes of one side
    static constexpr int kSlotE = kTcbE + 2 * kLRE;   // elements per stencil slot
    static constexpr int kEpiE = TJ * kRowE;          // elements per epilogue field
    static_assert(kRing >= 2 * kH + 1, "the queue and the plane computed fit in the ring");
    static_assert(TJ % kLRB == 0 && kLRB * 4 == kTK, "k-halo boxes share the component stride of the row boxes");
};

// epilogue operands per stage, in load order
//   FP64:  s=1,2: U0, A   s=3: A   s=5: U0
//   split: s=1,2: U0hi, A   s=3: U0hi, A, U0lo   s=4: U0lo   s=5: U0hi, U0lo
template <typename T, int STAGE> __host__ __device__ constexpr int epi_fields()
{
    if constexpr (sizeof(T) == 8)
        return (STAGE == 1 || STAGE == 2) ? 2 : ((STAGE == 3 || STAGE == 5) ? 1 : 0);
    else
        return (STAGE == 1 || STAGE == 2 || STAGE == 5) ? 2 : (STAGE == 3 ? 3 : (STAGE == 4 ? 1 : 0));
}

// ring data, the ring barriers, then (DIAG launches) kDiagParts doubles per
// consumer warp for the block's reduction and six per consumer thread for the
// running diagnostics
template <typename T, int NE, bool DIAG = false> constexpr size_t tma_smem_bytes()
{
    using C = TmaCfg<T>;
    return ((size_t)C::kRing * C::kSlotE + (size_t)C::kERing * NE * C::kEpiE) * sizeof(T) +
           8 * (2 * C::kRing + 2 * C::kERing) + (DIAG ? 8 * (kDiagParts + 6 * kTK) * C::kWarps : 0);
}

struct StageMaps {
    CUtensorMap tcbA, tcb3, tcbB;  // halo'd rows of the stencil field: TJ+6, 3 or TJ+3 rows
    CUtensorMap tcbC;              // its TJ tile rows alone (the queue-only planes)
    CUtensorMap lr;                // k-halo boxes (4 x 8 x 3) of the stencil field
    CUtensorMap e[3];              // epilogue operands
};

template <typename T, int STAGE, int EPI_E>
__device__ __forceinline__ void epi_read(const T *se, int c, T &e0, T &e1, T &lo)
{
    if constexpr (STAGE == 1 || STAGE == 2) {
        e0 = se[c * kTK];
        e1 = se[EPI_E + c * kTK];
    } else if constexpr (STAGE == 3) {
        if constexpr (sizeof(T) == 8) {
            e1 = se[c * kTK];
        } else {
            e0 = se[c * kTK];
            e1 = se[EPI_E + c * kTK];
            lo = se[2 * EPI_E + c * kTK];
        }
    } else if constexpr (STAGE == 4 && sizeof(T) == 4) {
        lo = se[c * kTK];
    } else if constexpr (STAGE == 5 && sizeof(T) == 8) {
        e0 = se[c * kTK];
    }
}

// DIAG (FP64, stages that read U itself: 0 and the literal 4, uniform
// periodic mesh): the block also reduces the history row's terms of U over its
// nodes (nova_diag.cuh: energy, |U|, U_x, the divergence the stage arithmetic
// forms anyway, and the two curls from the stencil values it holds) into
// dpart[block * kDiagParts] (the B terms zero).
// WALLS (FP32, walls on the y nodes j = 0 and j = N1 - 1): one row box per
// plane from j0 - H (the bulk copy fills rows outside 0..N1-1 with zeros, the
// last tile may be ragged); in a warp with a row within H of a wall, a valid
// row's j neighbour across the wall is the wall_ghost of its mirror row (the
// march's formula); rows past N1 - 1 compute but store nothing.  (FP64 wall
// stages stay on the march: at 96 registers a thread the ghost branch spills.)
template <typename T, int STAGE, bool STRETCH, class Args, bool DIAG, bool WALLS = false>
__global__ void __launch_bounds__(TmaCfg<T>::kThreads, TmaCfg<T>::kBlocksPerSM)
    k_stage_tma(Geo g, Coef<T> co, StageCoef<T> sc, const Walls<T> wl, const T *__restrict__ ia,
                const T *__restrict__ corr2, T dt, T visc, Args args, const __grid_constant__ StageMaps maps,
                int ichunk, int *err, double *dpart)
{
    static_assert(!DIAG || (sizeof(T) == 8 && (STAGE == 0 || STAGE == 4)), "diagnostics of an FP64 state only");
    static_assert(!(DIAG && WALLS), "diagnostics on periodic meshes");
    static_assert(!WALLS || sizeof(T) == 4, "FP64 wall stages run the register-queue march");
    using C = TmaCfg<T>;
    constexpr int H = kH, TJ = C::TJ, kRing = C::kRing, kERing = C::kERing;
    constexpr int kTcbE = C::kTcbE, kLRE = C::kLRE, kSlotE = C::kSlotE, kEpiE = C::kEpiE;
    constexpr int NE = epi_fields<T, STAGE>();
    constexpr uint32_t kSlotBytes = kSlotE * sizeof(T), kRowBytes = kRowE * sizeof(T), kEpiBytes = kEpiE * sizeof(T);
    constexpr uint32_t kLRBoxBytes = 3 * kLRB * 4 * sizeof(T);
    extern __shared__ __align__(128) unsigned char smraw[];
    const T *ring = reinterpret_cast<const T *>(smraw);
    const T *ering = ring + kRing * kSlotE;
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

    if (ty == C::kWarps && lane == 0) {  // the producer warp's lane initialises the barriers
        for (int r = 0; r < kRing; r++) {
            mbar_init(full(r), 1);
            mbar_init(empty(r), C::kWarps);
        }
        for (int r = 0; r < kERing; r++) {
            mbar_init(efull(r), 1);
            mbar_init(eempty(r), C::kWarps);
        }
        mbar_init_fence();
    }
    __syncthreads();

    // ---- producer warp: lane 0 issues every load of the block ----
    if (ty == C::kWarps) {
        if (lane != 0) return;
        const bool jlo = j0 < H, jhi = j0 + TJ + H > g.N1;
        const int kl = (k0 == 0 ? g.N2 : k0) - 4, kr = (k0 + kTK == g.N2) ? 0 : k0 + kTK;
        auto issue_s = [&](int n) -> bool {  // stencil load n: plane ib - H + n
            const int r = n % kRing;
            if (n >= kRing && !mbar_wait(empty(r), ((n / kRing) + 1) & 1, err)) return false;
            const uint32_t dst = s0 + r * kSlotBytes, bar = full(r);
            const int plane = wrapi(ib - H + n, g.N0);
            if (n < H || n >= H + nout) {
                // a queue-only plane: the consumers read the tile rows' centre values alone
                mbar_expect_tx(bar, TJ * kRowBytes);
                tma_load_4d(dst + H * kRowBytes, &maps.tcbC, bar, k0, 0, j0, plane);
                return true;
            }
            mbar_expect_tx(bar, kSlotBytes);
            if (WALLS) {
                tma_load_4d(dst, &maps.tcbA, bar, k0, 0, j0 - H, plane);
            } else if (jlo) {
                tma_load_4d(dst, &maps.tcb3, bar, k0, 0, g.N1 - H, plane);
                tma_load_4d(dst + H * kRowBytes, &maps.tcbB, bar, k0, 0, 0, plane);
            } else if (jhi) {
                tma_load_4d(dst, &maps.tcbB, bar, k0, 0, j0 - H, plane);
                tma_load_4d(dst + (TJ + H) * kRowBytes, &maps.tcb3, bar, k0, 0, 0, plane);
            } else {
                tma_load_4d(dst, &maps.tcbA, bar, k0, 0, j0 - H, plane);
            }
#pragma unroll
            for (int b = 0; b < TJ / kLRB; b++) {
                tma_load_4d(dst + kTcbE * sizeof(T) + b * kLRBoxBytes, &maps.lr, bar, kl, j0 + b * kLRB, 0, plane);
                tma_load_4d(dst + (kTcbE + kLRE) * sizeof(T) + b * kLRBoxBytes, &maps.lr, bar, kr, j0 + b * kLRB, 0,
                            plane);
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
        // in the order of need: stencil load t + 2H is the queue head of step t,
        // epilogue load t is read at step t
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
    // slot offset of the element at tile row r, tile column x (-4 <= x < kTK + 4):
    // the row box, or the left/right halo boxes ([box][c][8 rows][4]);
    // component stride kTK in both
    auto soff = [&](int r, int x) -> int {
        const int lrrow = (r / kLRB) * 3 * kLRB * 4 + (r % kLRB) * 4;
        return x < 0 ? kTcbE + lrrow + 4 + x : (x >= kTK ? kTcbE + kLRE + lrrow + (x - kTK) : (H + r) * kRowE + x);
    };

    // i-stencil queue of the centre values of planes cur-3 .. cur+3.
    // FP64: the queue shifts by one plane per step (q[s] = logical s); the
    // unrolled form below exceeds the FP64 kernel's 96-register budget.
    // FP32: plane ib - H + x lives in q[x % 7], so logical plane s (0..2H,
    // centre H) of step p is q[(p + s) % 7]; the loop is unrolled by 7
    // (= 2H + 1 = kRing) so that the rotation is register renaming and every
    // ring slot index is a compile-time constant of the unrolled step.
    // DIAG: the running diagnostics in shared memory (the registers hold the queue)
    double *dred = reinterpret_cast<double *>(smraw + (bar0 - s0) + 8 * (2 * kRing + 2 * kERing));
    DiagAccSm dacc{dred + kDiagParts * C::kWarps + ty * kTK + tx, C::kWarps * kTK};
    if constexpr (DIAG) dacc.init();
    if constexpr (sizeof(T) == 8) {
        const int kw = k0 + tx;
        const T iak = ia[kw];
        const T c2k = STRETCH ? corr2[kw] : T(0);
        const int cen = (H + ty) * kRowE + tx;
        auto zoff = [&](int s) -> int { return soff(ty, tx + s); };
        T q[2 * H + 1][3];
        bool ok = true;
        for (int n = 0; n < 2 * H; n++) {  // queue: planes ib-3 .. ib+2
            ok = mbar_wait(full(n % kRing), (n / kRing) & 1, err);
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
            const T *sl = ring + (n % kRing) * kSlotE;
#pragma unroll
            for (int c = 0; c < 3; c++) q[n + 1][c] = sl[cen + c * kTK];
            if (n < H || n >= H + nout) release(empty(n % kRing));  // queue-only plane
        }

        for (int p = 0; p < nout && ok; p++) {
            const int hd = p + 2 * H;  // queue head: plane ib + p + 3
            ok = mbar_wait(full(hd % kRing), (hd / kRing) & 1, err);
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
#pragma unroll
            for (int s = 0; s < 2 * H; s++)
#pragma unroll
                for (int c = 0; c < 3; c++) q[s][c] = q[s + 1][c];
            {
                const T *sh = ring + (hd % kRing) * kSlotE;
#pragma unroll
                for (int c = 0; c < 3; c++) q[2 * H][c] = sh[cen + c * kTK];
                if (hd >= H + nout) release(empty(hd % kRing));
            }

            const int cur = p + H;
            const T *sl = ring + (cur % kRing) * kSlotE;
            auto vx = [&](int c, int s) -> T { return q[H + s][c]; };
            auto vy = [&](int c, int s) -> T { return sl[cen + s * kRowE + c * kTK]; };
            auto vz = [&](int c, int s) -> T { return sl[zoff(s) + c * kTK]; };
            const T u0[3] = {q[H][0], q[H][1], q[H][2]};
            T rhs[3], divu;
            ns_rhs<T, H, STRETCH>(vx, vy, vz, u0, co, sc, iak, c2k, visc, rhs, divu);
            if constexpr (DIAG) {
                double q1, hs;
                curl_terms<H>(vx, vy, vz, 0, co.a[0], co.a[1], co.a[2], iak, q1, hs);
                dacc.add(u0, divu, q1, hs);
            }
            release(empty(cur % kRing));  // the slot's values are in registers

            T e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
            if constexpr (NE > 0) {
                ok = mbar_wait(efull(p % kERing), (p / kERing) & 1, err);
                if (!__all_sync(0xffffffffu, ok)) {
                    ok = false;
                    break;
                }
                const T *se = ering + (p % kERing) * NE * kEpiE + ty * kRowE + tx;
#pragma unroll
                for (int c = 0; c < 3; c++) epi_read<T, STAGE, kEpiE>(se, c, e0[c], e1[c], lo[c]);
                release(eempty(p % kERing));
            }
            const long long idx = (long long)(ib + p) * g.N12 + (long long)(j0 + ty) * g.N2 + kw;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const long long o = (long long)c * g.N3 + idx;
                if constexpr (sizeof(T) == 8)
                    rk_store64<STAGE>(args, o, q[H][c], e0[c], e1[c], dt * rhs[c]);
                else
                    rk_store32<STAGE>(args, o, q[H][c], e0[c], e1[c], lo[c], dt * rhs[c]);
            }
        }
    } else {
        // FP32: warp ty computes tile rows 2 ty and 2 ty + 1 (one per half-warp),
        // each lane the two adjacent k nodes kk, kk + 1 of its row in the paired
        // arithmetic (ns_rhs2); pairs load as 8-byte shared-memory words.
        static_assert(kRing == 2 * H + 1, "queue rotation and ring slots share one period");
        static_assert(2 * C::kWarps == TJ, "two tile rows per consumer warp");
        const int r = 2 * ty + (lane >> 4), kk = 2 * (lane & 15);
        const int cen = (H + r) * kRowE + kk;
        const int jrow = j0 + r;
        // the rows next to a wall take the j neighbours across it from ghosts
        // (the choice is made per warp: its two rows together)
        const bool nearw =
            WALLS && __any_sync(0xffffffffu, jrow < g.N1 && (jrow < H || jrow + H > g.N1 - 1));
        // the z neighbours' pairs starting at kk - 4, kk - 2, kk + 2, kk + 4
        const int zm4 = soff(r, kk - 4), zm2 = soff(r, kk - 2), zp2 = soff(r, kk + 2), zp4 = soff(r, kk + 4);
        const float2 iak = *reinterpret_cast<const float2 *>(ia + k0 + kk);
        const float2 c2k = STRETCH ? *reinterpret_cast<const float2 *>(corr2 + k0 + kk) : f2(0.0f);
        auto ld2 = [](const T *b, int o) -> float2 { return *reinterpret_cast<const float2 *>(b + o); };
        float2 q[2 * H + 1][3];
        bool ok = true;
        for (int n = 0; n < 2 * H; n++) {  // queue: planes ib-3 .. ib+2
            ok = mbar_wait(full(n % kRing), (n / kRing) & 1, err);
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
            const T *sl = ring + (n % kRing) * kSlotE;
#pragma unroll
            for (int c = 0; c < 3; c++) q[n][c] = ld2(sl, cen + c * kTK);
            if (n < H || n >= H + nout) release(empty(n % kRing));  // queue-only plane
        }

        int es = 0, eph = 0;  // epilogue ring slot and phase of step p
        // step p = 7 m + R: queue head plane hd = p + 2H, centre plane cur = p + H
        auto step = [&](auto Rc, int m, int p) -> bool {
            constexpr int R = decltype(Rc)::value;
            const int hd = p + 2 * H;
            constexpr int sHd = (R + 2 * H) % kRing, sCur = (R + H) % kRing;
            if (!__all_sync(0xffffffffu, mbar_wait(full(sHd), (m + (R + 2 * H) / kRing) & 1, err))) return false;
            {
                // the new head, plane ib + p + H, replaces plane ib + p - H - 1
                constexpr int kQ = (R + 2 * H) % (2 * H + 1);
                const T *sh = ring + sHd * kSlotE;
#pragma unroll
                for (int c = 0; c < 3; c++) q[kQ][c] = ld2(sh, cen + c * kTK);
                if (hd >= H + nout) release(empty(sHd));
            }
            const T *sl = ring + sCur * kSlotE;
            constexpr int kC = (R + H) % (2 * H + 1);
            auto vx = [&](int c, int s) -> float2 { return q[(R + H + s + 2 * H + 1) % (2 * H + 1)][c]; };
            auto vy = [&](int c, int s) -> float2 { return ld2(sl, cen + s * kRowE + c * kTK); };
            auto vyg = [&](int c, int s) -> float2 {
                const int jj = jrow + s;
                if (jrow < g.N1 && (jj < 0 || jj > g.N1 - 1)) {
                    const int side = jj < 0 ? 0 : 1, l = jj < 0 ? -jj : jj - (g.N1 - 1);
                    const int jm = jj < 0 ? l : g.N1 - 1 - l;  // the mirror row, inside the slot
                    const float2 f = ld2(sl, cen + (jm - jrow) * kRowE + c * kTK);
                    return make_float2(wall_ghost(wl, side, c, l, f.x), wall_ghost(wl, side, c, l, f.y));
                }
                return ld2(sl, cen + s * kRowE + c * kTK);
            };
            // odd offsets straddle two loaded pairs (the centre pair is the queue's)
            auto vz = [&](int c, int s) -> float2 {
                const int o = c * kTK;
                switch (s) {
                case -3: return make_float2(ld2(sl, zm4 + o).y, ld2(sl, zm2 + o).x);
                case -2: return ld2(sl, zm2 + o);
                case -1: return make_float2(ld2(sl, zm2 + o).y, q[kC][c].x);
                case 1: return make_float2(q[kC][c].y, ld2(sl, zp2 + o).x);
                case 2: return ld2(sl, zp2 + o);
                case 3: return make_float2(ld2(sl, zp2 + o).y, ld2(sl, zp4 + o).x);
                default: return q[kC][c];
                }
            };
            const float2 u0[3] = {q[kC][0], q[kC][1], q[kC][2]};
            float2 rhs[3];
            if (WALLS && nearw)
                ns_rhs2<H, STRETCH>(vx, vyg, vz, u0, co, sc, iak, c2k, visc, rhs);
            else
                ns_rhs2<H, STRETCH>(vx, vy, vz, u0, co, sc, iak, c2k, visc, rhs);
            release(empty(sCur));  // the slot's values are in registers

            const float2 zz = f2(0.0f);
            float2 e0[3] = {zz, zz, zz}, e1[3] = {zz, zz, zz}, lo[3] = {zz, zz, zz};
            if constexpr (NE > 0) {
                if (!__all_sync(0xffffffffu, mbar_wait(efull(es), eph, err))) return false;
                const T *se = ering + es * NE * kEpiE + r * kRowE + kk;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const int o = c * kTK;
                    if constexpr (STAGE == 1 || STAGE == 2) {
                        e0[c] = ld2(se, o);
                        e1[c] = ld2(se, kEpiE + o);
                    } else if constexpr (STAGE == 3) {
                        e0[c] = ld2(se, o);
                        e1[c] = ld2(se, kEpiE + o);
                        lo[c] = ld2(se, 2 * kEpiE + o);
                    } else if constexpr (STAGE == 4) {
                        lo[c] = ld2(se, o);
                    } else if constexpr (STAGE == 5) {
                        e0[c] = ld2(se, o);
                        lo[c] = ld2(se, kEpiE + o);
                    }
                }
                release(eempty(es));
                if (++es == kERing) {
                    es = 0;
                    eph ^= 1;
                }
            }
            const long long idx = (long long)(ib + p) * g.N12 + (long long)(j0 + r) * g.N2 + k0 + kk;
            if (!WALLS || jrow < g.N1) {
#pragma unroll
                for (int c = 0; c < 3; c++)
                    rk_store32x2<STAGE>(args, (long long)c * g.N3 + idx, u0[c], e0[c], e1[c], lo[c],
                                        mul2(f2(dt), rhs[c]));
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

    if constexpr (DIAG) {
        // consumer warps only (the producer has returned): fixed-order sums
        DiagAccU acc = dacc.load();
        acc.warp_reduce();
        double *red = dred;
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < kDiagParts; q++) red[q * C::kWarps + ty] = acc.part(q);
        asm volatile("bar.sync 1, %0;" ::"n"(C::kWarps * 32) : "memory");
        if (ty == 0 && lane < kDiagParts) {
            double a = 0.0;
            for (int w = 0; w < C::kWarps; w++)
                a = lane >= DP_DIVU ? fmax(a, red[lane * C::kWarps + w]) : a + red[lane * C::kWarps + w];
            const long long blk = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
            dpart[blk * kDiagParts + lane] = a;
        }
    }
}

// ------------------------------------------------------------------ host --
using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeFn encode_fn()
{
    static EncodeFn fn = []() -> EncodeFn {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeFn>(p);
    }();
    return fn;
}

template <typename T> constexpr CUtensorMapDataType tmap_type()
{
    return sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
}

// a 3-component field [c][i][j][k]; rows != 0: dims (k, c, j, i), box kTK x 3 x rows x 1;
// rows == 0: dims (k, j, c, i), box 4 x kLRB x 3 x 1 (the k halos)
template <typename T> bool encode(CUtensorMap *m, const T *base, const Geo &g, unsigned rows)
{
    EncodeFn fn = encode_fn();
    if (!fn || !base) return false;
    const cuuint64_t es = sizeof(T);
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    if (rows) {
        const cuuint64_t d[4] = {(cuuint64_t)g.N2, 3, (cuuint64_t)g.N1, (cuuint64_t)g.N0};
        const cuuint64_t s[3] = {(cuuint64_t)g.N3 * es, (cuuint64_t)g.N2 * es, (cuuint64_t)g.N12 * es};
        const cuuint32_t b[4] = {(cuuint32_t)kTK, 3, rows, 1};
        memcpy(dims, d, sizeof d), memcpy(strides, s, sizeof s), memcpy(box, b, sizeof b);
    } else {
        const cuuint64_t d[4] = {(cuuint64_t)g.N2, (cuuint64_t)g.N1, 3, (cuuint64_t)g.N0};
        const cuuint64_t s[3] = {(cuuint64_t)g.N2 * es, (cuuint64_t)g.N3 * es, (cuuint64_t)g.N12 * es};
        const cuuint32_t b[4] = {4, (cuuint32_t)kLRB, 3, 1};
        memcpy(dims, d, sizeof d), memcpy(strides, s, sizeof s), memcpy(box, b, sizeof b);
    }
    return fn(m, tmap_type<T>(), 4, const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// i-chunk of a TMA stage launch: >= ~4 waves of resident blocks, the 2H-plane
// warm-up kept small against the chunk length
template <typename T> int tma_ichunk(const Geo &g)
{
    using C = TmaCfg<T>;
    const long long tiles = (long long)(g.N2 / kTK) * ((g.N1 + C::TJ - 1) / C::TJ);
    int ch = g.N0;
    while (ch > 16 && tiles * ((g.N0 + ch - 1) / ch) < 148LL * C::kBlocksPerSM * 4) ch /= 2;
    return ch;
}

template <typename T, int STAGE, bool STRETCH, class Args, bool DIAG = false, bool WALLS = false>
cudaError_t launch_tma(const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc, const Args &a,
                       const T *Y, const T *const *ef, int *err, cudaStream_t st, double *dpart = nullptr,
                       const Walls<T> &wl = Walls<T>{})
{
    constexpr int NE = epi_fields<T, STAGE>();
    StageMaps maps;
    memset(&maps, 0, sizeof maps);
    using Cf = TmaCfg<T>;
    bool ok = encode(&maps.tcbA, Y, g, Cf::TJ + 2 * kH) && encode(&maps.tcb3, Y, g, kH) &&
              encode(&maps.tcbB, Y, g, Cf::TJ + kH) && encode(&maps.tcbC, Y, g, Cf::TJ) && encode(&maps.lr, Y, g, 0);
    for (int f = 0; f < NE; f++) ok = ok && encode(&maps.e[f], ef[f], g, Cf::TJ);
    if (!ok) return cudaErrorInvalidValue;
    constexpr size_t smem = tma_smem_bytes<T, NE, DIAG>();
    auto kern = k_stage_tma<T, STAGE, STRETCH, Args, DIAG, WALLS>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        attr = true;
    }
    const int ch = tma_ichunk<T>(g);
    const dim3 grid(g.N2 / kTK, (g.N1 + Cf::TJ - 1) / Cf::TJ, (g.N0 + ch - 1) / ch);
    kern<<<grid, dim3(kTK, Cf::kWarps + 1), smem, st>>>(g, co, stage_coef(co, visc), wl, ia, corr2, dt, visc, a, maps,
                                                     ch, err, dpart);
    return cudaSuccess;
}

template <typename T, bool STRETCH, class Args, bool WALLS>
cudaError_t launch_tma_stage_w(int stage, const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc,
                               const Args &a, const T *const *ef, int *err, cudaStream_t st, const Walls<T> &wl)
{
    switch (stage) {
    case 0: return launch_tma<T, 0, STRETCH, Args, false, WALLS>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st, nullptr, wl);
    case 1: return launch_tma<T, 1, STRETCH, Args, false, WALLS>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st, nullptr, wl);
    case 2: return launch_tma<T, 2, STRETCH, Args, false, WALLS>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st, nullptr, wl);
    case 3: return launch_tma<T, 3, STRETCH, Args, false, WALLS>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st, nullptr, wl);
    case 5: return launch_tma<T, 5, STRETCH, Args, false, WALLS>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st, nullptr, wl);
    default: return launch_tma<T, 4, STRETCH, Args, false, WALLS>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st, nullptr, wl);
    }
}

template <typename T, class Args>
cudaError_t launch_tma_stage(int stage, bool stretch, const Geo &g, const Coef<T> &co, const T *ia, const T *corr2,
                             T dt, T visc, const Args &a, const T *const *ef, int *err, cudaStream_t st,
                             const Walls<T> &wl)
{
    if constexpr (sizeof(T) == 4) {
        if (wl.on)
            return stretch
                       ? launch_tma_stage_w<T, true, Args, true>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st, wl)
                       : launch_tma_stage_w<T, false, Args, true>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st, wl);
    } else {
        if (wl.on) return cudaErrorNotSupported;
    }
    return stretch ? launch_tma_stage_w<T, true, Args, false>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st, wl)
                   : launch_tma_stage_w<T, false, Args, false>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st, wl);
}

}  // namespace

bool tma_encode_field(CUtensorMap *m, const double *base, const Geo &g, unsigned rows)
{
    return encode<double>(m, base, g, rows);
}

bool stage_tma_fits(const Geo &g, bool fp64)
{
    // tile width divides N2 (k halo boxes start at a wrapped column); periodic
    // y: the tile height (16 rows for FP64, 8 for FP32) divides N1 with at
    // most one wrap per tile in j; walls in y (FP32 only: the FP64 wall
    // stages run faster on the march): any N1 of at least two tiles (the
    // last tile may be ragged)
    const int tj = fp64 ? TmaCfg<double>::TJ : TmaCfg<float>::TJ;
    if (g.wallY && fp64) return false;
    return g.N2 % kTK == 0 && g.N1 >= 2 * tj && (g.wallY || g.N1 % tj == 0);
}

cudaError_t launch_stage_tma64(int stage, bool stretch, const Geo &g, const Walls<double> &wl, const Coef<double> &co,
                               const double *ia, const double *corr2, double dt, double visc, const StageArgs64 &a,
                               int *err, cudaStream_t st, const StageDiag *dg, bool *dg_done)
{
    const double *ef[3] = {nullptr, nullptr, nullptr};
    if (stage == 1 || stage == 2) {
        ef[0] = a.U0;
        ef[1] = a.A;
    } else if (stage == 3) {
        ef[0] = a.A;
    } else if (stage == 5) {
        ef[0] = a.U0;
    }
    if (dg && !stretch && !wl.on && (stage == 0 || stage == 4)) {
        using Cf = TmaCfg<double>;
        const int ch = tma_ichunk<double>(g);
        const long long nb = (long long)(g.N2 / kTK) * (g.N1 / Cf::TJ) * ((g.N0 + ch - 1) / ch);
        if (nb <= dg->cap) {
            const cudaError_t e =
                stage == 0 ? launch_tma<double, 0, false, StageArgs64, true>(g, co, ia, corr2, dt, visc, a, a.Y, ef,
                                                                             err, st, dg->part)
                           : launch_tma<double, 4, false, StageArgs64, true>(g, co, ia, corr2, dt, visc, a, a.Y, ef,
                                                                             err, st, dg->part);
            if (e != cudaSuccess) return e;
            launch_diag_final(dg->part, (int)nb, dg->fin, dg->row, dg->flag, st);
            if (dg_done) *dg_done = true;
            return cudaSuccess;
        }
    }
    return launch_tma_stage<double>(stage, stretch, g, co, ia, corr2, dt, visc, a, ef, err, st, wl);
}

cudaError_t launch_stage_tma32(int stage, bool stretch, const Geo &g, const Walls<float> &wl, const Coef<float> &co,
                               const float *ia, const float *corr2, float dt, float visc, const StageArgs32 &a,
                               int *err, cudaStream_t st)
{
    const float *ef[3] = {nullptr, nullptr, nullptr};
    if (stage == 1 || stage == 2) {
        ef[0] = a.U0hi;
        ef[1] = a.A;
    } else if (stage == 3) {
        ef[0] = a.U0hi;
        ef[1] = a.A;
        ef[2] = a.U0lo;
    } else if (stage == 4) {
        ef[0] = a.U0lo;
    } else if (stage == 5) {
        ef[0] = a.U0hi;
        ef[1] = a.U0lo;
    }
    return launch_tma_stage<float>(stage, stretch, g, co, ia, corr2, dt, visc, a, ef, err, st, wl);
}

}  // namespace nova
