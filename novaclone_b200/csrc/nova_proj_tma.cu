// Projection kernels fed by the warp-specialised TMA pipeline of the stage
// kernel (nova_stage_tma.cu): the same producer warp, mbarrier rings and
// periodic wrap by split boxes, with the per-component boxes each operator
// needs (src/ex/div/div.hxx:22-81, src/ex/grad/grad.cpp:25-62):
//   DIV:  rhs = div(U*)/divisor = (D_x U*_0 + D_y U*_1 + D_z U*_2) / divisor
//         slot = U_0 tile rows (the i stencil, kept in a register queue),
//                U_1 rows with their 3-row j halos, U_2 rows with 4-wide k halos
//   CORR: U = U* - s grad(p)
//         slot = p rows with j halos and k halos; epilogue ring = U* (3 components)
// FP32-split fields arrive as hi and lo boxes and are joined in FP64 as the
// march kernels do ((double)hi + (double)lo), so both produce the same bits.
// WALLS (walls on the y nodes j = 0 and j = N1 - 1): the j-halo rows arrive
// as one box from j0 - 3 (rows outside 0..N1-1 zero filled, the last tile
// may be ragged); in the warps of rows within 3 of a wall, a j neighbour
// across the wall is the wall_ghost of its mirror row (the field's BC: U*'s
// component 1 for DIV, p for CORR), the formula of the tiled kernels; rows
// past N1 - 1 store nothing.
// Every mbarrier wait is bounded (nova_tma.cuh).
#include "nova_internal.cuh"
#include "nova_tma.cuh"

#include <cudaTypedefs.h>

#include <cstring>
#include <type_traits>

namespace nova {

namespace {

constexpr int kH = 3;
constexpr int TJ = 16;                  // tile rows: one consumer warp per row
constexpr int kWarps = TJ;
constexpr int kThreads = kTK * (TJ + 1);  // plus the producer warp
constexpr int kRing = 7;
constexpr int kERing = 3;
constexpr int kLRB = 8;                 // rows of one k-halo box
constexpr int kRowsE = (TJ + 2 * kH) * kTK;  // a component's rows with the j halos
constexpr int kTileE = TJ * kTK;             // a component's tile rows
constexpr int kLRE = TJ * 4;                 // one side's k halo of a component

// PROJ_CORR_MIX: the correction of an FP32-split state whose U* arrives in FP64
enum ProjMode { PROJ_DIV = 0, PROJ_CORR = 1, PROJ_CORR_MIX = 2 };

// map indices
enum {
    M_C0 = 0,   // DIV: component 0 tile (box 32 x TJ); CORR: p's tile rows (the queue-only planes)
    M_RA = 1,   // rows with j halos: TJ + 6, 3, TJ + 3 rows (DIV: component 1, CORR: p)
    M_R3 = 2,
    M_RB = 3,
    M_C2 = 4,   // DIV: component 2 tile
    M_LR = 5,   // k halo boxes (4 x 8) (DIV: component 2, CORR: p)
    M_SET = 6,  // maps per field set (DIV split: hi set, then lo set)
    M_EPI = 12  // CORR: U* (box 32 x 3 x TJ), U*lo at M_EPI + 1
};

struct ProjMaps {
    CUtensorMap m[14];
};

template <int MODE, bool SPLIT> struct ProjCfg {
    static constexpr bool kDivLoads = MODE == PROJ_DIV;
    using TS = typename std::conditional<kDivLoads && SPLIT, float, double>::type;  // stencil element
    using TE = typename std::conditional<SPLIT && MODE == PROJ_CORR, float, double>::type;  // U* element
    static constexpr int kSets = (kDivLoads && SPLIT) ? 2 : 1;
    // elements of one set: DIV c0 tile | c1 rows | c2 tile | L | R;  CORR p rows | L | R
    static constexpr int kSetE = kDivLoads ? kTileE + kRowsE + kTileE + 2 * kLRE : kRowsE + 2 * kLRE;
    static constexpr int kSlotE = kSets * kSetE;
    static constexpr uint32_t kSlotBytes = kSlotE * sizeof(TS);
    static constexpr int kNE = MODE == PROJ_CORR ? (SPLIT ? 2 : 1) : (MODE == PROJ_CORR_MIX ? 1 : 0);  // epilogue fields
    static constexpr int kEpiE = 3 * kTileE;
    static constexpr uint32_t kEpiBytes = kEpiE * sizeof(TE);
    static constexpr size_t kSmem =
        (size_t)kRing * kSlotBytes + (size_t)kERing * kNE * kEpiBytes + 8 * 2 * (kRing + kERing) + 16 * kWarps;
};

struct ProjArgs {
    double divisor, s;
    double *rhs;                // DIV output
    double *U64;                // CORR output (FP64)
    float *hi, *lo;             // CORR output (split)
};

template <int MODE, bool SPLIT, bool WALLS>
__global__ void __launch_bounds__(kThreads, 2)
    k_proj_tma(Geo g, Coef<double> co, const Walls<double> wl, const double *__restrict__ ia, ProjArgs a,
               const __grid_constant__ ProjMaps maps, int ichunk, int *err)
{
    using C = ProjCfg<MODE, SPLIT>;
    using TS = typename C::TS;
    using TE = typename C::TE;
    constexpr int H = kH, NE = C::kNE;
    constexpr uint32_t kRowBytes = kTK * sizeof(TS);
    extern __shared__ __align__(128) unsigned char smraw[];
    const TS *ring = reinterpret_cast<const TS *>(smraw);
    const TE *ering = reinterpret_cast<const TE *>(smraw + kRing * C::kSlotBytes);
    const uint32_t s0 = smem_addr(smraw);
    const uint32_t e0addr = s0 + kRing * C::kSlotBytes;
    const uint32_t bar0 = e0addr + kERing * NE * C::kEpiBytes;
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

    // ---- producer warp ----
    if (ty == TJ) {
        if (lane != 0) return;
        const bool jlo = j0 < H, jhi = j0 + TJ + H > g.N1;
        const int kl = (k0 == 0 ? g.N2 : k0) - 4, kr = (k0 + kTK == g.N2) ? 0 : k0 + kTK;
        // rows with j halos of map set `ms` into dst
        auto rows = [&](int ms, uint32_t dst, uint32_t bar, int plane) {
            if (WALLS) {
                tma_load_3d(dst, &maps.m[ms + M_RA], bar, k0, j0 - H, plane);
            } else if (jlo) {
                tma_load_3d(dst, &maps.m[ms + M_R3], bar, k0, g.N1 - H, plane);
                tma_load_3d(dst + H * kRowBytes, &maps.m[ms + M_RB], bar, k0, 0, plane);
            } else if (jhi) {
                tma_load_3d(dst, &maps.m[ms + M_RB], bar, k0, j0 - H, plane);
                tma_load_3d(dst + (TJ + H) * kRowBytes, &maps.m[ms + M_R3], bar, k0, 0, plane);
            } else {
                tma_load_3d(dst, &maps.m[ms + M_RA], bar, k0, j0 - H, plane);
            }
        };
        auto halos = [&](int ms, uint32_t dstL, uint32_t bar, int plane) {
#pragma unroll
            for (int b = 0; b < TJ / kLRB; b++) {
                const uint32_t off = b * kLRB * 4 * sizeof(TS);
                tma_load_3d(dstL + off, &maps.m[ms + M_LR], bar, kl, j0 + b * kLRB, plane);
                tma_load_3d(dstL + kLRE * sizeof(TS) + off, &maps.m[ms + M_LR], bar, kr, j0 + b * kLRB, plane);
            }
        };
        auto issue_s = [&](int n) -> bool {  // stencil load n: plane ib - H + n
            const int r = n % kRing;
            if (n >= kRing && !mbar_wait(empty(r), ((n / kRing) + 1) & 1, err)) return false;
            const uint32_t bar = full(r);
            const int plane = wrapi(ib - H + n, g.N0);
            if (n < H || n >= H + nout) {
                // a queue-only plane: the consumers read the i-stencil component's
                // tile rows alone (DIV: component 0 at the set's start; CORR: p's
                // rows at their place after the H halo rows)
                mbar_expect_tx(bar, C::kSets * kTileE * sizeof(TS));
#pragma unroll
                for (int set = 0; set < C::kSets; set++) {
                    const uint32_t dst = s0 + r * C::kSlotBytes + set * C::kSetE * sizeof(TS);
                    tma_load_3d(C::kDivLoads ? dst : dst + H * kRowBytes, &maps.m[set * M_SET + M_C0], bar, k0, j0,
                                plane);
                }
                return true;
            }
            mbar_expect_tx(bar, C::kSlotBytes);
#pragma unroll
            for (int set = 0; set < C::kSets; set++) {
                const uint32_t dst = s0 + r * C::kSlotBytes + set * C::kSetE * sizeof(TS);
                const int ms = set * M_SET;
                if constexpr (C::kDivLoads) {
                    tma_load_3d(dst, &maps.m[ms + M_C0], bar, k0, j0, plane);
                    rows(ms, dst + kTileE * sizeof(TS), bar, plane);
                    tma_load_3d(dst + (kTileE + kRowsE) * sizeof(TS), &maps.m[ms + M_C2], bar, k0, j0, plane);
                    halos(ms, dst + (2 * kTileE + kRowsE) * sizeof(TS), bar, plane);
                } else {
                    rows(ms, dst, bar, plane);
                    halos(ms, dst + kRowsE * sizeof(TS), bar, plane);
                }
            }
            return true;
        };
        auto issue_e = [&](int n) -> bool {  // epilogue load n: plane ib + n
            const int r = n % kERing;
            if (n >= kERing && !mbar_wait(eempty(r), ((n / kERing) + 1) & 1, err)) return false;
            const uint32_t dst = e0addr + r * NE * C::kEpiBytes, bar = efull(r);
            mbar_expect_tx(bar, NE * C::kEpiBytes);
#pragma unroll
            for (int f = 0; f < NE; f++) tma_load_4d(dst + f * C::kEpiBytes, &maps.m[M_EPI + f], bar, k0, 0, j0, ib + n);
            return true;
        };
        int iss = 0, ise = 0;
        bool ok = true;
        for (int t = -2 * H; t < nout && ok; t++) {
            if ((ok = issue_s(t + 2 * H))) iss++;
            if (NE > 0 && ok && t >= 0 && (ok = issue_e(t))) ise++;
        }
        if (!ok) {
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
    double az[H];
#pragma unroll
    for (int l = 0; l < H; l++) az[l] = co.a[2][l] * ia[kw];
    // set-relative element offsets of this thread
    constexpr bool DL = C::kDivLoads;
    constexpr int oQ = DL ? 0 : H * kTK;                    // queue value (row ty of the tile)
    constexpr int oY = DL ? kTileE + H * kTK : H * kTK;     // j stencil centre
    constexpr int oZ = DL ? kTileE + kRowsE : H * kTK;      // k stencil centre row
    constexpr int oL = DL ? 2 * kTileE + kRowsE : kRowsE;   // left k halo
    const int qoff = oQ + ty * kTK + tx, yoff = oY + ty * kTK + tx;
    // walls: this warp's row, and whether its j stencil reaches across a wall
    // (the component whose j derivative is taken: U*_1 for DIV, p for CORR)
    constexpr int CY = MODE == PROJ_DIV ? 1 : 0;
    const int jrow = j0 + ty;
    const bool nearw = WALLS && jrow < g.N1 && (jrow < H || jrow + H > g.N1 - 1);
    auto zoff = [&](int s) -> int {
        const int x = tx + s;
        return x < 0 ? oL + ty * 4 + 4 + x : (x >= kTK ? oL + kLRE + ty * 4 + (x - kTK) : oZ + ty * kTK + x);
    };
    auto val = [&](const TS *sl, int o) -> double {
        if constexpr (C::kSets == 2)
            return (double)sl[o] + (double)sl[C::kSetE + o];
        else
            return (double)sl[o];
    };

    double q[2 * H + 1];
    bool ok = true;
    for (int n = 0; n < 2 * H; n++) {
        ok = mbar_wait(full(n % kRing), (n / kRing) & 1, err);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        q[n + 1] = val(ring + (n % kRing) * C::kSlotE, qoff);
        if (n < H || n >= H + nout) release(empty(n % kRing));
    }
    for (int p = 0; p < nout && ok; p++) {
        const int hd = p + 2 * H;
        ok = mbar_wait(full(hd % kRing), (hd / kRing) & 1, err);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
#pragma unroll
        for (int s = 0; s < 2 * H; s++) q[s] = q[s + 1];
        q[2 * H] = val(ring + (hd % kRing) * C::kSlotE, qoff);
        if (hd >= H + nout) release(empty(hd % kRing));

        const int cur = p + H;
        const TS *sl = ring + (cur % kRing) * C::kSlotE;
        auto vx = [&](int, int s) -> double { return q[H + s]; };
        auto vy = [&](int, int s) -> double { return val(sl, yoff + s * kTK); };
        auto vyg = [&](int, int s) -> double {
            const int jj = jrow + s;
            if (jj < 0 || jj > g.N1 - 1) {
                const int side = jj < 0 ? 0 : 1, l = jj < 0 ? -jj : jj - (g.N1 - 1);
                const int jm = jj < 0 ? l : g.N1 - 1 - l;  // the mirror row, inside the slot
                return wall_ghost(wl, side, CY, l, val(sl, yoff + (jm - jrow) * kTK));
            }
            return val(sl, yoff + s * kTK);
        };
        auto vz = [&](int, int s) -> double { return val(sl, zoff(s)); };
        const double dy = (WALLS && nearw) ? d1<double, H>(vyg, CY, co.a[1]) : d1<double, H>(vy, CY, co.a[1]);
        const bool store = !WALLS || jrow < g.N1;
        const long long idx = (long long)(ib + p) * g.N12 + (long long)(j0 + ty) * g.N2 + kw;
        if constexpr (MODE == PROJ_DIV) {
            const double d = d1<double, H>(vx, 0, co.a[0]) + dy + d1<double, H>(vz, 2, az);
            release(empty(cur % kRing));  // the slot's values are in registers
            if (store) a.rhs[idx] = d / a.divisor;
        } else {
            const double gr[3] = {d1<double, H>(vx, 0, co.a[0]), dy, d1<double, H>(vz, 0, az)};
            release(empty(cur % kRing));  // the slot's values are in registers
            ok = mbar_wait(efull(p % kERing), (p / kERing) & 1, err);
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
            const TE *se = ering + (p % kERing) * NE * C::kEpiE + ty * 3 * kTK + tx;
            double us[3];
#pragma unroll
            for (int c = 0; c < 3; c++)
                us[c] = (SPLIT && MODE == PROJ_CORR) ? (double)se[c * kTK] + (double)se[C::kEpiE + c * kTK]
                                                     : (double)se[c * kTK];
            release(eempty(p % kERing));
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (!store) break;
                const long long o = (long long)c * g.N3 + idx;
                const double x = us[c] - gr[c] * a.s;
                if constexpr (SPLIT) {
                    const float h = (float)x;
                    a.hi[o] = h;
                    a.lo[o] = (float)(x - (double)h);
                } else {
                    a.U64[o] = x;
                }
            }
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

// one component (dims k, j, i) with box bk x bj x 1
template <typename T> bool encode3(CUtensorMap *m, const T *base, const Geo &g, unsigned bk, unsigned bj)
{
    EncodeFn fn = encode_fn();
    if (!fn || !base) return false;
    const cuuint64_t es = sizeof(T);
    const cuuint64_t dims[3] = {(cuuint64_t)g.N2, (cuuint64_t)g.N1, (cuuint64_t)g.N0};
    const cuuint64_t strides[2] = {(cuuint64_t)g.N2 * es, (cuuint64_t)g.N12 * es};
    const cuuint32_t box[3] = {bk, bj, 1}, estr[3] = {1, 1, 1};
    return fn(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
              const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// three components (dims k, c, j, i) with box kTK x 3 x TJ x 1 (the epilogue operands)
template <typename T> bool encode4(CUtensorMap *m, const T *base, const Geo &g)
{
    EncodeFn fn = encode_fn();
    if (!fn || !base) return false;
    const cuuint64_t es = sizeof(T);
    const cuuint64_t dims[4] = {(cuuint64_t)g.N2, 3, (cuuint64_t)g.N1, (cuuint64_t)g.N0};
    const cuuint64_t strides[3] = {(cuuint64_t)g.N3 * es, (cuuint64_t)g.N2 * es, (cuuint64_t)g.N12 * es};
    const cuuint32_t box[4] = {(cuuint32_t)kTK, 3, (cuuint32_t)TJ, 1}, estr[4] = {1, 1, 1, 1};
    return fn(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
              const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the row maps (TJ + 6, 3, TJ + 3 rows) of one scalar field, at set offset ms
template <typename T> bool encode_rows(ProjMaps &pm, int ms, const T *f, const Geo &g)
{
    return encode3(&pm.m[ms + M_RA], f, g, kTK, TJ + 2 * kH) && encode3(&pm.m[ms + M_R3], f, g, kTK, kH) &&
           encode3(&pm.m[ms + M_RB], f, g, kTK, TJ + kH);
}

// i-chunk: at least `waves` waves of the 2 resident blocks per SM.  The 2H
// warm-up planes of a chunk load the queue's tile rows alone; for DIV that is
// a third of the slot (component 0's tile is in every slot), so its longer
// chunks (2 waves at 256^3) win, while the correction's p rows and halos make
// shorter chunks with a smaller last wave pay (4 waves: 156 -> 146 us at 256^3,
// DIV 115 -> 120 us)
int proj_ichunk(const Geo &g, int waves)
{
    const long long tiles = (long long)(g.N2 / kTK) * ((g.N1 + TJ - 1) / TJ);
    int ch = g.N0;
    while (ch > 16 && tiles * ((g.N0 + ch - 1) / ch) < 148LL * 2 * waves) ch /= 2;
    return ch;
}

template <int MODE, bool SPLIT, bool WALLS>
cudaError_t launch_w(const Geo &g, const Coef<double> &co, const Walls<double> &wl, const double *ia,
                     const ProjArgs &a, const ProjMaps &pm, int *err, cudaStream_t st)
{
    using C = ProjCfg<MODE, SPLIT>;
    auto kern = k_proj_tma<MODE, SPLIT, WALLS>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::kSmem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        attr = true;
    }
    const int ch = proj_ichunk(g, MODE == PROJ_DIV ? 2 : 4);
    const dim3 grid(g.N2 / kTK, (g.N1 + TJ - 1) / TJ, (g.N0 + ch - 1) / ch);
    kern<<<grid, dim3(kTK, TJ + 1), C::kSmem, st>>>(g, co, wl, ia, a, pm, ch, err);
    return cudaSuccess;
}

template <int MODE, bool SPLIT>
cudaError_t launch(const Geo &g, const Coef<double> &co, const Walls<double> &wl, const double *ia,
                   const ProjArgs &a, const ProjMaps &pm, int *err, cudaStream_t st)
{
    return wl.on ? launch_w<MODE, SPLIT, true>(g, co, wl, ia, a, pm, err, st)
                 : launch_w<MODE, SPLIT, false>(g, co, wl, ia, a, pm, err, st);
}

}  // namespace

// tile width divides N2; periodic y: the tile height divides N1; walls in y
// (the field's ghost BCs on, wl_on): any N1 of at least two tiles
bool proj_tma_fits(const Geo &g, bool wl_on)
{
    if (wl_on != (g.wallY != 0)) return false;
    return g.N2 % kTK == 0 && g.N1 >= 2 * TJ && (g.wallY || g.N1 % TJ == 0);
}

cudaError_t launch_div_tma(const Geo &g, const Coef<double> &co, const Walls<double> &wl, const double *ia,
                           const double *U64, const float *hi, const float *lo, double divisor, double *rhs, int *err,
                           cudaStream_t st)
{
    ProjMaps pm;
    memset(&pm, 0, sizeof pm);
    ProjArgs a{};
    a.divisor = divisor;
    a.rhs = rhs;
    // component 0: tile rows (i stencil), 1: rows with j halos, 2: tile rows and k halos
    auto set_maps = [&](int ms, const auto *f) {
        return encode3(&pm.m[ms + M_C0], f, g, kTK, TJ) && encode_rows(pm, ms, f + g.N3, g) &&
               encode3(&pm.m[ms + M_C2], f + 2 * g.N3, g, kTK, TJ) &&
               encode3(&pm.m[ms + M_LR], f + 2 * g.N3, g, 4, kLRB);
    };
    if (U64) {
        if (!set_maps(0, U64)) return cudaErrorInvalidValue;
        return launch<PROJ_DIV, false>(g, co, wl, ia, a, pm, err, st);
    }
    const bool ok = set_maps(0, hi) && set_maps(M_SET, lo);
    if (!ok) return cudaErrorInvalidValue;
    return launch<PROJ_DIV, true>(g, co, wl, ia, a, pm, err, st);
}

cudaError_t launch_correct_tma(const Geo &g, const Coef<double> &co, const Walls<double> &pw, const double *ia,
                               const double *p, double s, const double *Us64, double *U64, const float *Ushi,
                               const float *Uslo, float *hi, float *lo, int *err, cudaStream_t st)
{
    ProjMaps pm;
    memset(&pm, 0, sizeof pm);
    ProjArgs a{};
    a.s = s;
    a.U64 = U64;
    a.hi = hi;
    a.lo = lo;
    bool ok = encode_rows(pm, 0, p, g) && encode3(&pm.m[M_LR], p, g, 4, kLRB) && encode3(&pm.m[M_C0], p, g, kTK, TJ);
    if (Us64 && hi) {  // FP64 U*, FP32-split output
        ok = ok && encode4(&pm.m[M_EPI], Us64, g);
        if (!ok) return cudaErrorInvalidValue;
        return launch<PROJ_CORR_MIX, true>(g, co, pw, ia, a, pm, err, st);
    }
    if (Us64) {
        ok = ok && encode4(&pm.m[M_EPI], Us64, g);
        if (!ok) return cudaErrorInvalidValue;
        return launch<PROJ_CORR, false>(g, co, pw, ia, a, pm, err, st);
    }
    ok = ok && encode4(&pm.m[M_EPI], Ushi, g) && encode4(&pm.m[M_EPI + 1], Uslo, g);
    if (!ok) return cudaErrorInvalidValue;
    return launch<PROJ_CORR, true>(g, co, pw, ia, a, pm, err, st);
}

}  // namespace nova
