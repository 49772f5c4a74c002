// Navier-Stokes stage kernel fed by a TMA pipeline (sm_100a).
//
// Same arithmetic and stage update as the register-queue march of
// nova_stage.cu (nova_stage_math.cuh), different data movement.  A block owns
// a kTK(k) x kTJ(j) column of the grid and walks it along i.  For every plane
// one elected thread issues bulk tensor loads of
//   TCB: the tile's rows plus H halo rows on either side, all three
//        components, laid out [row][c][k] (box 32 x 3 x 14), and
//   L/R: the H-wide k halos left and right of the tile (boxes 4 x 8 x 3,
//        [c][j][k], 4 wide to keep the 16-byte TMA alignment),
// into a ring of kRing shared-memory slots, each completed by an mbarrier
// transaction count, and the pointwise epilogue operands of the plane (RK base
// and accumulator, box 32 x 3 x 8) into a second ring.  Periodic wrap needs
// no ghost storage: in k the halo boxes start at the wrapped column (the tile
// width divides N2), in j a boundary tile's rows arrive as two boxes (3 + 11
// rows) that land back to back in the slot.
//
// The consumer threads keep the i stencil in a register queue (the centre of
// each arriving plane), read the j and k stencils from the slot of the plane
// they are computing, and hand slots back through per-warp arrivals on the
// slot's `empty` barrier.  The producer runs kLookS planes ahead of the queue
// head (kLookS + H ahead of the plane being computed), so HBM latency is
// covered by the ring instead of by the math of one plane.
//
// Every mbarrier wait is bounded (nova_tma.cuh); a wait that gives up raises
// the error word and the block leaves its pipeline after the elected thread
// has waited, again bounded, for the loads it still has in flight.
#include "nova_internal.cuh"
#include "nova_stage_math.cuh"
#include "nova_tile.cuh"
#include "nova_tma.cuh"

#include <cudaTypedefs.h>

#include <cstring>

namespace nova {

namespace {

constexpr int kH = 3;
constexpr int kRing = 6;   // stencil slots: planes p .. p+5 live at step p
constexpr int kLookS = 2;  // stencil loads issued ahead of the queue head
constexpr int kERing = 3;  // epilogue slots
constexpr int kLookE = 2;  // epilogue loads issued ahead of the plane computed
constexpr int kWarps = kThreads / 32;
constexpr int kRowE = 3 * kTK;            // one halo'd row, three components
constexpr int kTcbE = (kTJ + 2 * kH) * kRowE;
constexpr int kLRE = 3 * kTJ * 4;         // one k-halo box
constexpr int kSlotE = kTcbE + 2 * kLRE;  // elements per stencil slot
constexpr int kEpiE = kTJ * kRowE;        // elements per epilogue field
static_assert(kRing >= kLookS + 2 * kH - 2, "a slot is reused only after its plane was computed");
static_assert(kERing >= kLookE + 1, "an epilogue slot is reused only after its plane was stored");
static_assert(kTJ * 4 == kTK, "k-halo boxes share the component stride of the row boxes");

// epilogue operands per stage, in load order
//   FP64:  s=1,2: U0, A   s=3: A
//   split: s=1,2: U0hi, A   s=3: U0hi, A, U0lo   s=4: U0lo
template <typename T, int STAGE> __host__ __device__ constexpr int epi_fields()
{
    if constexpr (sizeof(T) == 8)
        return (STAGE == 1 || STAGE == 2) ? 2 : (STAGE == 3 ? 1 : 0);
    else
        return (STAGE == 1 || STAGE == 2) ? 2 : (STAGE == 3 ? 3 : (STAGE == 4 ? 1 : 0));
}

template <typename T, int NE> constexpr size_t tma_smem_bytes()
{
    return ((size_t)kRing * kSlotE + (size_t)kERing * NE * kEpiE) * sizeof(T) + 8 * (2 * kRing + 2 * kERing);
}

struct StageMaps {
    CUtensorMap tcb14, tcb3, tcb11;  // halo'd rows of the stencil field: 14, 3 or 11 rows
    CUtensorMap lr;                  // k-halo boxes of the stencil field
    CUtensorMap e[3];                // epilogue operands
};

template <typename T, int STAGE>
__device__ __forceinline__ void epi_read(const T *se, int c, T &e0, T &e1, T &lo)
{
    if constexpr (STAGE == 1 || STAGE == 2) {
        e0 = se[c * kTK];
        e1 = se[kEpiE + c * kTK];
    } else if constexpr (STAGE == 3) {
        if constexpr (sizeof(T) == 8) {
            e1 = se[c * kTK];
        } else {
            e0 = se[c * kTK];
            e1 = se[kEpiE + c * kTK];
            lo = se[2 * kEpiE + c * kTK];
        }
    } else if constexpr (STAGE == 4 && sizeof(T) == 4) {
        lo = se[c * kTK];
    }
}

// resident blocks per SM: FP64 two (registers), FP32 three (shared memory of the rings)
template <typename T> __host__ __device__ constexpr int tma_blocks_per_sm() { return sizeof(T) == 8 ? 2 : 3; }

template <typename T, int STAGE, bool STRETCH, class Args>
__global__ void __launch_bounds__(kThreads, tma_blocks_per_sm<T>())
    k_stage_tma(Geo g, Coef<T> co, const T *__restrict__ ia, const T *__restrict__ corr2, T dt, T visc, Args args,
                const __grid_constant__ StageMaps maps, int ichunk, int *err)
{
    constexpr int H = kH;
    constexpr int NE = epi_fields<T, STAGE>();
    constexpr uint32_t kSlotBytes = kSlotE * sizeof(T), kRowBytes = kRowE * sizeof(T), kEpiBytes = kEpiE * sizeof(T);
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

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTK + tx, lane = tid & 31;
    const bool lead = tid == 0;
    const int k0 = blockIdx.x * kTK, j0 = blockIdx.y * kTJ;
    const int ib = blockIdx.z * ichunk, ie = min(ib + ichunk, g.N0);
    const int nout = ie - ib, nld = nout + 2 * H;

    if (lead) {
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

    // ---- producer (the elected thread) ----
    const bool jlo = j0 < H, jhi = j0 + kTJ + H > g.N1;
    const int kl = (k0 == 0 ? g.N2 : k0) - 4, kr = (k0 + kTK == g.N2) ? 0 : k0 + kTK;
    int iss = 0, ise = 0;  // loads issued
    bool ok = true;
    auto issue_s = [&](int n) -> bool {  // stencil load n: plane ib - H + n
        const int r = n % kRing;
        if (n >= kRing && !mbar_wait(empty(r), ((n / kRing) + 1) & 1, err)) return false;
        const uint32_t dst = s0 + r * kSlotBytes, bar = full(r);
        mbar_expect_tx(bar, kSlotBytes);
        const int plane = wrapi(ib - H + n, g.N0);
        if (jlo) {
            tma_load_4d(dst, &maps.tcb3, bar, k0, 0, g.N1 - H, plane);
            tma_load_4d(dst + H * kRowBytes, &maps.tcb11, bar, k0, 0, 0, plane);
        } else if (jhi) {
            tma_load_4d(dst, &maps.tcb11, bar, k0, 0, j0 - H, plane);
            tma_load_4d(dst + (kTJ + H) * kRowBytes, &maps.tcb3, bar, k0, 0, 0, plane);
        } else {
            tma_load_4d(dst, &maps.tcb14, bar, k0, 0, j0 - H, plane);
        }
        tma_load_4d(dst + kTcbE * sizeof(T), &maps.lr, bar, kl, j0, 0, plane);
        tma_load_4d(dst + (kTcbE + kLRE) * sizeof(T), &maps.lr, bar, kr, j0, 0, plane);
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
    auto produce = [&](int s_upto, int e_upto) {
        while (ok && iss < min(s_upto, nld)) {
            if (issue_s(iss)) iss++; else ok = false;
        }
        if constexpr (NE > 0) {
            while (ok && ise < min(e_upto, nout)) {
                if (issue_e(ise)) ise++; else ok = false;
            }
        }
    };
    auto release = [&](uint32_t bar) {
        __syncwarp();
        if (lane == 0) mbar_arrive(bar);
    };

    // ---- consumers (all threads) ----
    const int kw = k0 + tx;
    const T iak = ia[kw];
    const T c2k = STRETCH ? corr2[kw] : T(0);

    // slot offsets: centre, and the k neighbours at s = -3..-1, 1..3 (inside
    // the row box or in the left/right halo box); component stride kTK in both
    const int cen = (H + ty) * kRowE + tx;
    int oz[2 * H];
#pragma unroll
    for (int u = 0; u < 2 * H; u++) {
        const int s = u < H ? u - H : u - H + 1;
        const int x = tx + s;
        oz[u] = x < 0 ? kTcbE + ty * 4 + 4 + x : (x >= kTK ? kTcbE + kLRE + ty * 4 + (x - kTK) : cen + s);
    }

    T q[2 * H + 1][3];
    int cs = 0, ce = 0;  // loads waited for (the elected thread's drain bound)
    if (lead) produce(kLookS + 1, kLookE);
    for (int n = 0; n < 2 * H; n++) {  // queue: planes ib-3 .. ib+2
        if (lead) produce(n + kLookS + 1, kLookE);
        ok = ok && mbar_wait(full(n % kRing), (n / kRing) & 1, err);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        cs = n + 1;
        const T *sl = ring + (n % kRing) * kSlotE;
#pragma unroll
        for (int c = 0; c < 3; c++) q[n + 1][c] = sl[cen + c * kTK];
        if (n < H || n >= H + nout) release(empty(n % kRing));  // queue-only plane
    }

    for (int p = 0; p < nout && ok; p++) {
        const int hd = p + 2 * H;  // queue head: plane ib + p + 3
        if (lead) produce(hd + kLookS + 1, p + kLookE + 1);
        ok = ok && mbar_wait(full(hd % kRing), (hd / kRing) & 1, err);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        cs = hd + 1;
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
        auto vz = [&](int c, int s) -> T {
            return s == 0 ? sl[cen + c * kTK] : sl[oz[s < 0 ? s + H : s + H - 1] + c * kTK];
        };
        const T u0[3] = {q[H][0], q[H][1], q[H][2]};
        T rhs[3];
        ns_rhs<T, H, STRETCH>(vx, vy, vz, u0, co, iak, c2k, visc, rhs);

        T e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
        if constexpr (NE > 0) {
            ok = ok && mbar_wait(efull(p % kERing), (p / kERing) & 1, err);
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
            ce = p + 1;
            const T *se = ering + (p % kERing) * NE * kEpiE + ty * kRowE + tx;
#pragma unroll
            for (int c = 0; c < 3; c++) epi_read<T, STAGE>(se, c, e0[c], e1[c], lo[c]);
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
        if constexpr (NE > 0) release(eempty(p % kERing));
        release(empty(cur % kRing));
    }

    if (lead && !ok) {
        // loads issued but not waited for are still landing in this block's shared memory
        for (int n = cs; n < iss; n++) mbar_wait(full(n % kRing), (n / kRing) & 1, err, true);
        for (int n = ce; n < ise; n++) mbar_wait(efull(n % kERing), (n / kERing) & 1, err, true);
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

// a 3-component field [c][i][j][k]; rows != 0: dims (k, c, j, i), box kTK x 3 x rows;
// rows == 0: dims (k, j, c, i), box 4 x kTJ x 3 (the k halos)
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
        const cuuint32_t b[4] = {4, (cuuint32_t)kTJ, 3, 1};
        memcpy(dims, d, sizeof d), memcpy(strides, s, sizeof s), memcpy(box, b, sizeof b);
    }
    return fn(m, tmap_type<T>(), 4, const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, int STAGE, bool STRETCH, class Args>
cudaError_t launch_tma(const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc, const Args &a,
                       const T *Y, const T *const *ef, int *err, cudaStream_t st)
{
    constexpr int NE = epi_fields<T, STAGE>();
    StageMaps maps;
    memset(&maps, 0, sizeof maps);
    bool ok = encode(&maps.tcb14, Y, g, kTJ + 2 * kH) && encode(&maps.tcb3, Y, g, kH) &&
              encode(&maps.tcb11, Y, g, kTJ + kH) && encode(&maps.lr, Y, g, 0);
    for (int f = 0; f < NE; f++) ok = ok && encode(&maps.e[f], ef[f], g, kTJ);
    if (!ok) return cudaErrorInvalidValue;
    constexpr size_t smem = tma_smem_bytes<T, NE>();
    auto kern = k_stage_tma<T, STAGE, STRETCH, Args>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        attr = true;
    }
    const int ch = pick_ichunk(g, tma_blocks_per_sm<T>());
    kern<<<tile_grid(g, ch), dim3(kTK, kTJ), smem, st>>>(g, co, ia, corr2, dt, visc, a, maps, ch, err);
    return cudaSuccess;
}

template <typename T, bool STRETCH, class Args>
cudaError_t launch_tma_stage(int stage, const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc,
                             const Args &a, const T *const *ef, int *err, cudaStream_t st)
{
    switch (stage) {
    case 0: return launch_tma<T, 0, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st);
    case 1: return launch_tma<T, 1, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st);
    case 2: return launch_tma<T, 2, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st);
    case 3: return launch_tma<T, 3, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st);
    default: return launch_tma<T, 4, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, ef, err, st);
    }
}

}  // namespace

bool stage_tma_fits(const Geo &g)
{
    // tile width divides N2 (k halo boxes start at a wrapped column), tile
    // height divides N1 with at most one wrap per tile in j, periodic y
    return !g.wallY && g.N2 % kTK == 0 && g.N1 % kTJ == 0 && g.N1 >= 2 * kTJ;
}

cudaError_t launch_stage_tma64(int stage, bool stretch, const Geo &g, const Coef<double> &co, const double *ia,
                               const double *corr2, double dt, double visc, const StageArgs64 &a, int *err,
                               cudaStream_t st)
{
    const double *ef[3] = {nullptr, nullptr, nullptr};
    if (stage == 1 || stage == 2) {
        ef[0] = a.U0;
        ef[1] = a.A;
    } else if (stage == 3) {
        ef[0] = a.A;
    }
    return stretch ? launch_tma_stage<double, true>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st)
                   : launch_tma_stage<double, false>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st);
}

cudaError_t launch_stage_tma32(int stage, bool stretch, const Geo &g, const Coef<float> &co, const float *ia,
                               const float *corr2, float dt, float visc, const StageArgs32 &a, int *err,
                               cudaStream_t st)
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
    }
    return stretch ? launch_tma_stage<float, true>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st)
                   : launch_tma_stage<float, false>(stage, g, co, ia, corr2, dt, visc, a, ef, err, st);
}

}  // namespace nova
