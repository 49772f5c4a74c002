// MHD stage kernels fed by a TMA pipeline (sm_100a): the U loop
// (app/OT_Poisson/UEqn.H:16-31, B frozen) and the B loop (BEqn.H:15-35, U
// frozen), the same arithmetic (nova_stage_math.cuh: mhd_u_rhs, mhd_b_rhs)
// and stage update as the register-queue march of nova_stage.cu.
//
// The pipeline is the Navier-Stokes one of nova_stage_tma.cu with two halo'd
// fields per plane: a block owns a kTK(k) x TJ(j) column and walks it along i;
// its producer warp loads, for every plane, each field's tile rows with their
// H halo rows on either side (box 32 x 3 x rows, [row][c][k]) and its 4-wide
// k halos (boxes 4 x 8 x 3, [c][j][k]) into one slot of a kRing-slot shared
// ring, and the pointwise epilogue operands into a second ring; the consumer
// warps keep the six components' i stencil in a register queue and read the j
// and k stencils from the slot.  Periodic wrap: k halo boxes start at the
// wrapped column (the tile width divides N2), a boundary tile's j rows arrive
// as two boxes.  Every mbarrier wait is bounded (nova_tma.cuh).
//
// FP64: TJ = 8 (a slot of the two fields is 24 KB, 209 KB with the epilogue
// ring; one block of 9 warps per SM, up to 224 registers a thread); FP32:
// TJ = 16 (20 KB slots, 195 KB; one block of 17 warps).
#include "nova_internal.cuh"
#include "nova_stage_math.cuh"
#include "nova_tma.cuh"

#include <cudaTypedefs.h>

#include <cstring>
#include <type_traits>

namespace nova {

namespace {

constexpr int kH = 3;
constexpr int kRowE = 3 * kTK;  // one halo'd row of one field, three components
constexpr int kLRB = 8;         // rows of one k-halo box

template <typename T> struct MhdCfg {
    static constexpr int TJ = sizeof(T) == 8 ? 8 : 16;
    static constexpr int kWarps = TJ;
    static constexpr int kThreads = kTK * (TJ + 1);
    static constexpr int kRing = 7;
    static constexpr int kERing = 3;
    static constexpr int kTcbE = (TJ + 2 * kH) * kRowE;  // one field's halo'd rows
    static constexpr int kLRE = 3 * TJ * 4;              // one field's k halo, one side
    static constexpr int kFieldE = kTcbE + 2 * kLRE;
    static constexpr int kSlotE = 2 * kFieldE;           // the stage field, then the frozen one
    static constexpr int kEpiE = TJ * kRowE;
    static_assert(TJ % kLRB == 0 && kLRB * 4 == kTK, "k-halo boxes share the component stride of the row boxes");
};

// epilogue operands per stage, in load order (as nova_stage_tma.cu):
//   FP64:  s=1,2: U0, A   s=3: A
//   split: s=1,2: U0hi, A   s=3: U0hi, A, U0lo   s=4: U0lo
template <typename T, int STAGE> __host__ __device__ constexpr int mhd_epi_fields()
{
    if constexpr (sizeof(T) == 8)
        return (STAGE == 1 || STAGE == 2) ? 2 : (STAGE == 3 ? 1 : 0);
    else
        return (STAGE == 1 || STAGE == 2) ? 2 : (STAGE == 3 ? 3 : (STAGE == 4 ? 1 : 0));
}

template <typename T, int NE> constexpr size_t mhd_smem_bytes()
{
    using C = MhdCfg<T>;
    return ((size_t)C::kRing * C::kSlotE + (size_t)C::kERing * NE * C::kEpiE) * sizeof(T) +
           8 * (2 * C::kRing + 2 * C::kERing);
}

struct MhdMaps {
    CUtensorMap tcbA[2], tcb3[2], tcbB[2];  // halo'd rows of each field: TJ+6, 3 or TJ+3 rows
    CUtensorMap tcbC[2];                    // each field's TJ tile rows alone (the queue-only planes)
    CUtensorMap lr[2];                      // k-halo boxes (4 x 8 x 3) of each field
    CUtensorMap e[3];                       // epilogue operands
};

template <typename T, int STAGE, int EPI_E>
__device__ __forceinline__ void mhd_epi_read(const T *se, int c, T &e0, T &e1, T &lo)
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
    }
}

template <typename T, int PHYS, int STAGE, bool STRETCH, class Args>
__global__ void __launch_bounds__(MhdCfg<T>::kThreads, 1)
    k_mhd_tma(Geo g, Coef<T> co, StageCoef<T> sc, const T *__restrict__ ia, const T *__restrict__ corr2, T dt,
              T visc, Args args, const __grid_constant__ MhdMaps maps, int ichunk, int *err)
{
    using C = MhdCfg<T>;
    constexpr int H = kH, TJ = C::TJ, kRing = C::kRing, kERing = C::kERing;
    constexpr int kTcbE = C::kTcbE, kLRE = C::kLRE, kFieldE = C::kFieldE, kSlotE = C::kSlotE, kEpiE = C::kEpiE;
    constexpr int NE = mhd_epi_fields<T, STAGE>();
    constexpr uint32_t kSlotBytes = kSlotE * sizeof(T), kRowBytes = kRowE * sizeof(T), kEpiBytes = kEpiE * sizeof(T);
    constexpr uint32_t kLRBoxBytes = 3 * kLRB * 4 * sizeof(T), kFieldBytes = kFieldE * sizeof(T);
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
    const int nout = ie - ib;

    if (ty == TJ && lane == 0) {
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
    if (ty == TJ) {
        if (lane != 0) return;
        const bool jlo = j0 < H, jhi = j0 + TJ + H > g.N1;
        const int kl = (k0 == 0 ? g.N2 : k0) - 4, kr = (k0 + kTK == g.N2) ? 0 : k0 + kTK;
        auto issue_s = [&](int n) -> bool {  // stencil load n: plane ib - H + n, both fields
            const int r = n % kRing;
            if (n >= kRing && !mbar_wait(empty(r), ((n / kRing) + 1) & 1, err)) return false;
            const uint32_t bar = full(r);
            const int plane = wrapi(ib - H + n, g.N0);
            if (n < H || n >= H + nout) {
                // a queue-only plane: the consumers read the tile rows' centre values alone
                mbar_expect_tx(bar, 2 * TJ * kRowBytes);
#pragma unroll
                for (int f = 0; f < 2; f++)
                    tma_load_4d(s0 + r * kSlotBytes + f * kFieldBytes + H * kRowBytes, &maps.tcbC[f], bar, k0, 0, j0,
                                plane);
                return true;
            }
            mbar_expect_tx(bar, kSlotBytes);
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const uint32_t dst = s0 + r * kSlotBytes + f * kFieldBytes;
                if (jlo) {
                    tma_load_4d(dst, &maps.tcb3[f], bar, k0, 0, g.N1 - H, plane);
                    tma_load_4d(dst + H * kRowBytes, &maps.tcbB[f], bar, k0, 0, 0, plane);
                } else if (jhi) {
                    tma_load_4d(dst, &maps.tcbB[f], bar, k0, 0, j0 - H, plane);
                    tma_load_4d(dst + (TJ + H) * kRowBytes, &maps.tcb3[f], bar, k0, 0, 0, plane);
                } else {
                    tma_load_4d(dst, &maps.tcbA[f], bar, k0, 0, j0 - H, plane);
                }
#pragma unroll
                for (int b = 0; b < TJ / kLRB; b++) {
                    tma_load_4d(dst + kTcbE * sizeof(T) + b * kLRBoxBytes, &maps.lr[f], bar, kl, j0 + b * kLRB, 0,
                                plane);
                    tma_load_4d(dst + (kTcbE + kLRE) * sizeof(T) + b * kLRBoxBytes, &maps.lr[f], bar, kr,
                                j0 + b * kLRB, 0, plane);
                }
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
    const T iak = ia[kw];
    const T c2k = STRETCH ? corr2[kw] : T(0);

    // slot offsets within a field: centre, and the k neighbour at s (inside the
    // row box or in the left/right halo boxes); component stride kTK in both
    const int cen = (H + ty) * kRowE + tx;
    const int lrrow = (ty / kLRB) * 3 * kLRB * 4 + (ty % kLRB) * 4;
    auto zoff = [&](int s) -> int {
        const int x = tx + s;
        return x < 0 ? kTcbE + lrrow + 4 + x : (x >= kTK ? kTcbE + kLRE + lrrow + (x - kTK) : cen + s);
    };
    // component c (0-2 the stage field, 3-5 the frozen one) within a slot
    auto fc = [](int c) -> int { return (c / 3) * kFieldE + (c % 3) * kTK; };

    T q[2 * H + 1][6];
    bool ok = true;
    for (int n = 0; n < 2 * H; n++) {  // queue: planes ib-3 .. ib+2
        ok = mbar_wait(full(n % kRing), (n / kRing) & 1, err);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        const T *sl = ring + (n % kRing) * kSlotE;
#pragma unroll
        for (int c = 0; c < 6; c++) q[n + 1][c] = sl[cen + fc(c)];
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
            for (int c = 0; c < 6; c++) q[s][c] = q[s + 1][c];
        {
            const T *sh = ring + (hd % kRing) * kSlotE;
#pragma unroll
            for (int c = 0; c < 6; c++) q[2 * H][c] = sh[cen + fc(c)];
            if (hd >= H + nout) release(empty(hd % kRing));
        }

        const int cur = p + H;
        const T *sl = ring + (cur % kRing) * kSlotE;
        auto vx = [&](int c, int s) -> T { return q[H + s][c]; };
        auto vy = [&](int c, int s) -> T { return sl[cen + s * kRowE + fc(c)]; };
        auto vz = [&](int c, int s) -> T { return sl[zoff(s) + fc(c)]; };
        const T y0[3] = {q[H][0], q[H][1], q[H][2]};
        const T x0[3] = {q[H][3], q[H][4], q[H][5]};
        T rhs[3];
        mhd_rhs<T, H, STRETCH, PHYS == PHYS_MHD_U>(vx, vy, vz, y0, x0, co, sc, iak, c2k, visc, rhs);
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
            for (int c = 0; c < 3; c++) mhd_epi_read<T, STAGE, kEpiE>(se, c, e0[c], e1[c], lo[c]);
            release(eempty(p % kERing));
        }
        const long long idx = (long long)(ib + p) * g.N12 + (long long)(j0 + ty) * g.N2 + kw;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long o = (long long)c * g.N3 + idx;
            if constexpr (sizeof(T) == 8)
                rk_store64<STAGE>(args, o, y0[c], e0[c], e1[c], dt * rhs[c]);
            else
                rk_store32<STAGE>(args, o, y0[c], e0[c], e1[c], lo[c], dt * rhs[c]);
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
    return fn(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
              const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// i-chunk: >= ~4 waves of the one resident block per SM
template <typename T> int mhd_ichunk(const Geo &g)
{
    const long long tiles = (long long)(g.N2 / kTK) * (g.N1 / MhdCfg<T>::TJ);
    int ch = g.N0;
    while (ch > 16 && tiles * ((g.N0 + ch - 1) / ch) < 148LL * 4) ch /= 2;
    return ch;
}

template <typename T, int PHYS, int STAGE, bool STRETCH, class Args>
cudaError_t launch_mhd(const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc, const Args &a,
                       const T *Y, const T *X, const T *const *ef, int *err, cudaStream_t st)
{
    constexpr int NE = mhd_epi_fields<T, STAGE>();
    using Cf = MhdCfg<T>;
    MhdMaps maps;
    memset(&maps, 0, sizeof maps);
    const T *fld[2] = {Y, X};
    bool ok = true;
    for (int f = 0; f < 2; f++)
        ok = ok && encode(&maps.tcbA[f], fld[f], g, Cf::TJ + 2 * kH) && encode(&maps.tcb3[f], fld[f], g, kH) &&
             encode(&maps.tcbB[f], fld[f], g, Cf::TJ + kH) && encode(&maps.tcbC[f], fld[f], g, Cf::TJ) &&
             encode(&maps.lr[f], fld[f], g, 0);
    for (int f = 0; f < NE; f++) ok = ok && encode(&maps.e[f], ef[f], g, Cf::TJ);
    if (!ok) return cudaErrorInvalidValue;
    constexpr size_t smem = mhd_smem_bytes<T, NE>();
    auto kern = k_mhd_tma<T, PHYS, STAGE, STRETCH, Args>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        attr = true;
    }
    const int ch = mhd_ichunk<T>(g);
    const dim3 grid(g.N2 / kTK, g.N1 / Cf::TJ, (g.N0 + ch - 1) / ch);
    kern<<<grid, dim3(kTK, Cf::TJ + 1), smem, st>>>(g, co, stage_coef(co, visc), ia, corr2, dt, visc, a, maps, ch, err);
    return cudaSuccess;
}

template <typename T, int PHYS, bool STRETCH, class Args>
cudaError_t launch_mhd_stage(int stage, const Geo &g, const Coef<T> &co, const T *ia, const T *corr2, T dt, T visc,
                             const Args &a, const T *X, const T *const *ef, int *err, cudaStream_t st)
{
    switch (stage) {
    case 0: return launch_mhd<T, PHYS, 0, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, X, ef, err, st);
    case 1: return launch_mhd<T, PHYS, 1, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, X, ef, err, st);
    case 2: return launch_mhd<T, PHYS, 2, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, X, ef, err, st);
    case 3: return launch_mhd<T, PHYS, 3, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, X, ef, err, st);
    default: return launch_mhd<T, PHYS, 4, STRETCH>(g, co, ia, corr2, dt, visc, a, a.Y, X, ef, err, st);
    }
}

template <typename T, class Args>
cudaError_t launch_mhd_any(int phys, int stage, bool stretch, const Geo &g, const Coef<T> &co, const T *ia,
                           const T *corr2, T dt, T visc, const Args &a, const T *X, const T *const *ef, int *err,
                           cudaStream_t st)
{
    if (phys == PHYS_MHD_U)
        return stretch ? launch_mhd_stage<T, PHYS_MHD_U, true>(stage, g, co, ia, corr2, dt, visc, a, X, ef, err, st)
                       : launch_mhd_stage<T, PHYS_MHD_U, false>(stage, g, co, ia, corr2, dt, visc, a, X, ef, err, st);
    return stretch ? launch_mhd_stage<T, PHYS_MHD_B, true>(stage, g, co, ia, corr2, dt, visc, a, X, ef, err, st)
                   : launch_mhd_stage<T, PHYS_MHD_B, false>(stage, g, co, ia, corr2, dt, visc, a, X, ef, err, st);
}

}  // namespace

bool mhd_tma_fits(const Geo &g, bool fp64)
{
    const int tj = fp64 ? MhdCfg<double>::TJ : MhdCfg<float>::TJ;
    return !g.wallY && g.N2 % kTK == 0 && g.N1 % tj == 0 && g.N1 >= 2 * tj;
}

cudaError_t launch_mhd_tma64(int phys, int stage, bool stretch, const Geo &g, const Coef<double> &co, const double *ia,
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
    return launch_mhd_any<double>(phys, stage, stretch, g, co, ia, corr2, dt, visc, a, a.X, ef, err, st);
}

cudaError_t launch_mhd_tma32(int phys, int stage, bool stretch, const Geo &g, const Coef<float> &co, const float *ia,
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
    return launch_mhd_any<float>(phys, stage, stretch, g, co, ia, corr2, dt, visc, a, a.X, ef, err, st);
}

}  // namespace nova
