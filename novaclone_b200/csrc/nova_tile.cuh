// 2.5-D tile march shared by the fused forward and adjoint stage kernels and
// the tiled projection kernels.
//
// A block of kTK x kTJ threads owns a kTK(k) x kTJ(j) column of the grid and
// walks it along i over [ib, ie).  Each thread keeps its column's 2H+1 planes
// of the NC input components in a register queue (the i-direction stencil);
// the current plane plus its j/k halo is staged in shared memory (the j- and
// k-direction stencils).  Every index is wrapped modulo the grid, which
// synthesises the periodic ghosts (src/BC/periodicBC.hxx:1-66) at load time;
// with walls in y the j halo is mirrored with the Neumann/Dirichlet ghost
// formulas instead (Walls<T>).
//
// Pipelining: the shared plane is double-buffered, so one barrier per plane
// suffices; the global loads of the next plane (queue head, halo and, through
// the `pre` hook, the caller's pointwise operands) are issued right after that
// barrier, before the current plane's arithmetic, so their latency overlaps
// the math.
#pragma once

#include "nova_internal.cuh"

// unroll factor of the plane loop (2H+1 would turn the queue rotation into
// register renaming, but the extra live ranges cost more than the moves)
#ifndef NOVA_MARCH_UNROLL
#define NOVA_MARCH_UNROLL 1
#endif
#define NOVA_PRAGMA(x) _Pragma(#x)
#define NOVA_UNROLL(n) NOVA_PRAGMA(unroll n)

namespace nova {

template <typename T, int H, int NC> struct TileSmem {
    T v[2][NC][kTJ + 2 * H][kTK + 2 * H];
};

template <typename T, int H, int NC> constexpr size_t tile_smem_bytes() { return sizeof(TileSmem<T, H, NC>); }

struct NoPre {
    __device__ void operator()(long long, bool) const {}
};

// ld(c, o) returns component c at linear node index o.
// pre(idx, load) runs for valid threads once before the loop with the first
// plane's node (load = true) and then once per plane before body, with the
// next plane's node and load = (a next plane exists): it lets the caller
// rotate its own prefetched pointwise operands and issue the next ones.
// body(idx, q, vx, vy, vz) runs for valid threads once per plane, with idx
// the thread's node, q the register queue and vx/vy/vz(c, s) the neighbour
// accessors along i, j, k.
template <typename T, int H, int NC, bool WALLS, class Ld, class Pre, class Body>
__device__ __forceinline__ void tile_march(const Geo &g, const Walls<T> &wl, TileSmem<T, H, NC> &sm, const Ld &ld,
                                           int ib, int ie, Pre &&pre, Body &&body)
{
    constexpr int NJH = 2 * H * kTK;
    constexpr int NKH = 2 * H * kTJ;
    constexpr int NH = NJH + NKH;
    constexpr int HS = (NH + kThreads - 1) / kThreads;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTK + tx;
    const int k0 = blockIdx.x * kTK, j0 = blockIdx.y * kTJ;
    const int k = k0 + tx, j = j0 + ty;
    const bool valid = (k < g.N2) && (j < g.N1);
    const int kw = wrapi(k, g.N2);
    // rows past the north wall hold mirrored ghosts (read as neighbours only)
    int jw, tside = -1, tl = 0;
    if (WALLS && j >= g.N1) {
        tl = min(j - (g.N1 - 1), g.N1 - 1);
        tside = 1;
        jw = (g.N1 - 1) - tl;
    } else {
        jw = wrapi(j, g.N1);
    }

    int hrow[HS], hcol[HS], hside[HS], hl[HS];
    long long hoff[HS];
    bool hon[HS];
#pragma unroll
    for (int s = 0; s < HS; s++) {
        const int t = tid + s * kThreads;
        hon[s] = t < NH;
        int row, col;
        if (t < NJH) {
            const int r = t / kTK;
            row = r < H ? r : kTJ + r;
            col = H + t % kTK;
        } else {
            const int u = t - NJH;
            row = H + u / (2 * H);
            const int cc = u % (2 * H);
            col = cc < H ? cc : kTK + cc;
        }
        if (!hon[s]) { row = 0; col = 0; }
        hrow[s] = row;
        hcol[s] = col;
        int jg = j0 + row - H;
        hside[s] = -1;
        hl[s] = 0;
        if constexpr (WALLS) {  // mirror across the y walls
            if (jg < 0) {
                hside[s] = 0;
                hl[s] = min(-jg, g.N1 - 1);
                jg = hl[s];
            } else if (jg >= g.N1) {
                hside[s] = 1;
                hl[s] = min(jg - (g.N1 - 1), g.N1 - 1);
                jg = (g.N1 - 1) - hl[s];
            }
        } else {
            jg = wrapi(jg, g.N1);
        }
        hoff[s] = (long long)jg * g.N2 + wrapi(k0 + col - H, g.N2);
    }
    auto hload = [&](int s, int c, long long plane) -> T {
        const T v = ld(c, plane + hoff[s]);
        if constexpr (!WALLS) {
            return v;
        } else {
            return hside[s] < 0 ? v : wall_ghost(wl, hside[s], c, hl[s], v);
        }
    };

    const long long colOff = (long long)jw * g.N2 + kw;
    T q[2 * H + 1][NC];
#pragma unroll
    for (int s = 0; s < 2 * H; s++) {
        const long long p = (long long)wrapi(ib - H + s, g.N0) * g.N12 + colOff;
#pragma unroll
        for (int c = 0; c < NC; c++) q[s + 1][c] = ld(c, p);
    }
    // plane index of the queue head, kept wrapped incrementally
    int lead = wrapi(ib + H, g.N0);
    T qn[NC], hn[HS][NC];
    {
        const long long p = (long long)lead * g.N12 + colOff;
        const long long plane = (long long)ib * g.N12;
#pragma unroll
        for (int c = 0; c < NC; c++) qn[c] = ld(c, p);
#pragma unroll
        for (int s = 0; s < HS; s++)
#pragma unroll
            for (int c = 0; c < NC; c++) hn[s][c] = hon[s] ? hload(s, c, plane) : T(0);
        if (valid) pre(plane + colOff, true);
    }

    NOVA_UNROLL(NOVA_MARCH_UNROLL)
    for (int i = ib; i < ie; i++) {
        const int b = (i - ib) & 1;
#pragma unroll
        for (int s = 0; s < 2 * H; s++)
#pragma unroll
            for (int c = 0; c < NC; c++) q[s][c] = q[s + 1][c];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            q[2 * H][c] = qn[c];
            if constexpr (WALLS)
                sm.v[b][c][ty + H][tx + H] = (tside < 0) ? q[H][c] : wall_ghost(wl, 1, c, tl, q[H][c]);
            else
                sm.v[b][c][ty + H][tx + H] = q[H][c];
        }
#pragma unroll
        for (int s = 0; s < HS; s++)
            if (hon[s])
#pragma unroll
                for (int c = 0; c < NC; c++) sm.v[b][c][hrow[s]][hcol[s]] = hn[s][c];
        __syncthreads();
        const bool more = i + 1 < ie;
        const long long nplane = (long long)(i + 1) * g.N12;
        if (more) {  // next plane's loads fly during this plane's arithmetic
            lead = (lead + 1 == g.N0) ? 0 : lead + 1;
            const long long p = (long long)lead * g.N12 + colOff;
#pragma unroll
            for (int c = 0; c < NC; c++) qn[c] = ld(c, p);
#pragma unroll
            for (int s = 0; s < HS; s++)
                if (hon[s])
#pragma unroll
                    for (int c = 0; c < NC; c++) hn[s][c] = hload(s, c, nplane);
        }
        if (!valid) continue;
        pre(nplane + colOff, more);
        auto vx = [&](int c, int s) -> T { return q[H + s][c]; };
        auto vy = [&](int c, int s) -> T { return sm.v[b][c][ty + H + s][tx + H]; };
        auto vz = [&](int c, int s) -> T { return sm.v[b][c][ty + H][tx + H + s]; };
        body((long long)i * g.N12 + colOff, q, vx, vy, vz);
    }
}

template <typename T, int H, int NC, bool WALLS, class Ld, class Body>
__device__ __forceinline__ void tile_march(const Geo &g, const Walls<T> &wl, TileSmem<T, H, NC> &sm, const Ld &ld,
                                           int ib, int ie, Body &&body)
{
    tile_march<T, H, NC, WALLS>(g, wl, sm, ld, ib, ie, NoPre{}, body);
}

// grid shape of a tile march: k tiles x j tiles x i chunks
inline int pick_ichunk(const Geo &g, int blocks_per_sm)
{
    // >= ~4 waves of resident blocks on 148 SMs, with the 2H-plane warm-up
    // kept small against the chunk length
    const long long tiles = (long long)((g.N2 + kTK - 1) / kTK) * ((g.N1 + kTJ - 1) / kTJ);
    int ch = g.N0;
    while (ch > 16 && tiles * ((g.N0 + ch - 1) / ch) < 148LL * blocks_per_sm * 4) ch /= 2;
    return ch;
}

inline dim3 tile_grid(const Geo &g, int ch)
{
    return dim3((g.N2 + kTK - 1) / kTK, (g.N1 + kTJ - 1) / kTJ, (g.N0 + ch - 1) / ch);
}

}  // namespace nova
