// The row march of the 2D strip kernels, shared by the plain step (strip2d, one
// strip x chunk per block) and the batched step (batch2d, many strips x chunks of many
// instances per persistent block).
//
// One block of kStripNT lanes covers kStripNT consecutive columns starting at `jbase`
// (kStripW interior columns plus a halo column each side) and marches over rows
// i0-1 .. i1+1. Each row of each array arrives in shared memory by one TMA tile load
// into a kStages-deep ring of mbarrier-tracked stages; `ld` counts the loads this
// block has issued so far, so consecutive marches of one block reuse the ring without
// re-initialising the barriers. Every updated interior cell is handed to `sink`.
#pragma once

#include "hydro_rt.cuh"

namespace hydro {

constexpr int kStripNT = 128;
constexpr int kStripW = kStripNT - 2; // interior columns per strip
constexpr int kStages = 4;

__device__ __forceinline__ int wrap_row(int n, int nb_x) { return n == 0 ? nb_x : (n == nb_x + 1 ? 1 : n); }

template <class T> __device__ __forceinline__ typename Vec2<T>::type mk2(T a, T b)
{
    typename Vec2<T>::type v;
    v.x = a;
    v.y = b;
    return v;
}

template <class T> struct Smem2 {
    using V2 = typename Vec2<T>::type;
    __align__(128) V2 sr[kStages][kStripNT]; // (rho, E) rows
    __align__(128) V2 su[kStages][kStripNT]; // (rho u, rho v) rows
    // y-face inputs of every lane's cell (lane t at [t]) and every lane's right face flux
    // (lane t at [t+1]), as pairs so that each lane moves them with 128-bit (FP64) or 64-bit
    // (FP32) shared-memory accesses. Both are double-buffered by row parity, which leaves one
    // barrier per row: a lane may publish row n's inputs while its neighbour still reads row
    // n-1's, and the fluxes of row n-1 are read after row n's barrier.
    __align__(16) V2 xP[2][4][kStripNT + 1];
    __align__(16) V2 xF[2][2][kStripNT + 1];
    __align__(8) uint64_t full[kStages];
    int abort;
};

// One-time set-up of the stage barriers (thread 0), followed by a block barrier.
template <class T> __device__ __forceinline__ void march2d_init(Smem2<T> &S)
{
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&S.full[s], 1);
        fence_mbar_init();
        S.abort = 0;
    }
    __syncthreads();
}

struct March2 {
    int jbase, i0, i1; // columns jbase .. jbase+kStripNT-1, interior rows i0 .. i1
    int nb_x, nb_y;
    long long ys;
    int xwrap; // X neighbours of rows 1 and NB_X by periodic wrap (1) or ghost rows (0)
    // the input arrays, read directly by the per-lane loads (rows whose pitch TMA rejects)
    const void *in_r = nullptr, *in_u = nullptr;
};

// kEdge = false: a strip whose every lane holds a real column (1 <= j <= NB_Y), so no
// unit-state substitution and no wall face that an interior lane uses; kEdge = true: any
// strip. Both forms return false when a bounded barrier wait gave up (the block then
// stops).
//
// Lanes whose column is a ghost (j = 0, j = NB_Y+1) or past the array hold zeros; their
// primitives are never used, so they convert a unit state instead (keeps the reciprocal /
// square root of every lane on its regular path). A warp whose first column is past the
// last ghost column (NB_Y+1) computes nothing that is used: no interior cell, and its lane
// 0's cell only enters the face (NB_Y+1 | NB_Y+2) of the warp before it. It takes part in
// the row barriers only.

// Tensor-map form: each row of each array arrives by one TMA tile load issued by thread 0
// (16-byte row pitch). Per row m, the y face (j | j+1) of row m-1 (its neighbour's inputs
// were published before the previous barrier), the conversion of row m and the x face
// (row m-1 | row m) form one straight-line block ahead of the row's barrier, which gives
// the scheduler three independent chains; after the barrier only the update of row m-1
// remains. (Converting first and evaluating the faces after the barrier measured 77.3
// against 80.9 GCell/s at 40000 x 20000 FP64.)
template <bool kEdge, bool kF, class T, class Sink>
__device__ __forceinline__ bool march2d_tma(Smem2<T> &S, const CUtensorMap *tmr, const CUtensorMap *tmu,
                                            const March2 &g, T *rhoE_n, T *uv_n, const Phys<T> &ph, T DtDx, T DtDy,
                                            unsigned &ld, Sink &sink)
{
    using V2 = typename Vec2<T>::type;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr uint32_t kStageBytes = 2u * kStripNT * sizeof(V2);
    const int t = threadIdx.x;
    const int j = g.jbase + t;
    const int nrows = g.i1 - g.i0 + 3; // with one halo row above and below
    const bool interior = (t >= 1) && (t <= kStripW) && (!kEdge || j <= g.nb_y);
    const int xcoord = 2 * g.jbase;
    // the two wall faces live in at most two warps; the others skip the mirror selects
    const bool wall_warp = kEdge && __any_sync(FULL, j == 0 || j == g.nb_y);
    const bool real_col = (j >= 1) && (j <= g.nb_y);
    const bool dead_warp = kEdge && (g.jbase + (t & ~31) > g.nb_y + 1);
    const unsigned ld0 = ld;

    auto issue = [&](int m) {
        const unsigned q = ld0 + (unsigned)m;
        const int s = q % kStages;
        const int row = g.xwrap ? wrap_row(g.i0 - 1 + m, g.nb_x) : g.i0 - 1 + m;
        mbar_arrive_expect_tx(&S.full[s], kStageBytes);
        tma_load_2d(&S.sr[s][0], tmr, xcoord, row, &S.full[s]);
        tma_load_2d(&S.su[s][0], tmu, xcoord, row, &S.full[s]);
    };
    if (t == 0)
        for (int m = 0; m < kStages && m < nrows; ++m) issue(m);

    Cell2<T> Pm{};
    T Ur = 0, Uu = 0, Uv = 0, UE = 0;
    Flux2<T> fxlo{};
    int m = 0;
    bool aborted = false;
    // row mm's conserved values from its stage (every lane waits on the stage's barrier)
    auto load = [&](int mm, V2 &a, V2 &b) {
        const unsigned q = ld0 + (unsigned)mm;
        const int s = q % kStages;
        if (!mbar_wait_bounded(&S.full[s], (q / kStages) & 1)) S.abort = 1;
        a = S.sr[s][t];
        b = S.su[s][t];
        if (kEdge && !real_col) {
            a = mk2<T>(T(1), T(1));
            b = mk2<T>(T(0), T(0));
        }
    };
    // this lane's y-face inputs of row mm, for the previous lane's y face
    auto publish = [&](int mm, const Cell2<T> &P) {
        const FaceIn<T> me = face_y(P);
        S.xP[mm & 1][0][t] = mk2<T>(me.r, me.un);
        S.xP[mm & 1][1][t] = mk2<T>(me.p, me.Ka);
        S.xP[mm & 1][2][t] = mk2<T>(me.iKa, me.mn);
        S.xP[mm & 1][3][t] = mk2<T>(me.mt, me.eup);
    };
    // y face (j | j+1) of row mm-1, from this lane's cell of that row and the next lane's
    auto yface = [&](int mm) {
        const FaceIn<T> me = face_y(Pm);
        const V2 n0 = S.xP[(mm - 1) & 1][0][t + 1], n1 = S.xP[(mm - 1) & 1][1][t + 1],
                 n2 = S.xP[(mm - 1) & 1][2][t + 1], n3 = S.xP[(mm - 1) & 1][3][t + 1];
        FaceIn<T> L = me;
        FaceIn<T> R{n0.x, n0.y, n1.x, n1.y, n2.x, n2.y, n3.x, n3.y};
        if (wall_warp) {
            if (j == 0) L = mirror(R);       // wall at j = 1/2
            if (j == g.nb_y) R = mirror(me); // wall at j = NB_Y + 1/2
        }
        return face_flux<T, kF>(L, R, ph);
    };
    if (kEdge && dead_warp) {
        // (thread 0, which issues the row loads, is in warp 0: never dead)
        for (; m < nrows; ++m) {
            __syncthreads();
            if (S.abort) {
                aborted = true;
                break;
            }
        }
    } else {
        // row 0 (the halo row below) and row 1: conversion, row 1's y-face inputs and the
        // first x face
        for (; m < 2; ++m) {
            V2 a, b;
            load(m, a, b);
            const Cell2<T> P = make_cell2<T, kF>(a.x, b.x, b.y, a.y, ph);
            if (m == 1) {
                publish(m, P);
                fxlo = face_flux<T, kF>(face_x(Pm), face_x(P), ph);
            }
            __syncthreads(); // stage consumed by every lane; row 1's inputs published
            if (S.abort) {
                aborted = true;
                break;
            }
            if (t == 0 && m + kStages < nrows) issue(m + kStages);
            Pm = P;
            Ur = a.x; Uu = b.x; Uv = b.y; UE = a.y;
        }
        if (!aborted) {
#pragma unroll 2
            for (; m < nrows; ++m) {
                V2 a, b;
                load(m, a, b);
                const Flux2<T> fyr = yface(m);
                const Cell2<T> P = make_cell2<T, kF>(a.x, b.x, b.y, a.y, ph);
                const Flux2<T> fxhi = face_flux<T, kF>(face_x(Pm), face_x(P), ph);
                // row m-1's right face for the next lane (its left face), double-buffered
                // by row parity: the buffer of row m-3 was last read before the previous
                // barrier
                S.xF[(m - 1) & 1][0][t + 1] = mk2<T>(fyr.r, fyr.n);
                S.xF[(m - 1) & 1][1][t + 1] = mk2<T>(fyr.t, fyr.E);
                if (m <= nrows - 2) publish(m, P);
                __syncthreads(); // stage consumed; row m's inputs and row m-1's fluxes published
                if (S.abort) {
                    aborted = true;
                    break;
                }
                if (t == 0 && m + kStages < nrows) issue(m + kStages);
                if (interior) {
                    // row m-1's left face is lane t-1's right face of that row
                    const V2 f0 = S.xF[(m - 1) & 1][0][t], f1 = S.xF[(m - 1) & 1][1][t];
                    const Flux2<T> fyl{f0.x, f0.y, f1.x, f1.y};
                    const Upd2<T> o = update2<T, kF>(Ur, Uu, Uv, UE, fxlo, fxhi, fyl, fyr, DtDx, DtDy, ph);
                    const long long c = (long long)(g.i0 + m - 2) * g.ys + j;
                    reinterpret_cast<V2 *>(rhoE_n)[c] = mk2<T>(o.r, o.E);
                    reinterpret_cast<V2 *>(uv_n)[c] = mk2<T>(o.u, o.v);
                    sink(o);
                }
                fxlo = fxhi;
                Pm = P;
                Ur = a.x; Uu = b.x; Uv = b.y; UE = a.y;
            }
        }
    }
    ld = ld0 + (unsigned)nrows;
    if (aborted) {
        // gave up on a barrier: wait (bounded) for the loads still in flight before the
        // block's shared memory is released
        if (t == 0)
            for (int q = m; q < nrows && q < m + kStages; ++q)
                (void)mbar_wait_bounded(&S.full[(ld0 + q) % kStages], ((ld0 + q) / kStages) & 1);
        __syncthreads();
        return false;
    }
    return true;
}

// Per-lane form: each lane copies its own cell with cp.async (any pitch; 8-byte (FP32) or
// 16-byte (FP64) aligned arrays), so a lane reads only what it copied and the ring needs no
// barrier. Per row m: conversion of row m and publication of its y-face inputs, the
// barrier, then the x face (row m-1 | row m), the update of row m-1 and the y face of row m.
template <bool kEdge, bool kF, class T, class Sink>
__device__ __forceinline__ bool march2d_lane(Smem2<T> &S, const March2 &g, T *rhoE_n, T *uv_n, const Phys<T> &ph,
                                             T DtDx, T DtDy, unsigned &ld, Sink &sink)
{
    using V2 = typename Vec2<T>::type;
    constexpr unsigned FULL = 0xffffffffu;
    const int t = threadIdx.x;
    const int j = g.jbase + t;
    const int nrows = g.i1 - g.i0 + 3; // with one halo row above and below
    const bool interior = (t >= 1) && (t <= kStripW) && (!kEdge || j <= g.nb_y);
    const bool wall_warp = kEdge && __any_sync(FULL, j == 0 || j == g.nb_y);
    const bool real_col = (j >= 1) && (j <= g.nb_y);
    const bool dead_warp = kEdge && (g.jbase + (t & ~31) > g.nb_y + 1);
    const unsigned ld0 = ld;

    // this lane's cell of row m into its slot of stage (ld0 + m) % kStages
    const bool in_row = !kEdge || j <= g.nb_y + 1;
    auto issue_lane = [&](int m) {
        const int s = (ld0 + (unsigned)m) % kStages;
        if (m < nrows) {
            const int row = g.xwrap ? wrap_row(g.i0 - 1 + m, g.nb_x) : g.i0 - 1 + m;
            const long long c = in_row ? (long long)row * g.ys + j : 0;
            cp_async(&S.sr[s][t], static_cast<const V2 *>(g.in_r) + c, (int)sizeof(V2), in_row);
            cp_async(&S.su[s][t], static_cast<const V2 *>(g.in_u) + c, (int)sizeof(V2), in_row);
        }
        cp_async_commit();
    };
    for (int m = 0; m < kStages - 1; ++m) issue_lane(m);

    Cell2<T> Pm{};
    T Ur = 0, Uu = 0, Uv = 0, UE = 0;
    Flux2<T> fxlo{}, fyr{};
    int m = 0;
#pragma unroll 2
    for (; m < nrows; ++m) {
        const unsigned q = ld0 + (unsigned)m;
        const int s = q % kStages;
        if (kEdge && dead_warp) {
            __syncthreads();
            if (S.abort) break;
            continue;
        }
        issue_lane(m + kStages - 1); // into the slot this lane read for row m-1
        cp_async_wait<kStages - 1>(); // this lane's copy of row m landed
        V2 a = S.sr[s][t], b = S.su[s][t];
        if (kEdge && !real_col) {
            a = mk2<T>(T(1), T(1));
            b = mk2<T>(T(0), T(0));
        }
        const Cell2<T> P = make_cell2<T, kF>(a.x, b.x, b.y, a.y, ph);
        const bool yrow = (m >= 1) && (m <= nrows - 2);
        if (yrow) {
            const FaceIn<T> me = face_y(P);
            S.xP[m & 1][0][t] = mk2<T>(me.r, me.un);
            S.xP[m & 1][1][t] = mk2<T>(me.p, me.Ka);
            S.xP[m & 1][2][t] = mk2<T>(me.iKa, me.mn);
            S.xP[m & 1][3][t] = mk2<T>(me.mt, me.eup);
        }
        // this row's y-face inputs and the previous row's right-face fluxes published
        __syncthreads();
        if (S.abort) break;

        if (m >= 1) {
            // x face (row n-1 | row n) of this column; then the update of row n-1
            const Flux2<T> fxhi = face_flux<T, kF>(face_x(Pm), face_x(P), ph);
            if (m >= 2 && interior) {
                // row n-1's left face is lane t-1's right face of that row
                const V2 f0 = S.xF[(m - 1) & 1][0][t], f1 = S.xF[(m - 1) & 1][1][t];
                const Flux2<T> fyl{f0.x, f0.y, f1.x, f1.y};
                const Upd2<T> o = update2<T, kF>(Ur, Uu, Uv, UE, fxlo, fxhi, fyl, fyr, DtDx, DtDy, ph);
                const long long c = (long long)(g.i0 + m - 2) * g.ys + j;
                reinterpret_cast<V2 *>(rhoE_n)[c] = mk2<T>(o.r, o.E);
                reinterpret_cast<V2 *>(uv_n)[c] = mk2<T>(o.u, o.v);
                sink(o);
            }
            fxlo = fxhi;
        }
        if (yrow) {
            // y face (j | j+1) of row n, from this lane's cell and the next lane's
            const FaceIn<T> me = face_y(P);
            const V2 n0 = S.xP[m & 1][0][t + 1], n1 = S.xP[m & 1][1][t + 1], n2 = S.xP[m & 1][2][t + 1],
                     n3 = S.xP[m & 1][3][t + 1];
            FaceIn<T> L = me;
            FaceIn<T> R{n0.x, n0.y, n1.x, n1.y, n2.x, n2.y, n3.x, n3.y};
            if (wall_warp) {
                if (j == 0) L = mirror(R);       // wall at j = 1/2
                if (j == g.nb_y) R = mirror(me); // wall at j = NB_Y + 1/2
            }
            fyr = face_flux<T, kF>(L, R, ph);
            S.xF[m & 1][0][t + 1] = mk2<T>(fyr.r, fyr.n);
            S.xF[m & 1][1][t + 1] = mk2<T>(fyr.t, fyr.E);
        }
        Pm = P;
        Ur = a.x; Uu = b.x; Uv = b.y; UE = a.y;
    }
    ld = ld0 + (unsigned)nrows;
    cp_async_wait<0>();
    return m >= nrows;
}

// One strip march: the lean form away from the Y walls, the general one at them (the
// choice is uniform over the block). kTma: rows by tensor maps, else per-lane copies.
// kF: fused arithmetic (hydro_math.cuh).
template <class T, bool kTma = true, bool kF = false, class Sink>
__device__ __forceinline__ bool march2d(Smem2<T> &S, const CUtensorMap *tmr, const CUtensorMap *tmu, const March2 &g,
                                        T *rhoE_n, T *uv_n, const Phys<T> &ph, T DtDx, T DtDy, unsigned &ld,
                                        Sink &&sink)
{
    const bool lean = g.jbase >= 1 && g.jbase + kStripNT - 1 <= g.nb_y;
    if constexpr (kTma) {
        if (lean) return march2d_tma<false, kF>(S, tmr, tmu, g, rhoE_n, uv_n, ph, DtDx, DtDy, ld, sink);
        return march2d_tma<true, kF>(S, tmr, tmu, g, rhoE_n, uv_n, ph, DtDx, DtDy, ld, sink);
    } else {
        if (lean) return march2d_lane<false, kF>(S, g, rhoE_n, uv_n, ph, DtDx, DtDy, ld, sink);
        return march2d_lane<true, kF>(S, g, rhoE_n, uv_n, ph, DtDx, DtDy, ld, sink);
    }
}

} // namespace hydro
