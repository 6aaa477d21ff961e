// The X-march of the 3D strip kernels, shared by the plain step (strip3d, one tile x
// chunk per block) and the batched step (batch3d, tiles of many instances per persistent
// block).
//
// One block of W warps (8 by default) covers a tile of y rows x 32 z columns starting at
// (jbase, kbase): the interior columns plus a one-cell halo ring. Each X plane of the tile
// arrives in a shared-memory ring, in one of two forms:
//  - tensor maps (march3d_tma): one thread issues two 3D TMA tile loads per plane (the
//    (rho, E) pairs and the momentum triples of the tile's rows, x = the interleaved
//    components of 32 cells, y = the tile's rows, z = the plane) completing on the stage's
//    mbarrier; needs a row pitch of a multiple of 16 bytes (FP64 with even NB_Z) and even
//    kbase. Two tile layouts: W rows on W warps (warps 0 and W-1 hold the halo rows), or
//    W+1 rows on W warps (warp 0 holds both halo rows, all other warps interior rows);
//  - per-lane copies (march3d_lane): cp.async of any alignment of the interleaved
//    pairs/triples, in FP64 by every lane for its own cell, in FP32 by the two halo-row
//    warps for the whole tile; W rows on W warps.
// Each lane converts its cell to primitives once and publishes them as 16-byte pairs
// (double-buffered by plane parity; one barrier per plane). Per plane a lane computes one x
// face (registers), one z face (the next lane's cell from shared memory, the flux back by
// shuffles) and one y face (the row above's cell, the flux back through shared memory),
// then updates the plane behind it. Every updated interior cell is handed to `sink`.
#pragma once

#include "hydro_rt.cuh"

namespace hydro {

// Warps per block: 8 by default in both precisions (6 interior rows, or 7 in the 9-row
// tile that the FP64 tensor-map form uses by default). Resident blocks per SM of an 8-warp
// tile: FP64 two (the 128-register budget; with 16 warps it spills and keeps one block,
// 31.5 -> 28.4 GCell/s at 512^3 in an earlier form), FP32 three (80 registers without
// spills; 54.1 -> 56.2 GCell/s at 512^3 against two, and 16-warp tiles with one block give
// 53.7). The plain step also takes other tile heights, chosen at run time
// (hydro_set_launch_shape); the batched engine runs k3Warps-row tiles.
template <class T> constexpr int min_blocks3(int W) { return W <= 8 ? (sizeof(T) == 4 ? 3 : 2) : 1; }
template <class T> constexpr int k3Warps = 8;                        // y extent of the tile (with halo)
template <class T> constexpr int k3NT = 32 * k3Warps<T>;             // threads
template <class T> constexpr int k3TY = k3Warps<T> - 2;              // interior rows per tile
template <class T> constexpr int k3MinBlocks = min_blocks3<T>(k3Warps<T>); // resident blocks per SM
constexpr int k3TZ = 30;           // interior columns per tile
constexpr int k3Stages = 4;

__device__ __forceinline__ int wrap_plane(int n, int nb_x) { return n == 0 ? nb_x : (n == nb_x + 1 ? 1 : n); }

template <class T> __device__ __forceinline__ typename Vec2<T>::type pair3(T a, T b)
{
    typename Vec2<T>::type v;
    v.x = a;
    v.y = b;
    return v;
}

template <class T, int W_ = k3Warps<T>> struct Smem3 {
    using V2 = typename Vec2<T>::type;
    static constexpr int W = W_;
    static constexpr int NT = 32 * W;
    // tensor-map form: W rows on W warps, k3Stages stages
    static constexpr int NR = NT, NS = k3Stages;
    static constexpr bool kPair = false;
    union {
        T st[k3Stages][5][NT]; // per-lane copies, per plane: rho, E, rho_u, rho_v, rho_w
        struct {               // tensor-map boxes in tile order (lane t = 32 row + column)
            T r[k3Stages][NT][2]; // (rho, E)
            T u[k3Stages][NT][3]; // (rho u, rho v, rho w)
        } tm;
    };
    uint64_t full[k3Stages]; // tensor-map form: stage s holds its plane
    int abort;
    // each lane's cell by plane parity, as pairs (r,p) (Ka,iKa) (v,w) (mu,mv) (mw,eup_xy)
    // (eup_z,-): the warp below reads its y-face inputs, the previous lane its z-face inputs
    V2 xP[2][6][NT];
    V2 xF[2][2][NT]; // each lane's +y face flux by plane parity: (r,n) (t1,t2) ...
    T xFE[2][NT];    // ... and E
};

// a neighbour's face inputs from the exchange buffer (layout of Smem3::xP, NT lanes)
template <class T, int NT> __device__ __forceinline__ FaceIn3<T> xp_face_y(const typename Vec2<T>::type *x)
{
    const auto q0 = x[0 * NT], q1 = x[1 * NT], q2 = x[2 * NT], q3 = x[3 * NT], q4 = x[4 * NT];
    return FaceIn3<T>{q0.x, q2.x, q0.y, q1.x, q1.y, q3.y, q3.x, q4.x, q4.y}; // normal v: (v, u, w)
}
// (in fused arithmetic the z faces take the same upwinded energy as x and y faces, so
// the sixth pair is neither published nor read)
template <class T, int NT, bool kF = false>
__device__ __forceinline__ FaceIn3<T> xp_face_z(const typename Vec2<T>::type *x)
{
    const auto q0 = x[0 * NT], q1 = x[1 * NT], q2 = x[2 * NT], q3 = x[3 * NT], q4 = x[4 * NT];
    if constexpr (kF) return FaceIn3<T>{q0.x, q2.y, q0.y, q1.x, q1.y, q4.x, q3.y, q3.x, q4.y};
    const auto q5 = x[5 * NT];
    return FaceIn3<T>{q0.x, q2.y, q0.y, q1.x, q1.y, q4.x, q3.y, q3.x, q5.x}; // normal w: (w, v, u)
}

struct March3 {
    int kbase, jbase, i0, i1; // tile corner (halo included) and interior X planes
    int nb_x, nb_y, nb_z;
    long long zs, zy; // strides in cells of a Y row and of an X plane
    int xwrap;        // X neighbours of planes 1 and NB_X by periodic wrap (1) or ghost planes (0)
};

// kEdge = false: a tile whose every lane holds a real cell (1 <= j <= NB_Y,
// 1 <= k <= NB_Z) and whose faces used by interior lanes touch no wall; it needs neither
// the unit-state substitution nor the wall mirrors. kEdge = true: any tile.
// Tensor maps of the two input arrays for the kTma form (null otherwise).
struct Tmaps3 {
    const CUtensorMap *r = nullptr, *u = nullptr;
};

// Tile of W+1 rows on W = 8 warps for the tensor-map form (FP64): warp 0 holds both halo
// rows (0 and 8) and warps 1..7 the seven interior rows, so no warp idles on a halo row
// alone. Three stages in the ring (the shared memory of two blocks per SM). Slot of row r,
// column l: 32 r + l.
template <class T> struct Smem3P {
    using V2 = typename Vec2<T>::type;
    static constexpr int W = 8;
    static constexpr int NR = 32 * (W + 1), NS = 3;
    static constexpr bool kPair = true;
    struct {
        T r[NS][NR][2]; // (rho, E)
        T u[NS][NR][3]; // (rho u, rho v, rho w)
    } tm;
    uint64_t full[NS];
    int abort;
    V2 xP[2][6][NR];        // each cell's face inputs by plane parity (layout of Smem3::xP)
    V2 xF[2][2][32 * (W - 1)]; // +y face fluxes of rows 0 .. W-2 (the row above reads them)
    T xFE[2][32 * (W - 1)];
};

// One-time set-up of the stage barriers of the tensor-map form (thread 0), then a block
// barrier.
template <class SM> __device__ __forceinline__ void march3d_init(SM &S)
{
    if (threadIdx.x == 0) {
        for (int s = 0; s < SM::NS; ++s) mbar_init(&S.full[s], 1);
        fence_mbar_init();
        S.abort = 0;
    }
    __syncthreads();
}

// kEdge = false: a tile whose every lane holds a real cell (1 <= j <= NB_Y,
// 1 <= k <= NB_Z) and whose faces used by interior lanes touch no wall; it needs neither
// the unit-state substitution nor the wall mirrors. kEdge = true: any tile. Ghost cells
// (j or k = 0 or NB+1) and cells past the array are never used: they convert a unit state
// so every lane's reciprocal / square root stays regular.

// Tensor-map form. The plane loop is written once per warp role (interior rows, the
// bottom halo row, the top halo row), so no role test sits inside it. In the interior
// rows' loop the +y and +z faces of plane m-1 (their neighbours' inputs were published
// before the previous barrier), the conversion of plane m and the x face (m-1 | m) form one
// straight-line block ahead of the plane's barrier: independent chains the scheduler
// interleaves; after the barrier only the update of plane m-1 remains. (Converting first
// and evaluating the faces after the stage wait of the next plane measured 33.3 against
// 35.3 GCell/s strict at 512^3 with 8-row tiles; the 9-row tile 37.2.) Returns false when a
// bounded barrier wait gave up.
template <bool kEdge, bool kF, class SM, class T, class Sink>
__device__ __forceinline__ bool march3d_tma(SM &S, T *rhoE_n, T *uvw_n, const March3 &g, const Phys<T> &ph, T DtDx,
                                            T DtDy, T DtDz, const Tmaps3 &tm, Sink &sink)
{
    using V2 = typename Vec2<T>::type;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int W = SM::W, NR = SM::NR, NS = SM::NS;
    constexpr bool kPair = SM::kPair;
    constexpr int R = kPair ? W + 1 : W; // tile rows with halo
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int k = g.kbase + lane, j = g.jbase + w;
    const int nplanes = g.i1 - g.i0 + 3;
    const bool kreal = !kEdge || ((k >= 1) && (k <= g.nb_z));
    auto row_real = [&](int jj) { return !kEdge || ((jj >= 1) && (jj <= g.nb_y) && kreal); };

    __syncthreads(); // the previous march of this block is done with the stages and exchange buffers
    constexpr uint32_t kPlaneBytes = (uint32_t)(5 * NR * sizeof(T));
    // thread 0 loads plane m into stage m % NS (a single march per block: stage s
    // completes its phase (m / NS) & 1)
    auto issue_tma = [&](int m) {
        const int s = m % NS;
        const int plane = g.xwrap ? wrap_plane(g.i0 - 1 + m, g.nb_x) : g.i0 - 1 + m;
        mbar_arrive_expect_tx(&S.full[s], kPlaneBytes);
        tma_load_3d(&S.tm.r[s][0][0], tm.r, 2 * g.kbase, g.jbase, plane, &S.full[s]);
        tma_load_3d(&S.tm.u[s][0][0], tm.u, 3 * g.kbase, g.jbase, plane, &S.full[s]);
    };
    if (t == 0)
        for (int m = 0; m < NS - 1 && m < nplanes; ++m) issue_tma(m);

    // every lane waits for the stage's barrier; a time-out sets the block's abort flag,
    // which every warp reads after the plane's block barrier
    auto wait = [&](int mm) {
        if (!mbar_wait_bounded(&S.full[mm % NS], (uint32_t)(mm / NS) & 1u)) S.abort = 1;
    };
    auto load = [&](int mm, int slot, bool real, T &ur, T &uE, T &uu, T &uv, T &uw) {
        const int s = mm % NS;
        const V2 a = *reinterpret_cast<const V2 *>(&S.tm.r[s][slot][0]);
        ur = a.x;
        uE = a.y;
        uu = S.tm.u[s][slot][0];
        uv = S.tm.u[s][slot][1];
        uw = S.tm.u[s][slot][2];
        if (kEdge && !real) {
            ur = T(1);
            uE = T(1);
            uu = uv = uw = T(0);
        }
    };
    auto publish = [&](int mm, int slot, const Cell3<T> &P) {
        V2 *x = &S.xP[mm & 1][0][slot];
        x[0 * NR] = pair3<T>(P.r, P.p);
        x[1 * NR] = pair3<T>(P.Ka, P.iKa);
        x[2 * NR] = pair3<T>(P.v, P.w);
        x[3 * NR] = pair3<T>(P.mu, P.mv);
        x[4 * NR] = pair3<T>(P.mw, P.eup_xy);
        if constexpr (!kF) x[5 * NR] = pair3<T>(P.eup_z, T(0));
    };
    // +y face of (jj | jj+1) of plane mm-1, from the cell Pme and the row above's
    auto yface = [&](int mm, const Cell3<T> &Pme, int slot, int jj) {
        const FaceIn3<T> me = face3_y(Pme);
        const FaceIn3<T> nb = xp_face_y<T, NR>(&S.xP[(mm - 1) & 1][0][slot + 32]);
        FaceIn3<T> L = me, Rt = nb;
        if (kEdge) {
            if (jj == 0) L = mirror3(nb);
            if (jj == g.nb_y) Rt = mirror3(me);
        }
        return face_flux3<T, kF>(L, Rt, ph);
    };
    auto publish_y = [&](int mm, int slot, const Flux3<T> &fy) {
        S.xF[mm & 1][0][slot] = pair3<T>(fy.r, fy.n);
        S.xF[mm & 1][1][slot] = pair3<T>(fy.t1, fy.t2);
        S.xFE[mm & 1][slot] = fy.E;
    };

    int m = 0;
    bool aborted = false;
    // interior rows: 1 .. R-2 (warps past the grid's last row in an edge tile hold none)
    const bool iwarp = (w >= 1) && (w <= R - 2) && (!kEdge || (g.jbase + 1 <= g.nb_y));
    if (iwarp) {
        const bool real = row_real(j);
        const bool interior = (lane >= 1) && (lane <= k3TZ) && (!kEdge || ((j <= g.nb_y) && (k <= g.nb_z)));
        const bool pub = w <= R - 3; // the row above is interior and reads this +y flux
        const long long colofs = (long long)j * g.zs + k;
        Cell3<T> Pm{};
        T Ur = 0, Uu = 0, Uv = 0, Uw = 0, UE = 0;
        Flux3<T> fxlo{};
        // +z face of (k | k+1) of plane mm-1: the next lane's cell from the exchange buffer
        // (lane 31 reads the next row's lane 0, a face no interior lane uses)
        auto zface = [&](int mm) {
            const FaceIn3<T> mz = face3_z(Pm);
            const FaceIn3<T> nz = xp_face_z<T, NR, kF>(&S.xP[(mm - 1) & 1][0][t + 1]);
            FaceIn3<T> L = mz, Rt = nz;
            if (kEdge) {
                if (k == 0) L = mirror3(nz);
                if (k == g.nb_z) Rt = mirror3(mz);
            }
            return face_flux3<T, kF>(L, Rt, ph);
        };
        // planes 0 and 1: conversion, and plane 1's x face
        for (; m < 2; ++m) {
            T ur, uE, uu, uv, uw;
            wait(m);
            load(m, t, real, ur, uE, uu, uv, uw);
            const Cell3<T> P = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
            publish(m, t, P);
            if (m == 1) fxlo = face_flux3<T, kF>(face3_x(Pm), face3_x(P), ph);
            __syncthreads();
            if (S.abort) {
                aborted = true;
                break;
            }
            Pm = P;
            Ur = ur; Uu = uu; Uv = uv; Uw = uw; UE = uE;
        }
        if (!aborted) {
#pragma unroll 2
            for (; m < nplanes; ++m) {
                T ur, uE, uu, uv, uw;
                wait(m);
                load(m, t, real, ur, uE, uu, uv, uw);
                const Flux3<T> fy = yface(m, Pm, t, j);
                const Flux3<T> fz = zface(m);
                const Cell3<T> P = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
                const Flux3<T> fxhi = face_flux3<T, kF>(face3_x(Pm), face3_x(P), ph);
                if (pub) publish_y(m, t, fy);
                publish(m, t, P);
                __syncthreads(); // plane m's cells and plane m-1's +y faces published
                if (S.abort) {
                    aborted = true;
                    break;
                }
                Flux3<T> fzl;
                fzl.r = __shfl_up_sync(FULL, fz.r, 1);
                fzl.n = __shfl_up_sync(FULL, fz.n, 1);
                fzl.t1 = __shfl_up_sync(FULL, fz.t1, 1);
                fzl.t2 = __shfl_up_sync(FULL, fz.t2, 1);
                fzl.E = __shfl_up_sync(FULL, fz.E, 1);
                if (interior) {
                    const auto a0 = S.xF[m & 1][0][t - 32], a1 = S.xF[m & 1][1][t - 32];
                    const Flux3<T> fyl{a0.x, a0.y, a1.x, a1.y, S.xFE[m & 1][t - 32]};
                    const Upd3<T> o =
                        update3<T, kF>(Ur, Uu, Uv, Uw, UE, fxlo, fxhi, fyl, fy, fzl, fz, DtDx, DtDy, DtDz, ph);
                    const long long c = (long long)(g.i0 + m - 2) * g.zy + colofs;
                    rhoE_n[2 * c] = o.r;
                    rhoE_n[2 * c + 1] = o.E;
                    uvw_n[3 * c] = o.u;
                    uvw_n[3 * c + 1] = o.v;
                    uvw_n[3 * c + 2] = o.w;
                    sink(o);
                }
                fxlo = fxhi;
                Pm = P;
                Ur = ur; Uu = uu; Uv = uv; Uw = uw; UE = uE;
            }
        }
    } else if (w == 0) {
        // the bottom halo row: conversion, and from plane 2 on its +y face (the first
        // interior row's -y face); with kPair also the top halo row. Thread 0 refills the
        // stage of plane m-1 (every lane read it before the previous barrier).
        const int jt = g.jbase + R - 1, st = 32 * (R - 1) + lane;
        const bool real0 = row_real(j), realt = row_real(jt);
        Cell3<T> Pm0{};
        for (; m < nplanes; ++m) {
            if (t == 0 && m + NS - 1 < nplanes) issue_tma(m + NS - 1);
            T ur, uE, uu, uv, uw;
            wait(m);
            load(m, lane, real0, ur, uE, uu, uv, uw);
            if (m >= 2) publish_y(m, lane, yface(m, Pm0, lane, j));
            const Cell3<T> P0 = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
            publish(m, lane, P0);
            if constexpr (kPair) {
                T vr, vE, vu, vv, vw;
                load(m, st, realt, vr, vE, vu, vv, vw);
                publish(m, st, make_cell3<T, kF>(vr, vu, vv, vw, vE, ph));
            }
            __syncthreads();
            if (S.abort) {
                aborted = true;
                break;
            }
            Pm0 = P0;
        }
    } else {
        // the top halo row (8-row layout), or rows past the grid in an edge tile:
        // conversion only
        const bool real = row_real(j);
        for (; m < nplanes; ++m) {
            T ur, uE, uu, uv, uw;
            wait(m);
            load(m, t, real, ur, uE, uu, uv, uw);
            publish(m, t, make_cell3<T, kF>(ur, uu, uv, uw, uE, ph));
            __syncthreads();
            if (S.abort) {
                aborted = true;
                break;
            }
        }
    }
    if (aborted) {
        // gave up on a barrier: wait (bounded) for the loads still in flight before the
        // block's shared memory is released
        if (t == 0)
            for (int q = m; q < nplanes && q < m + NS; ++q)
                (void)mbar_wait_bounded(&S.full[q % NS], (uint32_t)(q / NS) & 1u);
        __syncthreads();
        return false;
    }
    return true;
}

// Per-lane copies (any alignment): cp.async of the interleaved pairs/triples into a
// k3Stages-deep ring. FP32 tiles: the two halo-row warps, which have the least work per
// plane, stage the whole tile (warp 0 copies tile rows 0 .. W/2-1 and warp W-1 rows
// W/2 .. W-1, each lane its column k). FP64 tiles: every lane copies its own cell. Measured
// at 512^3: FP32 49.8 -> 50.7-52.3 GCell/s with the halo warps loading, FP64 31.6 -> 30.9,
// so each precision keeps the faster form. Cells past the array load as zeros.
template <bool kEdge, bool kF, class T, int W, class Sink>
__device__ __forceinline__ bool march3d_lane(Smem3<T, W> &S, const T *rhoE, const T *uvw, T *rhoE_n, T *uvw_n,
                                             const March3 &g, const Phys<T> &ph, T DtDx, T DtDy, T DtDz, Sink &sink)
{
    constexpr unsigned FULL = 0xffffffffu;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int k = g.kbase + lane, j = g.jbase + w;
    const int nplanes = g.i1 - g.i0 + 3;
    const bool interior =
        (w >= 1) && (w <= (W - 2)) && (lane >= 1) && (lane <= k3TZ) && (!kEdge || ((j <= g.nb_y) && (k <= g.nb_z)));
    const bool iwarp = (w >= 1) && (w <= (W - 2)) && (!kEdge || (g.jbase + 1 <= g.nb_y)); // warp holds interior rows
    const long long colofs = (long long)j * g.zs + k;
    const bool real = !kEdge || ((j >= 1) && (j <= g.nb_y) && (k >= 1) && (k <= g.nb_z));
    constexpr bool kHaloLoads = sizeof(T) == 4;
    const bool loader = kHaloLoads ? ((w == 0) || (w == W - 1)) : true;
    const int rbase = kHaloLoads ? ((w == 0) ? 0 : W / 2) : w;
    constexpr int kRows = kHaloLoads ? W / 2 : 1; // tile rows each loading lane copies
    const bool kin = !kEdge || (k <= g.nb_z + 1);

    __syncthreads(); // the previous march of this block is done with the stages and exchange buffers
    auto issue = [&](int m) { // loading lanes only
        const int s = m % k3Stages;
        if (m < nplanes) {
            const long long pl =
                (long long)(g.xwrap ? wrap_plane(g.i0 - 1 + m, g.nb_x) : g.i0 - 1 + m) * g.zy + (long long)g.jbase * g.zs + k;
#pragma unroll
            for (int rr = 0; rr < kRows; ++rr) {
                const int r = rbase + rr;
                const bool ok = kin && (!kEdge || g.jbase + r <= g.nb_y + 1);
                const long long c = pl + (long long)r * g.zs;
                const T *pr = ok ? rhoE + 2 * c : rhoE;
                const T *pu = ok ? uvw + 3 * c : uvw;
                const int tt = 32 * r + lane;
                cp_async(&S.st[s][0][tt], pr, sizeof(T), ok);
                cp_async(&S.st[s][1][tt], pr + 1, sizeof(T), ok);
                cp_async(&S.st[s][2][tt], pu, sizeof(T), ok);
                cp_async(&S.st[s][3][tt], pu + 1, sizeof(T), ok);
                cp_async(&S.st[s][4][tt], pu + 2, sizeof(T), ok);
            }
        }
        cp_async_commit();
    };
    if (loader) {
#pragma unroll
        for (int m = 0; m < k3Stages - 1; ++m) issue(m);
    }
    if (kHaloLoads) {
        if (loader) cp_async_wait<k3Stages - 2>(); // plane 0 landed
        __syncthreads();                          // plane 0 visible to every lane
    }

    Cell3<T> Pm{};
    T Ur = 0, Uu = 0, Uv = 0, Uw = 0, UE = 0;
    Flux3<T> fxlo{};
    int m = 0;
#pragma unroll 2
    for (; m < nplanes; ++m) {
        // the stage of plane m-1 is refilled with plane m+k3Stages-1 (every lane read it
        // before the previous plane's barrier). Halo loads: plane m landed before the
        // previous plane's barrier, and plane m+1 must land before this plane's. Own loads:
        // each lane waits for its own copy of plane m.
        const int s = m % k3Stages;
        if (loader) issue(m + k3Stages - 1);
        if (kHaloLoads) {
            if (loader) cp_async_wait<k3Stages - 2>();
        } else {
            cp_async_wait<k3Stages - 1>();
        }
        T ur = S.st[s][0][t], uE = S.st[s][1][t], uu = S.st[s][2][t], uv = S.st[s][3][t], uw = S.st[s][4][t];
        if (kEdge && !real) {
            ur = T(1);
            uE = T(1);
            uu = uv = uw = T(0);
        }
        const Cell3<T> P = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
        {
            typename Smem3<T, W>::V2 *x = &S.xP[m & 1][0][t];
            x[0 * (32 * W)] = pair3<T>(P.r, P.p);
            x[1 * (32 * W)] = pair3<T>(P.Ka, P.iKa);
            x[2 * (32 * W)] = pair3<T>(P.v, P.w);
            x[3 * (32 * W)] = pair3<T>(P.mu, P.mv);
            x[4 * (32 * W)] = pair3<T>(P.mw, P.eup_xy);
            if constexpr (!kF) x[5 * (32 * W)] = pair3<T>(P.eup_z, T(0));
        }
        // +y face of (j | j+1), from this lane's previous-plane cell and the warp above's
        auto yface = [&]() {
            const FaceIn3<T> me = face3_y(Pm);
            const FaceIn3<T> nb = xp_face_y<T, 32 * W>(&S.xP[(m - 1) & 1][0][t + 32]);
            FaceIn3<T> L = me, R = nb;
            if (kEdge) {
                if (j == 0) L = mirror3(nb);
                if (j == g.nb_y) R = mirror3(me);
            }
            return face_flux3<T, kF>(L, R, ph);
        };
        // +z face of (k | k+1): the next lane's cell from the exchange buffer (lane 31
        // reads the next warp's lane 0, a face no interior lane uses)
        auto zface = [&]() {
            const FaceIn3<T> mz = face3_z(Pm);
            const FaceIn3<T> nz = xp_face_z<T, 32 * W, kF>(&S.xP[(m - 1) & 1][0][t + 1]);
            FaceIn3<T> L = mz, R = nz;
            if (kEdge) {
                if (k == 0) L = mirror3(nz);
                if (k == g.nb_z) R = mirror3(mz);
            }
            return face_flux3<T, kF>(L, R, ph);
        };
        auto publish_y = [&](const Flux3<T> &fy) {
            S.xF[m & 1][0][t] = pair3<T>(fy.r, fy.n);
            S.xF[m & 1][1][t] = pair3<T>(fy.t1, fy.t2);
            S.xFE[m & 1][t] = fy.E;
        };
        Flux3<T> fxhi{};
        if (m >= 2) {
            // faces of plane m-1 (an interior plane when 2 <= m): the warps holding interior
            // rows evaluate their x, y and z faces together (independent work the compiler
            // can interleave); the halo row above them only its +y face
            Flux3<T> fy{}, fz{};
            if (iwarp) {
                fxhi = face_flux3<T, kF>(face3_x(Pm), face3_x(P), ph);
                fy = yface();
                fz = zface();
                publish_y(fy);
            } else if (w < W - 1) {
                fy = yface();
                publish_y(fy);
            }
            __syncthreads(); // +y faces of this plane published
            if (iwarp) {
                Flux3<T> fzl;
                fzl.r = __shfl_up_sync(FULL, fz.r, 1);
                fzl.n = __shfl_up_sync(FULL, fz.n, 1);
                fzl.t1 = __shfl_up_sync(FULL, fz.t1, 1);
                fzl.t2 = __shfl_up_sync(FULL, fz.t2, 1);
                fzl.E = __shfl_up_sync(FULL, fz.E, 1);
                if (interior) {
                    const auto a0 = S.xF[m & 1][0][t - 32], a1 = S.xF[m & 1][1][t - 32];
                    const Flux3<T> fyl{a0.x, a0.y, a1.x, a1.y, S.xFE[m & 1][t - 32]};
                    const Upd3<T> o =
                        update3<T, kF>(Ur, Uu, Uv, Uw, UE, fxlo, fxhi, fyl, fy, fzl, fz, DtDx, DtDy, DtDz, ph);
                    const long long c = (long long)(g.i0 + m - 2) * g.zy + colofs;
                    rhoE_n[2 * c] = o.r;
                    rhoE_n[2 * c + 1] = o.E;
                    uvw_n[3 * c] = o.u;
                    uvw_n[3 * c + 1] = o.v;
                    uvw_n[3 * c + 2] = o.w;
                    sink(o);
                }
            }
        } else {
            if (m >= 1 && iwarp) fxhi = face_flux3<T, kF>(face3_x(Pm), face3_x(P), ph);
            __syncthreads(); // keep one barrier per plane: publishes this plane's xP
        }
        fxlo = fxhi;
        Pm = P;
        Ur = ur; Uu = uu; Uv = uv; Uw = uw; UE = uE;
    }
    cp_async_wait<0>();
    return true;
}

// Per-lane copies, strict FP64: the plane loop written once per warp role, with the
// interior rows' +y / +z faces of plane m-1, conversion of plane m and x face in one block
// ahead of the barrier, as in the tensor-map form (FP64 with an odd NB_Z, 512 x 512 x 511:
// 31.3 -> 34.0 GCell/s, no spills against 12 bytes). FP32 keeps march3d_lane: this form
// ran 56.0 -> 57.2 GCell/s strict at 512^3 but 0.407 -> 0.454 ms at 256^3 (short chunks);
// in fused arithmetic it measured slower (FP32 63.6 -> 60.4, FP64 35.9 -> 30.7 with spills).
template <bool kEdge, bool kF, class T, int W, class Sink>
__device__ __forceinline__ bool march3d_lane_roles(Smem3<T, W> &S, const T *rhoE, const T *uvw, T *rhoE_n, T *uvw_n,
                                               const March3 &g, const Phys<T> &ph, T DtDx, T DtDy, T DtDz, Sink &sink)
{
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int NT = 32 * W;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int k = g.kbase + lane, j = g.jbase + w;
    const int nplanes = g.i1 - g.i0 + 3;
    const bool real = !kEdge || ((j >= 1) && (j <= g.nb_y) && (k >= 1) && (k <= g.nb_z));
    constexpr bool kHaloLoads = sizeof(T) == 4;
    const bool loader = kHaloLoads ? ((w == 0) || (w == W - 1)) : true;
    const int rbase = kHaloLoads ? ((w == 0) ? 0 : W / 2) : w;
    constexpr int kRows = kHaloLoads ? W / 2 : 1;
    const bool kin = !kEdge || (k <= g.nb_z + 1);

    __syncthreads();
    auto issue = [&](int m) {
        const int s = m % k3Stages;
        if (m < nplanes) {
            const long long pl =
                (long long)(g.xwrap ? wrap_plane(g.i0 - 1 + m, g.nb_x) : g.i0 - 1 + m) * g.zy + (long long)g.jbase * g.zs + k;
#pragma unroll
            for (int rr = 0; rr < kRows; ++rr) {
                const int r = rbase + rr;
                const bool ok = kin && (!kEdge || g.jbase + r <= g.nb_y + 1);
                const long long c = pl + (long long)r * g.zs;
                const T *pr = ok ? rhoE + 2 * c : rhoE;
                const T *pu = ok ? uvw + 3 * c : uvw;
                const int tt = 32 * r + lane;
                cp_async(&S.st[s][0][tt], pr, sizeof(T), ok);
                cp_async(&S.st[s][1][tt], pr + 1, sizeof(T), ok);
                cp_async(&S.st[s][2][tt], pu, sizeof(T), ok);
                cp_async(&S.st[s][3][tt], pu + 1, sizeof(T), ok);
                cp_async(&S.st[s][4][tt], pu + 2, sizeof(T), ok);
            }
        }
        cp_async_commit();
    };
    if (loader) {
#pragma unroll
        for (int m = 0; m < k3Stages - 1; ++m) issue(m);
    }
    if (kHaloLoads) {
        if (loader) cp_async_wait<k3Stages - 2>();
        __syncthreads();
    }
    // plane m into this lane's registers: the loading lanes refill the stage of plane m-1
    // and wait for their copies (halo loads: of plane m+1, made visible by this plane's
    // barrier; own loads: of plane m)
    auto load = [&](int m, T &ur, T &uE, T &uu, T &uv, T &uw) {
        const int s = m % k3Stages;
        if (loader) {
            issue(m + k3Stages - 1);
            if (kHaloLoads)
                cp_async_wait<k3Stages - 2>();
            else
                cp_async_wait<k3Stages - 1>();
        }
        ur = S.st[s][0][t];
        uE = S.st[s][1][t];
        uu = S.st[s][2][t];
        uv = S.st[s][3][t];
        uw = S.st[s][4][t];
        if (kEdge && !real) {
            ur = T(1);
            uE = T(1);
            uu = uv = uw = T(0);
        }
    };
    auto publish = [&](int m, const Cell3<T> &P) {
        typename Smem3<T, W>::V2 *x = &S.xP[m & 1][0][t];
        x[0 * NT] = pair3<T>(P.r, P.p);
        x[1 * NT] = pair3<T>(P.Ka, P.iKa);
        x[2 * NT] = pair3<T>(P.v, P.w);
        x[3 * NT] = pair3<T>(P.mu, P.mv);
        x[4 * NT] = pair3<T>(P.mw, P.eup_xy);
        if constexpr (!kF) x[5 * NT] = pair3<T>(P.eup_z, T(0));
    };
    auto yface = [&](int m, const Cell3<T> &Pme) {
        const FaceIn3<T> me = face3_y(Pme);
        const FaceIn3<T> nb = xp_face_y<T, NT>(&S.xP[(m - 1) & 1][0][t + 32]);
        FaceIn3<T> L = me, R = nb;
        if (kEdge) {
            if (j == 0) L = mirror3(nb);
            if (j == g.nb_y) R = mirror3(me);
        }
        return face_flux3<T, kF>(L, R, ph);
    };
    auto publish_y = [&](int m, const Flux3<T> &fy) {
        S.xF[m & 1][0][t] = pair3<T>(fy.r, fy.n);
        S.xF[m & 1][1][t] = pair3<T>(fy.t1, fy.t2);
        S.xFE[m & 1][t] = fy.E;
    };
    int m = 0;
    const bool iwarp = (w >= 1) && (w <= (W - 2)) && (!kEdge || (g.jbase + 1 <= g.nb_y));
    if (iwarp) {
        const bool interior = (lane >= 1) && (lane <= k3TZ) && (!kEdge || ((j <= g.nb_y) && (k <= g.nb_z)));
        const long long colofs = (long long)j * g.zs + k;
        Cell3<T> Pm{};
        T Ur = 0, Uu = 0, Uv = 0, Uw = 0, UE = 0;
        Flux3<T> fxlo{};
        auto zface = [&](int mm) {
            const FaceIn3<T> mz = face3_z(Pm);
            const FaceIn3<T> nz = xp_face_z<T, NT, kF>(&S.xP[(mm - 1) & 1][0][t + 1]);
            FaceIn3<T> L = mz, R = nz;
            if (kEdge) {
                if (k == 0) L = mirror3(nz);
                if (k == g.nb_z) R = mirror3(mz);
            }
            return face_flux3<T, kF>(L, R, ph);
        };
        for (; m < 2; ++m) {
            T ur, uE, uu, uv, uw;
            load(m, ur, uE, uu, uv, uw);
            const Cell3<T> P = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
            publish(m, P);
            if (m == 1) fxlo = face_flux3<T, kF>(face3_x(Pm), face3_x(P), ph);
            __syncthreads();
            Pm = P;
            Ur = ur; Uu = uu; Uv = uv; Uw = uw; UE = uE;
        }
#pragma unroll 2
        for (; m < nplanes; ++m) {
            T ur, uE, uu, uv, uw;
            load(m, ur, uE, uu, uv, uw);
            const Flux3<T> fy = yface(m, Pm);
            const Flux3<T> fz = zface(m);
            const Cell3<T> P = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
            const Flux3<T> fxhi = face_flux3<T, kF>(face3_x(Pm), face3_x(P), ph);
            publish_y(m, fy);
            publish(m, P);
            __syncthreads();
            Flux3<T> fzl;
            fzl.r = __shfl_up_sync(FULL, fz.r, 1);
            fzl.n = __shfl_up_sync(FULL, fz.n, 1);
            fzl.t1 = __shfl_up_sync(FULL, fz.t1, 1);
            fzl.t2 = __shfl_up_sync(FULL, fz.t2, 1);
            fzl.E = __shfl_up_sync(FULL, fz.E, 1);
            if (interior) {
                const auto a0 = S.xF[m & 1][0][t - 32], a1 = S.xF[m & 1][1][t - 32];
                const Flux3<T> fyl{a0.x, a0.y, a1.x, a1.y, S.xFE[m & 1][t - 32]};
                const Upd3<T> o = update3<T, kF>(Ur, Uu, Uv, Uw, UE, fxlo, fxhi, fyl, fy, fzl, fz, DtDx, DtDy, DtDz, ph);
                const long long c = (long long)(g.i0 + m - 2) * g.zy + colofs;
                rhoE_n[2 * c] = o.r;
                rhoE_n[2 * c + 1] = o.E;
                uvw_n[3 * c] = o.u;
                uvw_n[3 * c + 1] = o.v;
                uvw_n[3 * c + 2] = o.w;
                sink(o);
            }
            fxlo = fxhi;
            Pm = P;
            Ur = ur; Uu = uu; Uv = uv; Uw = uw; UE = uE;
        }
    } else if (w == 0) {
        Cell3<T> Pm0{};
        for (; m < nplanes; ++m) {
            T ur, uE, uu, uv, uw;
            load(m, ur, uE, uu, uv, uw);
            if (m >= 2) publish_y(m, yface(m, Pm0));
            const Cell3<T> P0 = make_cell3<T, kF>(ur, uu, uv, uw, uE, ph);
            publish(m, P0);
            __syncthreads();
            Pm0 = P0;
        }
    } else {
        for (; m < nplanes; ++m) {
            T ur, uE, uu, uv, uw;
            load(m, ur, uE, uu, uv, uw);
            publish(m, make_cell3<T, kF>(ur, uu, uv, uw, uE, ph));
            __syncthreads();
        }
    }
    cp_async_wait<0>();
    return true;
}

// One tile march: the lean form for tiles away from walls and ghosts, the general one
// elsewhere (the choice is uniform over the block). kF: fused arithmetic (hydro_math.cuh).
// kTma: planes staged by the tensor maps `tm` (march3d_init first); else per-lane copies
// (march3d_lane_roles in strict FP64 when kLaneRoles, else march3d_lane; the batched
// engine keeps march3d_lane, where the role split spills in its persistent loop).
// Returns false when a bounded barrier wait gave up.
template <class T, bool kF = false, bool kTma = false, int W = k3Warps<T>, bool kLaneRoles = true, class Sink>
__device__ __forceinline__ bool march3d(Smem3<T, W> &S, const T *rhoE, const T *uvw, T *rhoE_n, T *uvw_n,
                                        const March3 &g, const Phys<T> &ph, T DtDx, T DtDy, T DtDz, Sink &&sink,
                                        const Tmaps3 &tm = Tmaps3{})
{
    const bool inner = g.jbase >= 1 && g.jbase + W - 1 <= g.nb_y && g.kbase >= 1 && g.kbase + 31 <= g.nb_z;
    if constexpr (kTma) {
        if (inner) return march3d_tma<false, kF>(S, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, tm, sink);
        return march3d_tma<true, kF>(S, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, tm, sink);
    } else {
        if constexpr (!kF && kLaneRoles && sizeof(T) == 8) {
            if (inner) return march3d_lane_roles<false, kF>(S, rhoE, uvw, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, sink);
            return march3d_lane_roles<true, kF>(S, rhoE, uvw, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, sink);
        } else {
            if (inner) return march3d_lane<false, kF>(S, rhoE, uvw, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, sink);
            return march3d_lane<true, kF>(S, rhoE, uvw, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, sink);
        }
    }
}

// The same for the tile of W+1 rows on W warps (tensor maps only).
template <class T, bool kF = false, class Sink>
__device__ __forceinline__ bool march3d(Smem3P<T> &S, T *rhoE_n, T *uvw_n, const March3 &g, const Phys<T> &ph, T DtDx,
                                        T DtDy, T DtDz, Sink &&sink, const Tmaps3 &tm)
{
    constexpr int R = Smem3P<T>::W + 1;
    const bool inner = g.jbase >= 1 && g.jbase + R - 1 <= g.nb_y && g.kbase >= 1 && g.kbase + 31 <= g.nb_z;
    if (inner) return march3d_tma<false, kF>(S, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, tm, sink);
    return march3d_tma<true, kF>(S, rhoE_n, uvw_n, g, ph, DtDx, DtDy, DtDz, tm, sink);
}

} // namespace hydro
