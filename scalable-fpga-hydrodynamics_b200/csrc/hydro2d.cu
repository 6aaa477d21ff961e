// 2D finite-volume step on B200: the device replacement of kernel_hydro_fvm
// (hydro2d/kernel.cxx:132-319).
//
// Data layout (fixed by the reference host, hydro2d/main.cxx:80-81,120-128): the grid
// is (NB_X+2) x (NB_Y+2) cells, row-major with Y fastest, c = i*(NB_Y+2) + j. Two
// arrays of interleaved pairs: rhoE[c] = (rho, E), uv[c] = (rho*u, rho*v), i.e. one
// 16-byte (FP64) or 8-byte (FP32) vector per cell per array.
//
// Boundaries: X is periodic by in-kernel wrap (row 0 reads row NB_X, row NB_X+1 reads
// row 1: the single-rank ghost copy of hydro2d/main.cxx:349-378 done by addressing),
// so the ghost rows of the input are never read. Y walls are reflective: the face
// flux at j=1/2 and j=NB_Y+1/2 uses the mirrored state of the wall cell
// (hydro2d/kernel.cxx:212-251).
//
// Kernels:
//  strip2d   one CTA = 128 lanes over 128 consecutive columns (126 interior + one
//            halo column each side), marching down `chunk` rows. Each row arrives in
//            shared memory through two TMA tile loads (one per array) into a 4-deep
//            mbarrier ring (or per-lane cp.async where TMA rejects the row pitch); each
//            lane converts its cell to primitives once, computes the x face below it and
//            the y face to its right once (neighbour inputs and fluxes exchanged through
//            shared memory with 128-bit accesses), updates the row behind, stores it with
//            128-bit stores and folds mass, signal speed and the error checks into the
//            fused epilogue.
//  direct2d  one thread per cell, scalar loads of the 5-point stencil, every face
//            evaluated from both sides like the reference. Any alignment, any size;
//            used when the strip kernel's TMA rules do not hold and as a cross-check.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <stddef.h>
#include <stdio.h>

#include "../../include/hydro_b200.h"
#include "hydro_host.h"
#include "strip2d_march.cuh"

namespace hydro {

template <class T> struct Args2 {
    const T *rhoE, *uv;
    T *rhoE_n, *uv_n;
    T *Dt_next;
    Phys<T> ph;
    T DtDx, DtDy;
    int nb_x, nb_y;
    long long ys;
    int chunk;
    StepScratch *scr;
    double2 *partials;
    StepStatus *status;
    unsigned seq;
    unsigned long long key; // problem key for the signal-speed skip (0: never skip)
    float ggm1;             // gamma * (gamma - 1), for the signal-speed skip test
    int xwrap;              // X neighbours by periodic wrap (1) or from the ghost rows (0)
};

// The float skip threshold, rounded down so that every skipped cell is provably below
// the double threshold the last block checks against.
__device__ __forceinline__ float skip_threshold_f(const StepScratch *scr, unsigned long long key)
{
    return __double2float_rd(skip_threshold(scr, key));
}


// ------------------------------------------------------------------ direct kernel ---
constexpr int kDirectNT = 128;

template <class T> __device__ __forceinline__ Cell2<T> load_cell2(const Args2<T> &g, long long c)
{
    return make_cell2<T>(g.rhoE[2 * c], g.uv[2 * c], g.uv[2 * c + 1], g.rhoE[2 * c + 1], g.ph);
}

template <class T> __global__ void __launch_bounds__(kDirectNT) direct2d(Args2<T> g)
{
    StepAcc acc;
    const int j = 1 + blockIdx.x * kDirectNT + threadIdx.x;
    for (int i = 1 + blockIdx.y; i <= g.nb_x; i += gridDim.y) {
        if (j > g.nb_y) continue;
        const long long c = (long long)i * g.ys + j;
        const T ur = g.rhoE[2 * c], uE = g.rhoE[2 * c + 1], uu = g.uv[2 * c], uv = g.uv[2 * c + 1];
        const Cell2<T> P = make_cell2<T>(ur, uu, uv, uE, g.ph);
        const Cell2<T> PL = load_cell2(g, (long long)(g.xwrap ? wrap_row(i - 1, g.nb_x) : i - 1) * g.ys + j);
        const Cell2<T> PR = load_cell2(g, (long long)(g.xwrap ? wrap_row(i + 1, g.nb_x) : i + 1) * g.ys + j);
        const Flux2<T> fx1 = face_flux(face_x(PL), face_x(P), g.ph);
        const Flux2<T> fx2 = face_flux(face_x(P), face_x(PR), g.ph);
        const FaceIn<T> me = face_y(P);
        const FaceIn<T> lo = (j == 1) ? mirror(me) : face_y(load_cell2(g, c - 1));
        const FaceIn<T> hi = (j == g.nb_y) ? mirror(me) : face_y(load_cell2(g, c + 1));
        const Flux2<T> fy1 = face_flux(lo, me, g.ph);
        const Flux2<T> fy2 = face_flux(me, hi, g.ph);
        const Upd2<T> o = update2(ur, uu, uv, uE, fx1, fx2, fy1, fy2, g.DtDx, g.DtDy, g.ph);
        g.rhoE_n[2 * c] = o.r;
        g.rhoE_n[2 * c + 1] = o.E;
        g.uv_n[2 * c] = o.u;
        g.uv_n[2 * c + 1] = o.v;
        acc.add_cell(o.r, speed2(o.r, o.u, o.v, o.E, g.ph));
    }
    step_epilogue<kDirectNT, T>(acc, g.scr, g.partials, gridDim.x * gridDim.y, blockIdx.x + blockIdx.y * gridDim.x,
                                g.ph.C_min, g.Dt_next, g.status, g.seq, 0.0, g.key);
}

// Redo pass: the exact signal speed of every interior cell of the new state, when the
// step's skip threshold turned out too high (StepScratch::redo); exits at once otherwise.
constexpr int kRedoNT = 256;
template <class T, bool kF = false> __global__ void __launch_bounds__(kRedoNT) redo2d(Args2<T> g)
{
    if (*reinterpret_cast<const volatile unsigned *>(&g.scr->redo) == 0u) return;
    StepAcc acc;
    const long long n = (long long)g.nb_x * g.nb_y;
    for (long long q = blockIdx.x * (long long)kRedoNT + threadIdx.x; q < n; q += (long long)gridDim.x * kRedoNT) {
        const long long c = (1 + q / g.nb_y) * g.ys + 1 + q % g.nb_y;
        acc.add_speed(
            speed2<T, kF>(g.rhoE_n[2 * c], g.uv_n[2 * c], g.uv_n[2 * c + 1], g.rhoE_n[2 * c + 1], g.ph));
    }
    redo_epilogue<kRedoNT, T>(acc.vmax, acc.err, g.scr, gridDim.x, g.ph.C_min, g.Dt_next, g.status, g.key);
}

// ------------------------------------------------------------------- strip kernel ---
// kTma: rows staged by TMA tile loads (16-byte row pitch), else by per-lane cp.async.
// kF: fused arithmetic (hydro_math.cuh). kMinB: resident blocks per SM the registers are
// budgeted for (a launch-shape choice: more blocks, fewer registers per thread).
template <class T, bool kTma, bool kF, int kMinB = 4>
__global__ void __launch_bounds__(kStripNT, kMinB)
    strip2d(const __grid_constant__ CUtensorMap tmr, const __grid_constant__ CUtensorMap tmu, Args2<T> g)
{
    __shared__ Smem2<T> S;
    if (kTma && threadIdx.x == 0) {
        prefetch_tensormap(&tmr);
        prefetch_tensormap(&tmu);
    }
    march2d_init(S);
    const int i0 = 1 + g.chunk * (int)blockIdx.y;
    const March2 geo{kStripW * (int)blockIdx.x, i0, min(i0 + g.chunk - 1, g.nb_x), g.nb_x, g.nb_y, g.ys, g.xwrap,
                     g.rhoE, g.uv};
    StepAcc acc;
    const float tlof = skip_threshold_f(g.scr, g.key);
    const float tlo2 = skip_tlo2(tlof), ggm1 = g.ggm1;
    const Phys<T> ph = g.ph;
    unsigned ld = 0;
    const bool ok = march2d<T, kTma, kF>(S, &tmr, &tmu, geo, g.rhoE_n, g.uv_n, ph, g.DtDx, g.DtDy, ld,
                                         [&](const Upd2<T> &o) {
                                             acc.add_mass(o.r);
                                             if (!state_below(o, ggm1, tlo2))
                                                 acc.add_speed(speed2<T, kF>(o.r, o.u, o.v, o.E, ph));
                                         });
    if (!ok) acc.err |= kErrWaitTimeout;
    step_epilogue<kStripNT, T>(acc, g.scr, g.partials, gridDim.x * gridDim.y, blockIdx.x + blockIdx.y * gridDim.x,
                               g.ph.C_min, g.Dt_next, g.status, g.seq, (double)tlof, g.key);
}

// ------------------------------------------------------------- initial condition ---
// hydro2d/main.cxx:280-338: rho = u_in inside the circle of radius min(cx,cy)/3
// centred at ((NB_X+1)/2, (NB_Y+1)/2) in ghost-shifted indices, u_out outside;
// E = p/(gamma-1); zero momentum. First Dt = min over cells of C_min/(c_s + |u|).
// The local Dt of a uniform state at rest: C_min / (c_s + |u|) with the reference's
// per-cell operations (hydro2d/main.cxx:318-336), as the bits of a double.
template <class T>
__device__ __forceinline__ unsigned long long rest_dt_bits2(T ur, T uE, T C_min, T gamma, T gm1)
{
    using A = Ar<T>;
    const T inv = A::rcp(ur);
    const T qu = A::mul(T(0), inv), qv = A::mul(T(0), inv);
    const T temp = A::add(A::mul(qu, qu), A::mul(qv, qv));
    const T e_int = A::sub(A::mul(uE, inv), A::mul(A::half, temp));
    const T qp = A::mul(A::mul(gm1, ur), e_int);
    const T cs = A::sqrt(A::mul(A::mul(gamma, qp), inv));
    const T un = A::sqrt(temp);
    return (unsigned long long)__double_as_longlong((double)A::div(C_min, A::add(cs, un)));
}

// The circle splits the cells into two uniform states, so their energy p/(gamma-1) and
// local Dt are evaluated once per thread for the states its cells hold, not once per
// cell: the same operations on the same operands, hence the same bits. Per cell: the
// distance test and the stores. Each thread covers the rows i = 1 + blockIdx.y + k *
// gridDim.y of its column j.
template <class T>
__global__ void init2d_kernel(T *rhoE, T *uv, int nb_x, int nb_y, long long ys, double cx, double cy, double radius,
                              T u_in, T u_out, T p_in, T p_out, T C_min, T gamma, T gm1, unsigned long long *min_bits)
{
    using A = Ar<T>;
    const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const T E_in = A::div(p_in, gm1), E_out = A::div(p_out, gm1);
    bool any_in = false, any_out = false;
    if (j <= nb_y) {
        const double dy = __dsub_rn((double)j, cy), dy2 = __dmul_rn(dy, dy);
        for (int i = 1 + blockIdx.y; i <= nb_x; i += gridDim.y) {
            const double dx = __dsub_rn((double)i, cx);
            const double d = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), dy2));
            const bool in = d <= radius;
            const long long c = (long long)i * ys + j;
            rhoE[2 * c] = in ? u_in : u_out;
            rhoE[2 * c + 1] = in ? E_in : E_out;
            uv[2 * c] = T(0);
            uv[2 * c + 1] = T(0);
            any_in |= in;
            any_out |= !in;
        }
    }
    unsigned long long best = ~0ull;
    if (any_in) best = rest_dt_bits2(u_in, E_in, C_min, gamma, gm1);
    if (any_out) {
        const unsigned long long b = rest_dt_bits2(u_out, E_out, C_min, gamma, gm1);
        best = b < best ? b : best;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(0xffffffffu, best, o);
        best = ob < best ? ob : best;
    }
    if ((threadIdx.x & 31) == 0 && best != ~0ull) atomicMin(min_bits, best);
}

// ------------------------------------------------------------------ mass kernel ---
// Warp-wide compensated merge in a fixed lane order; the result lands in every lane.
__device__ __forceinline__ void warp_neumaier(double &s, double &c)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double s2 = __shfl_xor_sync(0xffffffffu, s, o);
        const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
        if (lane & o) {
            double a = s2, b = c2;
            neumaier_merge(a, b, s, c);
            s = a;
            c = b;
        } else {
            neumaier_merge(s, c, s2, c2);
        }
    }
}

// Compensated sum of the interior density, one partial per block. Rows of interior
// cells (2D: i; 3D: (i, j)) go to blocks in turn and their cells to the threads, so
// each cell's address needs no division.
template <class T>
__global__ void mass_kernel(const T *rhoE, int nb_x, int nb_y, int nb_z, double2 *partials)
{
    const bool three = nb_z > 0;
    const long long zs = three ? (long long)nb_z + 2 : 1;
    const long long ys = (long long)(nb_y + 2) * zs;
    const int nj = three ? nb_y : 1; // rows (i, j): j only in 3D
    const int rowlen = three ? nb_z : nb_y;
    const int step_i = (int)(gridDim.x / nj), step_j = (int)(gridDim.x % nj);
    int i = (int)(blockIdx.x / nj), j = (int)(blockIdx.x % nj);
    double s = 0.0, c = 0.0;
    while (i < nb_x) {
        const long long base = (1 + (long long)i) * ys + (three ? (1 + (long long)j) * zs : 0) + 1;
        for (int t = threadIdx.x; t < rowlen; t += blockDim.x) neumaier_add(s, c, (double)rhoE[2 * (base + t)]);
        i += step_i;
        j += step_j;
        if (j >= nj) {
            j -= nj;
            ++i;
        }
    }
    __shared__ double ss[32], sc[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    warp_neumaier(s, c);
    if (lane == 0) { ss[warp] = s; sc[warp] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) neumaier_merge(s, c, ss[w], sc[w]);
        partials[blockIdx.x] = make_double2(s, c);
    }
}

// One warp: lane l merges partials l, l + 32, ... in order, then the lanes merge in a
// fixed order (deterministic).
__global__ void sum_partials_kernel(const double2 *partials, int n, double *out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    double s = 0.0, c = 0.0;
    for (int b = threadIdx.x; b < n; b += 32) neumaier_merge(s, c, partials[b].x, partials[b].y);
    warp_neumaier(s, c);
    if (threadIdx.x == 0) *out = __dadd_rn(s, c);
}

// ----------------------------------------------------------------- host drivers ---
namespace {
template <class T> CUtensorMapDataType tmap_type();
template <> CUtensorMapDataType tmap_type<double>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT64; }
template <> CUtensorMapDataType tmap_type<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }

bool aligned(const void *p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }
} // namespace

template <class T, int kMinB>
void launch_strip2d(bool tma, bool fused, dim3 grid, cudaStream_t stream, const CUtensorMap &tmr,
                    const CUtensorMap &tmu, const Args2<T> &g)
{
    if (tma && fused)
        strip2d<T, true, true, kMinB><<<grid, kStripNT, 0, stream>>>(tmr, tmu, g);
    else if (tma)
        strip2d<T, true, false, kMinB><<<grid, kStripNT, 0, stream>>>(tmr, tmu, g);
    else if (fused)
        strip2d<T, false, true, kMinB><<<grid, kStripNT, 0, stream>>>(tmr, tmu, g);
    else
        strip2d<T, false, false, kMinB><<<grid, kStripNT, 0, stream>>>(tmr, tmu, g);
}

template <class T>
int step2d(const T *rhoE, const T *uv, T *rhoE_next, T *uv_next, T *Dt_next, const Phys<T> &ph, size_t nb_x,
           size_t nb_y, T DtDx, T DtDy, cudaStream_t stream, Kernel which, bool sync, StepInfo *info, bool xwrap,
           bool fused)
{
    if (!rhoE || !uv || !rhoE_next || !uv_next || !Dt_next) {
        set_error(kErrArg, "step2d: null pointer argument");
        return kErrArg;
    }
    if (nb_x > (1u << 30) || nb_y > (1u << 30) || (nb_x + 2) * (nb_y + 2) > (size_t(1) << 40)) {
        set_error(kErrArg, "step2d: grid %zu x %zu too large", nb_x, nb_y);
        return kErrArg;
    }
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    if (nb_x == 0 || nb_y == 0) {
        // no interior cell: the reference leaves max_speed at 0 and writes C_min / 0
        const T dt = div_zero(ph.C_min);
        cudaError_t e = cudaMemcpyAsync(Dt_next, &dt, sizeof(T), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            set_error(kErrCuda, "step2d: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        if (info) *info = StepInfo{};
        return kOk;
    }
    if (ctx->dirty) {
        cudaMemsetAsync(ctx->scr, 0, sizeof(StepScratch), stream);
        ctx->dirty = false;
    }

    Args2<T> g;
    g.rhoE = rhoE; g.uv = uv; g.rhoE_n = rhoE_next; g.uv_n = uv_next; g.Dt_next = Dt_next;
    g.ph = ph; g.DtDx = DtDx; g.DtDy = DtDy;
    g.nb_x = (int)nb_x; g.nb_y = (int)nb_y; g.ys = (long long)nb_y + 2;
    g.scr = ctx->scr; g.status = ctx->status_d; g.seq = ++ctx->seq;
    g.key = problem_key(Dt_next, nb_x, nb_y, 0, sizeof(T), ph);
    g.ggm1 = skip_ggm1(ph.gamma, ph.gm1);
    g.xwrap = xwrap ? 1 : 0;

    using V2 = typename Vec2<T>::type;
    const size_t rowbytes = 2 * sizeof(T) * (nb_y + 2);
    // the strip kernel stages rows by TMA when the arrays are 16-byte aligned and the row
    // pitch a multiple of 16 bytes, else by per-lane cp.async (cells aligned to their size)
    bool tma_ok = aligned(rhoE, 16) && aligned(uv, 16) && aligned(rhoE_next, sizeof(V2)) &&
                  aligned(uv_next, sizeof(V2)) && rowbytes % 16 == 0;
    CUtensorMap tmr, tmu;
    std::memset(&tmr, 0, sizeof tmr);
    std::memset(&tmu, 0, sizeof tmu);
    if (tma_ok && which != Kernel::Direct) {
        tma_ok = encode_tmap_2d(&tmr, tmap_type<T>(), rhoE, 2 * (nb_y + 2), nb_x + 2, rowbytes, 2 * kStripNT, 1) &&
                 encode_tmap_2d(&tmu, tmap_type<T>(), uv, 2 * (nb_y + 2), nb_x + 2, rowbytes, 2 * kStripNT, 1);
    }
    const bool strip_ok = tma_ok || (aligned(rhoE, sizeof(V2)) && aligned(uv, sizeof(V2)) &&
                                     aligned(rhoE_next, sizeof(V2)) && aligned(uv_next, sizeof(V2)));
    if (which == Kernel::Strip && !strip_ok) {
        set_error(kErrArg, "step2d: strip kernel needs arrays aligned to their cell size");
        return kErrArg;
    }
    const bool use_strip = strip_ok && which != Kernel::Direct;

    cudaError_t e;
    unsigned nblocks;
    if (use_strip) {
        const int nstrips = (int)((nb_y + kStripW - 1) / kStripW);
        // rows per block: sized for about 24 blocks per SM, at least 16 and at most the cap
        // (the tuned value when one is set with hydro_set_launch_shape, else 256), so that
        // small grids still fill the GPU
        const LaunchShape shape = launch_shape(2, sizeof(T));
        const int cap = shape.chunk > 0 ? shape.chunk : 256;
        const int target = device_sms() * 3 * 8;
        int nchunks = (target + nstrips - 1) / nstrips;
        int chunk = (int)((nb_x + nchunks - 1) / nchunks);
        chunk = std::min(cap, std::max(std::min(16, cap), chunk));
        nchunks = (int)((nb_x + chunk - 1) / chunk);
        if (nchunks > 65535) {
            chunk = (int)((nb_x + 65534) / 65535);
            nchunks = (int)((nb_x + chunk - 1) / chunk);
        }
        g.chunk = chunk;
        nblocks = (unsigned)nstrips * (unsigned)nchunks;
        if ((err = ctx_reserve(ctx, nblocks)) != kOk) return err;
        g.partials = ctx->partials;
        ctx->last_warps = 0;
        ctx->last_chunk = chunk;
        ctx->last_tma = tma_ok;
        const dim3 grid(nstrips, nchunks);
        constexpr int kAltB = sizeof(T) == 8 ? 5 : 8; // the other register budget built
        const bool alt = shape.blocks == kAltB;
        ctx->last_blocks = alt ? kAltB : 4;
        if (alt)
            launch_strip2d<T, kAltB>(tma_ok, fused, grid, stream, tmr, tmu, g);
        else
            launch_strip2d<T, 4>(tma_ok, fused, grid, stream, tmr, tmu, g);
    } else {
        const int gx = (int)((nb_y + kDirectNT - 1) / kDirectNT);
        const int gy = (int)std::min<size_t>(nb_x, 65535);
        nblocks = (unsigned)gx * (unsigned)gy;
        if ((err = ctx_reserve(ctx, nblocks)) != kOk) return err;
        g.partials = ctx->partials;
        g.chunk = 0;
        direct2d<T><<<dim3(gx, gy), kDirectNT, 0, stream>>>(g);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx->dirty = true;
        set_error(kErrCuda, "step2d launch: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    ctx->last_kernel = (int)(use_strip ? Kernel::Strip : Kernel::Direct);
    const unsigned redo_blocks = (unsigned)device_sms() * 4;
    // the redo pass recomputes the signal speed in the arithmetic of the step that ran
    // (the direct kernel is always strict)
    const bool fused_ran = fused && use_strip;
    auto redo = [&]() {
        if (fused_ran)
            redo2d<T, true><<<redo_blocks, kRedoNT, 0, stream>>>(g);
        else
            redo2d<T, false><<<redo_blocks, kRedoNT, 0, stream>>>(g);
    };
    if (!sync) {
        // enqueued unconditionally; returns at once unless the step asked for it
        redo();
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            ctx->dirty = true;
            set_error(kErrCuda, "step2d launch: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        if (info) info->kernel = ctx->last_kernel;
        return kOk;
    }
    e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && read_status(ctx->status_h).redo) {
        redo();
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    }
    if (e != cudaSuccess) {
        ctx->dirty = true;
        set_error(kErrCuda, "step2d: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    const StepStatus st = read_status(ctx->status_h);
    if (info) {
        info->mass = st.mass + st.mass_comp;
        info->max_speed = st.max_speed;
        info->err = st.err;
        info->kernel = (int)(use_strip ? Kernel::Strip : Kernel::Direct);
    }
    if (st.err & kErrWaitTimeout) {
        ctx->dirty = true;
        set_error(kErrTimeout, "step2d: a TMA barrier wait timed out");
        return kErrTimeout;
    }
    if (st.err & kErrNonPhysical) {
        set_error(kErrPhys, "step2d: non-physical state (rho <= 0 or non-finite signal speed)");
        return kErrPhys;
    }
    return kOk;
}

template <class T>
int init2d_at(T *rhoE, T *uv, size_t nb_x, size_t nb_y, double cx, double cy, double radius, T u_in, T u_out, T p_in,
              T p_out, T C_min, T gamma, T *min_dt, cudaStream_t stream, unsigned long long *bits, long long ys)
{
    if (!rhoE || !uv || !min_dt || !bits || nb_x == 0 || nb_y == 0 || nb_x > (1u << 30) || nb_y > (1u << 30)) {
        set_error(kErrArg, "init2d: invalid argument");
        return kErrArg;
    }
    const T big = T(1e20);
    const unsigned long long init = (unsigned long long)__builtin_bit_cast(long long, (double)big);
    const T gm1 = gamma - T(1);
    cudaError_t e = cudaMemcpyAsync(bits, &init, sizeof init, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        // 16 blocks of 128 threads per SM; each thread takes nb_x / gy rows of its column
        const int gx = (int)((nb_y + 127) / 128);
        const int gy = (int)std::max<size_t>(1, std::min<size_t>({nb_x, 65535, (size_t)std::max(1, device_sms() * 16 / gx)}));
        init2d_kernel<T><<<dim3(gx, gy), 128, 0, stream>>>(rhoE, uv, (int)nb_x, (int)nb_y, ys > 0 ? ys : (long long)nb_y + 2, cx, cy,
                                                           radius, u_in, u_out, p_in, p_out, C_min, gamma, gm1, bits);
        e = cudaGetLastError();
    }
    unsigned long long res = 0;
    const unsigned long long zero = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&res, bits, sizeof res, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bits, &zero, sizeof zero, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "init2d: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    *min_dt = (T)__builtin_bit_cast(double, (long long)res);
    return kOk;
}

template <class T>
int init2d(T *rhoE, T *uv, size_t nb_x, size_t nb_y, T u_in, T u_out, T p_in, T p_out, T C_min, T gamma,
           T *min_dt, cudaStream_t stream)
{
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    // the reference's circle: centre ((NB_X+1)/2, (NB_Y+1)/2), radius min(cx, cy)/3
    const double cx = double(nb_x + 1) / 2.0, cy = double(nb_y + 1) / 2.0;
    const double radius = std::min(cx, cy) / 3;
    // the scratch max word is borrowed while no step is in flight
    return init2d_at<T>(rhoE, uv, nb_x, nb_y, cx, cy, radius, u_in, u_out, p_in, p_out, C_min, gamma, min_dt, stream,
                        &ctx->scr->max_bits);
}

template <class T> int mass_sum(const T *rhoE, size_t nb_x, size_t nb_y, size_t nb_z, double *out, cudaStream_t s)
{
    if (!rhoE || !out) {
        set_error(kErrArg, "mass_sum: null pointer");
        return kErrArg;
    }
    if (nb_x == 0 || nb_y == 0) {
        *out = 0.0;
        return kOk;
    }
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    const int nb = device_sms() * 8;
    if ((err = ctx_reserve(ctx, nb + 1)) != kOk) return err;
    double *dres = reinterpret_cast<double *>(ctx->partials + nb);
    mass_kernel<T><<<nb, 256, 0, s>>>(rhoE, (int)nb_x, (int)nb_y, (int)nb_z, ctx->partials);
    sum_partials_kernel<<<1, 32, 0, s>>>(ctx->partials, nb, dres);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dres, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "mass_sum: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    return kOk;
}

template int step2d<double>(const double *, const double *, double *, double *, double *, const Phys<double> &,
                            size_t, size_t, double, double, cudaStream_t, Kernel, bool, StepInfo *, bool, bool);
template int step2d<float>(const float *, const float *, float *, float *, float *, const Phys<float> &, size_t,
                           size_t, float, float, cudaStream_t, Kernel, bool, StepInfo *, bool, bool);
template int init2d<double>(double *, double *, size_t, size_t, double, double, double, double, double, double,
                            double *, cudaStream_t);
template int init2d_at<double>(double *, double *, size_t, size_t, double, double, double, double, double, double,
                               double, double, double, double *, cudaStream_t, unsigned long long *, long long);
template int init2d_at<float>(float *, float *, size_t, size_t, double, double, double, float, float, float, float,
                              float, float, float *, cudaStream_t, unsigned long long *, long long);
template int init2d<float>(float *, float *, size_t, size_t, float, float, float, float, float, float, float *,
                           cudaStream_t);
template int mass_sum<double>(const double *, size_t, size_t, size_t, double *, cudaStream_t);
template int mass_sum<float>(const float *, size_t, size_t, size_t, double *, cudaStream_t);

} // namespace hydro

// ------------------------------------------------------------ allocation-free step ---
// hydro2d_step_f64_noalloc: the 2D FP64 step for callers that cannot allocate device or
// pinned host memory. All scratch of the step (the reduction words, one partial sum per
// block, the status record) lives in the fixed array below, which every GPU that loads
// this library holds until the process exits.
namespace hydro {
namespace {

constexpr unsigned kNoAllocMaxBlocks = 65536; // at most this many blocks per launch
constexpr size_t kNoAllocHeader = 256;         // StepScratch, then StepStatus
constexpr size_t kNoAllocBytes = kNoAllocHeader + size_t(kNoAllocMaxBlocks) * sizeof(double2);
static_assert(sizeof(StepScratch) + sizeof(StepStatus) <= kNoAllocHeader, "header layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// The array's device address differs per CUDA context (a device's primary context, or a
// context the caller created with the driver API), so it is looked up once per context
// and kept with the kernel the context's last step ran.
struct NoAllocEntry {
    CUcontext ctx;
    unsigned char *base;
    int last_kernel;
};
std::mutex g_noalloc_mu;
NoAllocEntry g_noalloc[128];
int g_noalloc_n = 0;

CUcontext current_context()
{
    using Fn = CUresult (*)(CUcontext *);
    static Fn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<Fn>(p);
    });
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// The entry of the current context, created (address looked up) on its first use.
NoAllocEntry *noalloc_entry(const char *who, int *rc)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "%s: cudaGetDevice failed: %s", who, cudaGetErrorString(e));
        *rc = kErrCuda;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    CUcontext ctx = current_context();
    for (int i = 0; ctx && i < g_noalloc_n; ++i)
        if (g_noalloc[i].ctx == ctx) {
            *rc = kOk;
            return &g_noalloc[i];
        }
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch); // makes the device's context current if none was
    if (e != cudaSuccess || !p) {
        set_error(kErrCuda, "%s: cudaGetSymbolAddress failed: %s", who, cudaGetErrorString(e));
        *rc = kErrCuda;
        return nullptr;
    }
    ctx = current_context();
    for (int i = 0; ctx && i < g_noalloc_n; ++i)
        if (g_noalloc[i].ctx == ctx) {
            *rc = kOk;
            return &g_noalloc[i];
        }
    if (!ctx || g_noalloc_n == (int)(sizeof g_noalloc / sizeof g_noalloc[0])) {
        set_error(kErrCuda, "%s: no current CUDA context, or too many contexts", who);
        *rc = kErrCuda;
        return nullptr;
    }
    g_noalloc[g_noalloc_n] = NoAllocEntry{ctx, static_cast<unsigned char *>(p), 0};
    *rc = kOk;
    return &g_noalloc[g_noalloc_n++];
}

// Launch shape of the allocation-free step: the strip kernel's grid as step2d sizes it,
// with the chunk grown until the blocks fit the fixed partials, or the direct kernel's
// grid capped the same way. Returns the number of blocks, 0 if the grid cannot fit.
unsigned noalloc_shape(size_t nb_x, size_t nb_y, bool strip, int sms, int *chunk, unsigned *gx, unsigned *gy)
{
    if (nb_x == 0 || nb_y == 0 || sms <= 0) return 0;
    if (strip) {
        const size_t nstrips = (nb_y + kStripW - 1) / kStripW;
        if (nstrips > kNoAllocMaxBlocks) return 0;
        const size_t max_chunks = std::min<size_t>(kNoAllocMaxBlocks / nstrips, 65535);
        const size_t target = (size_t)sms * 3 * 8;
        size_t nchunks = (target + nstrips - 1) / nstrips;
        size_t c = std::min<size_t>(256, std::max<size_t>(16, (nb_x + nchunks - 1) / nchunks));
        c = std::max(c, (nb_x + max_chunks - 1) / max_chunks);
        nchunks = (nb_x + c - 1) / c;
        *chunk = (int)c;
        *gx = (unsigned)nstrips;
        *gy = (unsigned)nchunks;
    } else {
        const size_t gxd = (nb_y + kDirectNT - 1) / kDirectNT;
        if (gxd > kNoAllocMaxBlocks) return 0;
        *chunk = 0;
        *gx = (unsigned)gxd;
        *gy = (unsigned)std::max<size_t>(1, std::min<size_t>({nb_x, 65535, kNoAllocMaxBlocks / gxd}));
    }
    return *gx * *gy;
}

} // namespace
} // namespace hydro

extern "C" int hydro2d_step_f64_noalloc(const double *d_rhoE, const double *d_uv, double *d_rhoE_next,
                                        double *d_uv_next, double *Dt_next, double C_min, double gamma,
                                        double gamma_minus_one, double divgamma, double K, size_t NB_X, size_t NB_Y,
                                        double DtDx, double DtDy, void *stream, int sync, hydro_step_info_t *info)
{
    using namespace hydro;
    using T = double;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!d_rhoE || !d_uv || !d_rhoE_next || !d_uv_next || !Dt_next) {
        set_error(kErrArg, "hydro2d_step_f64_noalloc: null pointer argument");
        return kErrArg;
    }
    const size_t nstrips = NB_Y == 0 ? 0 : (NB_Y + kStripW - 1) / kStripW;
    const size_t gx_direct = NB_Y == 0 ? 0 : (NB_Y + kDirectNT - 1) / kDirectNT;
    if (NB_X > (1u << 30) || NB_Y > (1u << 30) || nstrips > kNoAllocMaxBlocks || gx_direct > kNoAllocMaxBlocks) {
        set_error(kErrArg,
                  "hydro2d_step_f64_noalloc: grid %zu x %zu exceeds the fixed scratch (at most %u blocks of "
                  "partial sums: NB_Y <= %zu)",
                  NB_X, NB_Y, kNoAllocMaxBlocks, size_t(kStripW) * kNoAllocMaxBlocks);
        return kErrArg;
    }
    int rc;
    NoAllocEntry *ent = noalloc_entry("hydro2d_step_f64_noalloc", &rc);
    if (!ent) return rc;
    unsigned char *base = ent->base;
    StepScratch *scr = reinterpret_cast<StepScratch *>(base);
    StepStatus *status = reinterpret_cast<StepStatus *>(base + sizeof(StepScratch));
    double2 *partials = reinterpret_cast<double2 *>(base + kNoAllocHeader);

    const Phys<T> ph = Phys<T>::make(C_min, gamma, gamma_minus_one, divgamma, K);
    if (NB_X == 0 || NB_Y == 0) {
        const T dt = div_zero(C_min);
        cudaError_t e = cudaMemcpyAsync(Dt_next, &dt, sizeof(T), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            set_error(kErrCuda, "hydro2d_step_f64_noalloc: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        if (info) *info = hydro_step_info_t{0.0, 0.0, 0u, 0};
        return kOk;
    }
    // the reduction words and the status record must start at zero: clear them (the skip
    // history between them is kept, a stale one only costs a redo pass)
    cudaError_t e = cudaMemsetAsync(scr, 0, offsetof(StepScratch, hist_key), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(StepStatus), st);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "hydro2d_step_f64_noalloc: %s", cudaGetErrorString(e));
        return kErrCuda;
    }

    Args2<T> g;
    g.rhoE = d_rhoE; g.uv = d_uv; g.rhoE_n = d_rhoE_next; g.uv_n = d_uv_next; g.Dt_next = Dt_next;
    g.ph = ph; g.DtDx = DtDx; g.DtDy = DtDy;
    g.nb_x = (int)NB_X; g.nb_y = (int)NB_Y; g.ys = (long long)NB_Y + 2;
    g.scr = scr; g.partials = partials; g.status = status; g.seq = 0;
    g.key = problem_key(Dt_next, NB_X, NB_Y, 0, sizeof(T), ph);
    g.ggm1 = skip_ggm1(gamma, gamma_minus_one);
    g.xwrap = 1;

    const size_t rowbytes = 2 * sizeof(T) * (NB_Y + 2);
    bool strip_ok = aligned(d_rhoE, 16) && aligned(d_uv, 16) && aligned(d_rhoE_next, 16) && aligned(d_uv_next, 16) &&
                    rowbytes % 16 == 0;
    CUtensorMap tmr, tmu;
    if (strip_ok)
        strip_ok = encode_tmap_2d(&tmr, tmap_type<T>(), d_rhoE, 2 * (NB_Y + 2), NB_X + 2, rowbytes, 2 * kStripNT, 1) &&
                   encode_tmap_2d(&tmu, tmap_type<T>(), d_uv, 2 * (NB_Y + 2), NB_X + 2, rowbytes, 2 * kStripNT, 1);
    int chunk = 0;
    unsigned gx = 0, gy = 0;
    if (!noalloc_shape(NB_X, NB_Y, strip_ok, device_sms(), &chunk, &gx, &gy)) {
        set_error(kErrArg, "hydro2d_step_f64_noalloc: grid %zu x %zu exceeds the fixed scratch", NB_X, NB_Y);
        return kErrArg;
    }
    g.chunk = chunk;
    const int kernel = (int)(strip_ok ? Kernel::Strip : Kernel::Direct);
    if (strip_ok)
        strip2d<T, true, false><<<dim3(gx, gy), kStripNT, 0, st>>>(tmr, tmu, g);
    else
        direct2d<T><<<dim3(gx, gy), kDirectNT, 0, st>>>(g);
    // the redo pass returns at once unless the step left Dt_next to it
    redo2d<T><<<(unsigned)device_sms() * 4, kRedoNT, 0, st>>>(g);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(kErrCuda, "hydro2d_step_f64_noalloc launch: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        ent->last_kernel = kernel;
    }
    if (!sync) {
        if (info) info->kernel = kernel;
        return kOk;
    }
    StepStatus s;
    e = cudaMemcpyAsync(&s, status, sizeof s, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "hydro2d_step_f64_noalloc: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    if (info) *info = hydro_step_info_t{s.mass + s.mass_comp, s.max_speed, s.err, kernel};
    if (s.err & kErrWaitTimeout) {
        set_error(kErrTimeout, "hydro2d_step_f64_noalloc: a TMA barrier wait timed out");
        return kErrTimeout;
    }
    if (s.err & kErrNonPhysical) {
        set_error(kErrPhys, "hydro2d_step_f64_noalloc: non-physical state (rho <= 0 or non-finite signal speed)");
        return kErrPhys;
    }
    return kOk;
}

extern "C" int hydro2d_noalloc_last_info(void *stream, hydro_step_info_t *info)
{
    using namespace hydro;
    if (!info) {
        set_error(kErrArg, "hydro2d_noalloc_last_info: null info");
        return kErrArg;
    }
    int rc;
    NoAllocEntry *ent = noalloc_entry("hydro2d_noalloc_last_info", &rc);
    if (!ent) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    StepStatus s;
    cudaError_t e = cudaMemcpyAsync(&s, ent->base + sizeof(StepScratch), sizeof s, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "hydro2d_noalloc_last_info: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    int kernel;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        kernel = ent->last_kernel;
    }
    *info = hydro_step_info_t{s.mass + s.mass_comp, s.max_speed, s.err, kernel};
    if (s.err & kErrWaitTimeout) return kErrTimeout;
    return (s.err & kErrNonPhysical) ? kErrPhys : kOk;
}

extern "C" unsigned hydro2d_noalloc_launch_shape(size_t NB_X, size_t NB_Y, int strip, int sms, int *chunk,
                                                 unsigned *grid_x, unsigned *grid_y)
{
    int c = 0;
    unsigned gx = 0, gy = 0;
    const unsigned n = hydro::noalloc_shape(NB_X, NB_Y, strip != 0, sms, &c, &gx, &gy);
    if (chunk) *chunk = c;
    if (grid_x) *grid_x = gx;
    if (grid_y) *grid_y = gy;
    return n;
}
