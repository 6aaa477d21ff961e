// 3D finite-volume step on B200: the device replacement of kernel_hydro3d_fvm
// (hydro3d/kernel.cxx:145-407).
//
// Layout (hydro3d/main.cxx:80-87,120-130): (NB_X+2)(NB_Y+2)(NB_Z+2) cells, Z fastest,
// c = i*(NB_Y+2)(NB_Z+2) + j*(NB_Z+2) + k; rhoE[c] = (rho, E) pairs and
// uvw[c] = (rho*u, rho*v, rho*w) triples.
// Boundaries: periodic X by in-kernel wrap; reflective Y and Z walls from the mirrored
// wall cell (hydro3d/kernel.cxx:238-320).
//
// Kernels:
//  strip3d   one CTA of W warps over a tile of rows (y) x 32 (z) columns with a one-cell
//            halo ring, marching down `chunk` X planes: by default 9 rows on 8 warps
//            (7 x 30 interior cells; warp 0 holds both halo rows) where tensor maps stage
//            the planes (FP64, even NB_Z), else 8 rows on 8 warps (6 x 30). Planes arrive
//            in a shared-memory ring by tensor-map TMA loads or per-lane cp.async (any
//            alignment of the interleaved pairs/triples); each lane converts its cell to
//            primitives once and per plane computes one x face (registers), one z face
//            (flux back by warp shuffles) and one y face (shared memory, double-buffered by
//            plane parity, one barrier per plane), then updates the plane behind it.
//  direct3d  one thread per cell, the 7-point stencil loaded directly, every face
//            evaluated from both sides like the reference.
#include <algorithm>
#include <type_traits>
#include <cstring>
#include <stdio.h>

#include "hydro_host.h"
#include "strip3d_march.cuh"

namespace hydro {

template <class T> struct Args3 {
    const T *rhoE, *uvw;
    T *rhoE_n, *uvw_n;
    T *Dt_next;
    Phys<T> ph;
    T DtDx, DtDy, DtDz;
    int nb_x, nb_y, nb_z;
    long long zs, zy;
    int chunk;
    StepScratch *scr;
    double2 *partials;
    StepStatus *status;
    unsigned seq;
    unsigned long long key; // problem key for the signal-speed skip (0: never skip)
    float ggm1;             // gamma * (gamma - 1), for the signal-speed skip test
    int xwrap;              // X neighbours by periodic wrap (1) or from the ghost planes (0)
};


template <class T> __device__ __forceinline__ Cell3<T> load_cell3(const Args3<T> &g, long long c)
{
    return make_cell3<T>(g.rhoE[2 * c], g.uvw[3 * c], g.uvw[3 * c + 1], g.uvw[3 * c + 2], g.rhoE[2 * c + 1], g.ph);
}

// ------------------------------------------------------------------ direct kernel ---
template <class T> __global__ void __launch_bounds__(128) direct3d(Args3<T> g)
{
    StepAcc acc;
    const int k = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    for (int i = 1 + blockIdx.z; i <= g.nb_x; i += gridDim.z) {
        if (k > g.nb_z || j > g.nb_y) continue;
        const long long c = (long long)i * g.zy + (long long)j * g.zs + k;
        const T ur = g.rhoE[2 * c], uE = g.rhoE[2 * c + 1];
        const T uu = g.uvw[3 * c], uv = g.uvw[3 * c + 1], uw = g.uvw[3 * c + 2];
        const Cell3<T> P = make_cell3<T>(ur, uu, uv, uw, uE, g.ph);
        const long long cxm = (long long)(g.xwrap ? wrap_plane(i - 1, g.nb_x) : i - 1) * g.zy + (long long)j * g.zs + k;
        const long long cxp = (long long)(g.xwrap ? wrap_plane(i + 1, g.nb_x) : i + 1) * g.zy + (long long)j * g.zs + k;
        const Flux3<T> fx1 = face_flux3(face3_x(load_cell3(g, cxm)), face3_x(P), g.ph);
        const Flux3<T> fx2 = face_flux3(face3_x(P), face3_x(load_cell3(g, cxp)), g.ph);
        const FaceIn3<T> my = face3_y(P);
        const FaceIn3<T> ylo = (j == 1) ? mirror3(my) : face3_y(load_cell3(g, c - g.zs));
        const FaceIn3<T> yhi = (j == g.nb_y) ? mirror3(my) : face3_y(load_cell3(g, c + g.zs));
        const Flux3<T> fy1 = face_flux3(ylo, my, g.ph);
        const Flux3<T> fy2 = face_flux3(my, yhi, g.ph);
        const FaceIn3<T> mz = face3_z(P);
        const FaceIn3<T> zlo = (k == 1) ? mirror3(mz) : face3_z(load_cell3(g, c - 1));
        const FaceIn3<T> zhi = (k == g.nb_z) ? mirror3(mz) : face3_z(load_cell3(g, c + 1));
        const Flux3<T> fz1 = face_flux3(zlo, mz, g.ph);
        const Flux3<T> fz2 = face_flux3(mz, zhi, g.ph);
        const Upd3<T> o = update3(ur, uu, uv, uw, uE, fx1, fx2, fy1, fy2, fz1, fz2, g.DtDx, g.DtDy, g.DtDz, g.ph);
        g.rhoE_n[2 * c] = o.r;
        g.rhoE_n[2 * c + 1] = o.E;
        g.uvw_n[3 * c] = o.u;
        g.uvw_n[3 * c + 1] = o.v;
        g.uvw_n[3 * c + 2] = o.w;
        acc.add_cell(o.r, speed3(o.r, o.u, o.v, o.w, o.E, g.ph));
    }
    step_epilogue<128, T>(acc, g.scr, g.partials, gridDim.x * gridDim.y * gridDim.z,
                          blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z), g.ph.C_min, g.Dt_next,
                          g.status, g.seq, 0.0, g.key);
}

// Redo pass (see StepScratch): the exact signal speed of every interior cell.
constexpr int k3RedoNT = 256;
template <class T, bool kF = false> __global__ void __launch_bounds__(k3RedoNT) redo3d(Args3<T> g)
{
    if (*reinterpret_cast<const volatile unsigned *>(&g.scr->redo) == 0u) return;
    StepAcc acc;
    const long long ncol = (long long)g.nb_y * g.nb_z;
    const long long n = (long long)g.nb_x * ncol;
    for (long long q = blockIdx.x * (long long)k3RedoNT + threadIdx.x; q < n; q += (long long)gridDim.x * k3RedoNT) {
        const long long r = q % ncol;
        const long long c = (1 + q / ncol) * g.zy + (1 + r / g.nb_z) * g.zs + 1 + r % g.nb_z;
        acc.add_speed(speed3<T, kF>(g.rhoE_n[2 * c], g.uvw_n[3 * c], g.uvw_n[3 * c + 1], g.uvw_n[3 * c + 2],
                                    g.rhoE_n[2 * c + 1], g.ph));
    }
    redo_epilogue<k3RedoNT, T>(acc.vmax, acc.err, g.scr, gridDim.x, g.ph.C_min, g.Dt_next, g.status, g.key);
}

// ------------------------------------------------------------------- strip kernel ---
// kF: fused arithmetic (hydro_math.cuh). kTma: planes staged by the tensor maps tmr/tmu
// (FP64, even NB_Z), else by per-lane cp.async. W: warps per block. Tile rows with halo:
// W, or W + 1 with kPair (tensor maps, W = 8: warp 0 holds both halo rows).
template <class T, bool kF, bool kTma, int W, bool kPair = false>
__global__ void __launch_bounds__(32 * W, min_blocks3<T>(W))
    strip3d(const __grid_constant__ CUtensorMap tmr, const __grid_constant__ CUtensorMap tmu, Args3<T> g)
{
    static_assert(!kPair || (kTma && W == 8), "the W+1-row tile is built for tensor maps and 8 warps");
    using SM = std::conditional_t<kPair, Smem3P<T>, Smem3<T, W>>;
    constexpr int kRows = kPair ? W + 1 : W;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SM &S = *reinterpret_cast<SM *>(smem_raw);
    if constexpr (kTma) {
        if (threadIdx.x == 0) {
            prefetch_tensormap(&tmr);
            prefetch_tensormap(&tmu);
        }
        march3d_init(S);
    }
    const int i0 = 1 + g.chunk * (int)blockIdx.z;
    const March3 geo{k3TZ * (int)blockIdx.x, (kRows - 2) * (int)blockIdx.y, i0, min(i0 + g.chunk - 1, g.nb_x),
                     g.nb_x, g.nb_y, g.nb_z, g.zs, g.zy, g.xwrap};
    StepAcc acc;
    const float tlof = __double2float_rd(skip_threshold(g.scr, g.key));
    const float tlo2 = skip_tlo2(tlof), ggm1 = g.ggm1;
    const Phys<T> ph = g.ph;
    auto sink = [&](const Upd3<T> &o) {
        acc.add_mass(o.r);
        if (!state_below(o, ggm1, tlo2))
            acc.add_speed(speed3<T, kF>(o.r, o.u, o.v, o.w, o.E, ph));
    };
    bool ok;
    if constexpr (kPair)
        ok = march3d<T, kF>(S, g.rhoE_n, g.uvw_n, geo, ph, g.DtDx, g.DtDy, g.DtDz, sink, Tmaps3{&tmr, &tmu});
    else
        ok = march3d<T, kF, kTma, W>(S, g.rhoE, g.uvw, g.rhoE_n, g.uvw_n, geo, ph, g.DtDx, g.DtDy, g.DtDz, sink,
                                     Tmaps3{&tmr, &tmu});
    if (!ok) acc.err |= kErrWaitTimeout;
    step_epilogue<32 * W, T>(acc, g.scr, g.partials, gridDim.x * gridDim.y * gridDim.z,
                             blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z), g.ph.C_min, g.Dt_next,
                             g.status, g.seq, (double)tlof, g.key);
}

// Tile heights (rows with halo) the plain 3D step is built for: FP64 8, 9 (8 warps, warp 0
// holding both halo rows; tensor-map staging only), 12 and 16; FP32 8 and 16. The
// tensor-map staging is built for FP64 only.
template <class T> constexpr bool tile3_built(int rows)
{
    return sizeof(T) == 8 ? (rows == 8 || rows == 9 || rows == 12 || rows == 16) : (rows == 8 || rows == 16);
}
// The built-in tile height: 9 rows where tensor maps stage the planes (FP64: 37.2 against
// 35.3 GCell/s strict at 512^3 for 8 rows), else 8.
template <class T> int default_rows3(bool tma) { return (sizeof(T) == 8 && tma) ? 9 : k3Warps<T>; }

template <class T, int W, bool kPair = false>
cudaError_t launch_strip3d(bool fused, bool tma, dim3 grid, cudaStream_t stream, const CUtensorMap &tmr,
                           const CUtensorMap &tmu, const Args3<T> &g)
{
    void (*kern)(const CUtensorMap, const CUtensorMap, Args3<T>);
    int smem;
    if constexpr (kPair) {
        kern = fused ? strip3d<T, true, true, W, true> : strip3d<T, false, true, W, true>;
        smem = (int)sizeof(Smem3P<T>);
    } else {
        if constexpr (sizeof(T) == 8)
            kern = fused ? (tma ? strip3d<T, true, true, W> : strip3d<T, true, false, W>)
                         : (tma ? strip3d<T, false, true, W> : strip3d<T, false, false, W>);
        else
            kern = fused ? strip3d<T, true, false, W> : strip3d<T, false, false, W>;
        smem = (int)sizeof(Smem3<T, W>);
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, 32 * W, smem, stream>>>(tmr, tmu, g);
    return cudaGetLastError();
}

// ------------------------------------------------------------- initial condition ---
// hydro3d/main.cxx:296-363. The local Dt of a uniform state at rest, C_min/(c_s + |u|),
// with the reference's per-cell operations, as the bits of a double.
template <class T>
__device__ __forceinline__ unsigned long long rest_dt_bits3(T ur, T uE, T C_min, T gamma, T gm1)
{
    using A = Ar<T>;
    const T inv = A::rcp(ur);
    const T q = A::mul(T(0), inv);
    const T temp = A::add(A::add(A::mul(q, q), A::mul(q, q)), A::mul(q, q));
    const T e_int = A::sub(A::mul(uE, inv), A::mul(A::half, temp));
    const T qp = A::mul(A::mul(gm1, ur), e_int);
    const T cs = A::sqrt(A::mul(A::mul(gamma, qp), inv));
    const T un = A::sqrt(temp);
    return (unsigned long long)__double_as_longlong((double)A::div(C_min, A::add(cs, un)));
}

// The sphere splits the cells into two uniform states: their energy p/(gamma-1) and
// local Dt are evaluated once per thread for the states its cells hold (the same
// operations on the same operands, so the same bits); per cell only the distance test
// and the stores remain. Each thread covers the planes i = 1 + blockIdx.z + m * gridDim.z
// of its column (j, k).
template <class T>
__global__ void init3d_kernel(T *rhoE, T *uvw, int nb_x, int nb_y, int nb_z, long long zs, long long zy, double cx,
                              double cy, double cz, double radius, T u_in, T u_out, T p_in, T p_out, T C_min,
                              T gamma, T gm1, unsigned long long *min_bits)
{
    using A = Ar<T>;
    const int k = 1 + blockIdx.x * 32 + threadIdx.x;
    const int j = 1 + blockIdx.y * 4 + threadIdx.y;
    const T E_in = A::div(p_in, gm1), E_out = A::div(p_out, gm1);
    bool any_in = false, any_out = false;
    if (k <= nb_z && j <= nb_y) {
        const double dy = __dsub_rn((double)j, cy), dz = __dsub_rn((double)k, cz);
        const double dy2 = __dmul_rn(dy, dy), dz2 = __dmul_rn(dz, dz);
        for (int i = 1 + blockIdx.z; i <= nb_x; i += gridDim.z) {
            const double dx = __dsub_rn((double)i, cx);
            const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), dy2), dz2));
            const bool in = d <= radius;
            const long long c = (long long)i * zy + (long long)j * zs + k;
            rhoE[2 * c] = in ? u_in : u_out;
            rhoE[2 * c + 1] = in ? E_in : E_out;
            uvw[3 * c] = T(0);
            uvw[3 * c + 1] = T(0);
            uvw[3 * c + 2] = T(0);
            any_in |= in;
            any_out |= !in;
        }
    }
    unsigned long long best = ~0ull;
    if (any_in) best = rest_dt_bits3(u_in, E_in, C_min, gamma, gm1);
    if (any_out) {
        const unsigned long long b = rest_dt_bits3(u_out, E_out, C_min, gamma, gm1);
        best = b < best ? b : best;
    }
    const int tl = threadIdx.x + 32 * threadIdx.y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(0xffffffffu, best, o);
        best = ob < best ? ob : best;
    }
    if ((tl & 31) == 0 && best != ~0ull) atomicMin(min_bits, best);
}

// ----------------------------------------------------------------- host drivers ---
namespace {
template <class T> CUtensorMapDataType tmap_type3();
template <> CUtensorMapDataType tmap_type3<double>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT64; }
template <> CUtensorMapDataType tmap_type3<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) % 16) == 0; }
} // namespace

template <class T>
int step3d(const T *rhoE, const T *uvw, T *rhoE_next, T *uvw_next, T *Dt_next, const Phys<T> &ph, size_t nb_x,
           size_t nb_y, size_t nb_z, T DtDx, T DtDy, T DtDz, cudaStream_t stream, Kernel which, bool sync,
           StepInfo *info, bool xwrap, bool fused)
{
    if (!rhoE || !uvw || !rhoE_next || !uvw_next || !Dt_next) {
        set_error(kErrArg, "step3d: null pointer argument");
        return kErrArg;
    }
    if (nb_x > (1u << 30) || nb_y > (1u << 30) || nb_z > (1u << 30) ||
        (double)(nb_x + 2) * (nb_y + 2) * (nb_z + 2) > 1.0e12) {
        set_error(kErrArg, "step3d: grid %zu x %zu x %zu too large", nb_x, nb_y, nb_z);
        return kErrArg;
    }
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    if (nb_x == 0 || nb_y == 0 || nb_z == 0) {
        const T dt = div_zero(ph.C_min);
        cudaError_t e = cudaMemcpyAsync(Dt_next, &dt, sizeof(T), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            set_error(kErrCuda, "step3d: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        if (info) *info = StepInfo{};
        return kOk;
    }
    if (ctx->dirty) {
        cudaMemsetAsync(ctx->scr, 0, sizeof(StepScratch), stream);
        ctx->dirty = false;
    }
    Args3<T> g;
    g.rhoE = rhoE; g.uvw = uvw; g.rhoE_n = rhoE_next; g.uvw_n = uvw_next; g.Dt_next = Dt_next;
    g.ph = ph; g.DtDx = DtDx; g.DtDy = DtDy; g.DtDz = DtDz;
    g.nb_x = (int)nb_x; g.nb_y = (int)nb_y; g.nb_z = (int)nb_z;
    g.zs = (long long)nb_z + 2; g.zy = (long long)(nb_y + 2) * g.zs;
    g.scr = ctx->scr; g.status = ctx->status_d; g.seq = ++ctx->seq;
    g.key = problem_key(Dt_next, nb_x, nb_y, nb_z, sizeof(T), ph);
    g.ggm1 = skip_ggm1(ph.gamma, ph.gm1);
    g.xwrap = xwrap ? 1 : 0;

    const bool use_strip = which != Kernel::Direct;
    unsigned nblocks;
    if (use_strip) {
        // tile height and planes per block: the tuned shape when one is set
        // (hydro_set_launch_shape), else the built-in one
        const LaunchShape shape = launch_shape(3, sizeof(T));
        // planes by tensor maps where the rows of both arrays are 16-byte pitched (FP64
        // with even NB_Z; the tile's kbase is a multiple of 30, so even) and the arrays
        // 16-byte aligned; by per-lane copies otherwise
        bool tma = sizeof(T) == 8 && (nb_z + 2) % 2 == 0 && aligned16(rhoE) && aligned16(uvw);
        // tile rows with halo; the 9-row tile needs the tensor maps (else 8 rows)
        int rows = (shape.warps > 0 && tile3_built<T>(shape.warps)) ? shape.warps : default_rows3<T>(tma);
        if (rows == 9 && !tma) rows = 8;
        const int W = rows == 9 ? 8 : rows; // warps per block
        const int nz = (int)((nb_z + k3TZ - 1) / k3TZ), ny = (int)((nb_y + (rows - 2) - 1) / (rows - 2));
        if (ny > 65535) {
            set_error(kErrArg, "step3d: NB_Y %zu too large for the strip kernel", nb_y);
            return kErrArg;
        }
        // planes per block: sized for about 8 waves of resident blocks, at least 8 and at
        // most the cap (the tuned value when one is set, else 256)
        const int cap = shape.chunk > 0 ? shape.chunk : 256;
        const int target = device_sms() * min_blocks3<T>(W) * 8;
        int nchunks = std::max(1, (target + nz * ny - 1) / (nz * ny));
        int chunk = (int)((nb_x + nchunks - 1) / nchunks);
        chunk = std::min(cap, std::max(std::min(8, cap), chunk));
        nchunks = (int)((nb_x + chunk - 1) / chunk);
        if (nchunks > 65535) {
            chunk = (int)((nb_x + 65534) / 65535);
            nchunks = (int)((nb_x + chunk - 1) / chunk);
        }
        g.chunk = chunk;
        nblocks = (unsigned)nz * ny * nchunks;
        if ((err = ctx_reserve(ctx, nblocks)) != kOk) return err;
        g.partials = ctx->partials;
        CUtensorMap tmr, tmu;
        std::memset(&tmr, 0, sizeof tmr);
        std::memset(&tmu, 0, sizeof tmu);
        if (tma) {
            const uint64_t zs = nb_z + 2, ys = nb_y + 2, xs = nb_x + 2;
            tma = encode_tmap_3d(&tmr, tmap_type3<T>(), rhoE, 2 * zs, ys, xs, 2 * zs * sizeof(T), 2 * zs * ys * sizeof(T),
                                 64, (uint32_t)rows, 1) &&
                  encode_tmap_3d(&tmu, tmap_type3<T>(), uvw, 3 * zs, ys, xs, 3 * zs * sizeof(T), 3 * zs * ys * sizeof(T),
                                 96, (uint32_t)rows, 1);
            if (!tma && rows == 9) {
                set_error(kErrCuda, "step3d: tensor maps of the 9-row tile rejected");
                return kErrCuda;
            }
        }
        const dim3 grid(nz, ny, nchunks);
        cudaError_t ea;
        if (rows == 9) {
            if constexpr (sizeof(T) == 8)
                ea = launch_strip3d<T, 8, true>(fused, true, grid, stream, tmr, tmu, g);
            else
                ea = cudaErrorInvalidValue;
        } else if (W == 8) {
            ea = launch_strip3d<T, 8>(fused, tma, grid, stream, tmr, tmu, g);
        } else if constexpr (sizeof(T) == 8) {
            if (W == 12)
                ea = launch_strip3d<T, 12>(fused, tma, grid, stream, tmr, tmu, g);
            else
                ea = launch_strip3d<T, 16>(fused, tma, grid, stream, tmr, tmu, g);
        } else {
            ea = launch_strip3d<T, 16>(fused, tma, grid, stream, tmr, tmu, g);
        }
        if (ea != cudaSuccess) {
            ctx->dirty = true;
            set_error(kErrCuda, "step3d launch: %s", cudaGetErrorString(ea));
            return kErrCuda;
        }
        ctx->last_warps = rows;
        ctx->last_chunk = chunk;
        ctx->last_blocks = min_blocks3<T>(W);
        ctx->last_tma = tma;
    } else {
        const int gx = (int)((nb_z + 31) / 32), gy = (int)((nb_y + 3) / 4), gz = (int)std::min<size_t>(nb_x, 65535);
        if (gy > 65535) {
            set_error(kErrArg, "step3d: NB_Y %zu too large", nb_y);
            return kErrArg;
        }
        nblocks = (unsigned)gx * gy * gz;
        if ((err = ctx_reserve(ctx, nblocks)) != kOk) return err;
        g.partials = ctx->partials;
        g.chunk = 0;
        direct3d<T><<<dim3(gx, gy, gz), dim3(32, 4), 0, stream>>>(g);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx->dirty = true;
        set_error(kErrCuda, "step3d launch: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    ctx->last_kernel = (int)(use_strip ? Kernel::Strip : Kernel::Direct);
    const unsigned redo_blocks = (unsigned)device_sms() * 4;
    // the redo pass recomputes the signal speed in the arithmetic of the step that ran
    // (the direct kernel is always strict)
    const bool fused_ran = fused && use_strip;
    auto redo = [&]() {
        if (fused_ran)
            redo3d<T, true><<<redo_blocks, k3RedoNT, 0, stream>>>(g);
        else
            redo3d<T, false><<<redo_blocks, k3RedoNT, 0, stream>>>(g);
    };
    if (!sync) {
        // enqueued unconditionally; returns at once unless the step asked for it
        redo();
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            ctx->dirty = true;
            set_error(kErrCuda, "step3d launch: %s", cudaGetErrorString(e));
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
        set_error(kErrCuda, "step3d: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    const StepStatus st = read_status(ctx->status_h);
    if (info) {
        info->mass = st.mass + st.mass_comp;
        info->max_speed = st.max_speed;
        info->err = st.err;
        info->kernel = (int)(use_strip ? Kernel::Strip : Kernel::Direct);
    }
    if (st.err & kErrNonPhysical) {
        set_error(kErrPhys, "step3d: non-physical state (rho <= 0 or non-finite signal speed)");
        return kErrPhys;
    }
    return kOk;
}

template <class T>
int init3d_at(T *rhoE, T *uvw, size_t nb_x, size_t nb_y, size_t nb_z, double cx, double cy, double cz, double radius,
              T u_in, T u_out, T p_in, T p_out, T C_min, T gamma, T *min_dt, cudaStream_t stream,
              unsigned long long *bits)
{
    if (!rhoE || !uvw || !min_dt || !bits || nb_x == 0 || nb_y == 0 || nb_z == 0 || nb_x > (1u << 30) ||
        (nb_y + 3) / 4 > 65535) {
        set_error(kErrArg, "init3d: invalid argument");
        return kErrArg;
    }
    const T big = T(1e20);
    const unsigned long long init = (unsigned long long)__builtin_bit_cast(long long, (double)big);
    const T gm1 = gamma - T(1);
    cudaError_t e = cudaMemcpyAsync(bits, &init, sizeof init, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        const long long zs = (long long)nb_z + 2, zy = (long long)(nb_y + 2) * zs;
        // 16 blocks of 128 threads per SM; each thread takes nb_x / gz planes of its column
        const size_t gxy = ((nb_z + 31) / 32) * ((nb_y + 3) / 4);
        const size_t gz = std::max<size_t>(1, std::min<size_t>({nb_x, 65535, (size_t)device_sms() * 16 / std::min<size_t>(gxy, (size_t)device_sms() * 16)}));
        dim3 grid((unsigned)((nb_z + 31) / 32), (unsigned)((nb_y + 3) / 4), (unsigned)gz);
        init3d_kernel<T><<<grid, dim3(32, 4), 0, stream>>>(rhoE, uvw, (int)nb_x, (int)nb_y, (int)nb_z, zs, zy, cx, cy,
                                                           cz, radius, u_in, u_out, p_in, p_out, C_min, gamma, gm1,
                                                           bits);
        e = cudaGetLastError();
    }
    unsigned long long res = 0;
    const unsigned long long zero = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&res, bits, sizeof res, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bits, &zero, sizeof zero, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "init3d: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    *min_dt = (T)__builtin_bit_cast(double, (long long)res);
    return kOk;
}

template <class T>
int init3d(T *rhoE, T *uvw, size_t nb_x, size_t nb_y, size_t nb_z, T u_in, T u_out, T p_in, T p_out, T C_min,
           T gamma, T *min_dt, cudaStream_t stream)
{
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    // the reference's sphere: centre ((N+1)/2 per axis), radius min(centres)/3
    const double cx = double(nb_x + 1) / 2.0, cy = double(nb_y + 1) / 2.0, cz = double(nb_z + 1) / 2.0;
    const double radius = std::min({cx, cy, cz}) / 3;
    return init3d_at<T>(rhoE, uvw, nb_x, nb_y, nb_z, cx, cy, cz, radius, u_in, u_out, p_in, p_out, C_min, gamma,
                        min_dt, stream, &ctx->scr->max_bits);
}

template int init3d_at<double>(double *, double *, size_t, size_t, size_t, double, double, double, double, double,
                               double, double, double, double, double, double *, cudaStream_t, unsigned long long *);
template int init3d_at<float>(float *, float *, size_t, size_t, size_t, double, double, double, double, float, float,
                              float, float, float, float, float *, cudaStream_t, unsigned long long *);

template int step3d<double>(const double *, const double *, double *, double *, double *, const Phys<double> &,
                            size_t, size_t, size_t, double, double, double, cudaStream_t, Kernel, bool, StepInfo *,
                            bool, bool);
template int step3d<float>(const float *, const float *, float *, float *, float *, const Phys<float> &, size_t,
                           size_t, size_t, float, float, float, cudaStream_t, Kernel, bool, StepInfo *, bool, bool);
template int init3d<double>(double *, double *, size_t, size_t, size_t, double, double, double, double, double,
                            double, double *, cudaStream_t);
template int init3d<float>(float *, float *, size_t, size_t, size_t, float, float, float, float, float, float,
                           float *, cudaStream_t);

} // namespace hydro
