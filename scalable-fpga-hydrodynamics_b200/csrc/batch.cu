// Batched step: many independent 2D or 3D blast instances of uneven sizes advanced by
// one persistent kernel per step, each instance with its own time step, boundaries and
// simulated time (the layered "batching" change of the plain path; no counterpart in the
// reference, whose host loop advances one domain, hydro2d/main.cxx:689-815).
//
// Each instance keeps the plain path's arithmetic: the same strip march
// (strip2d_march.cuh / strip3d_march.cuh), so an instance's state after n batched steps
// is bit-identical to n plain steps in the same precision. 2D instances keep the pair
// layout with rows padded to 16 bytes (TMA-fed); 3D instances keep the reference's
// pair/triple layout (cp.async-fed). Work is a flat list of (instance, tile x chunk)
// items; persistent blocks take items from an atomic counter. Every item writes its max
// signal speed and error bits to its own slot; the item that completes an instance's
// step (ticket per instance) merges that instance's slots -- the result depends neither
// on which block ran which item nor on the other instances in the batch -- and advances
// the instance on the device:
//   Dt = min(1e20, C_min / max_speed)   (hydro2d/kernel.cxx:318, main.cxx:706-781)
//   t += Dt (FP64 accumulator), DtDx = Dt / DX ... (main.cxx:703-704, in T)
//   active while t < t_end and steps < max_steps (main.cxx:689)
// so a step needs no host round trip and n steps are captured as one CUDA graph. The
// graph ends with one pass over the final state that forms each instance's compensated
// FP64 conservation sums (mass, momenta, energy) over the same items, merged per
// instance in a fixed order (the step kernels carry no sums: fewer registers, more
// resident blocks). The signal speed uses the plain path's exact skip (see
// batch_threshold).
#include <algorithm>
#include <stdio.h>
#include <string.h>
#include <vector>

#include "../../include/hydro_b200.h"
#include "hydro_host.h"
#include "strip2d_march.cuh"
#include "strip3d_march.cuh"

namespace hydro {

constexpr int kSums = 5; // rho, rho u, rho v, rho w (0 in 2D), E

template <class T> struct alignas(128) Inst2 {
    CUtensorMap tm[2][2]; // [buffer][0: (rho, E), 1: (rho u, rho v)]
    T *rhoE[2], *uv[2];
    Phys<T> ph;
    T DX, DY, dt, DtDx, DtDy;
    double t, t_end;
    double vmax_prev; // exact max signal speed of the previous step (0 before the first)
    float ggm1;       // gamma * (gamma - 1), for the signal-speed skip test
    long long exact_passes;
    unsigned sum_items; // items of the end-of-run conservation sums done
    long long ys;
    long long steps, max_steps;
    int nb_x, nb_y, nstrips, chunk;
    int parity, active;
    unsigned done_items, err;
};

template <class T> struct alignas(128) Inst3 {
    T *rhoE[2], *uvw[2];
    Phys<T> ph;
    T DX, DY, DZ, dt, DtDx, DtDy, DtDz;
    double t, t_end;
    double vmax_prev; // exact max signal speed of the previous step (0 before the first)
    float ggm1;       // gamma * (gamma - 1), for the signal-speed skip test
    long long exact_passes;
    unsigned sum_items; // items of the end-of-run conservation sums done
    long long zs, zy;
    long long steps, max_steps;
    int nb_x, nb_y, nb_z, ntz, nty, chunk;
    int parity, active;
    unsigned done_items, err;
};

struct ItemPart {
    double s[kSums], c[kSums];
    unsigned long long maxbits;
    unsigned err, pad;
};

// per-slot status, host-mapped, written by the finalising item
struct SlotStatus {
    double t, dt, sums[kSums], max_speed;
    long long steps, exact_passes;
    int active;
    unsigned err;
};

// The end-of-run conservation sums of one item (compensated FP64), merged per instance.
struct BatchAcc {
    double s[kSums] = {0, 0, 0, 0, 0}, c[kSums] = {0, 0, 0, 0, 0};
    double vmax = 0.0;
    unsigned err = 0;

    __device__ __forceinline__ void kahan(int q, double x)
    {
        const double y = __dadd_rn(x, c[q]);
        const double tt = __dadd_rn(s[q], y);
        c[q] = __dsub_rn(y, __dsub_rn(tt, s[q]));
        s[q] = tt;
    }
    // conservation sums of one updated cell (the rho w sum stays 0 in 2D)
    template <int D, class T> __device__ __forceinline__ void add_sums(T r, T mu, T mv, T mw, T E)
    {
        kahan(0, (double)r);
        kahan(1, (double)mu);
        kahan(2, (double)mv);
        if (D == 3) kahan(3, (double)mw);
        kahan(4, (double)E);
        if (!(r > T(0))) err |= kErrNonPhysical;
    }
};

// What a step accumulates per cell: the max exact signal speed and error bits.
struct MaxAcc {
    double vmax = 0.0;
    unsigned err = 0;
    __device__ __forceinline__ void add_speed(double sp)
    {
        vmax = (sp > vmax) ? sp : vmax;
        if (!(sp <= 1.0e300)) err |= kErrNonPhysical;
    }
};

// deterministic merge of (s, c) pairs: the lower lane's value first
__device__ __forceinline__ void merge_pair(double &s, double &c, double s2, double c2, bool upper)
{
    if (upper) {
        double a = s2, b = c2;
        neumaier_merge(a, b, s, c);
        s = a;
        c = b;
    } else {
        neumaier_merge(s, c, s2, c2);
    }
}

// Block-wide reduction of a BatchAcc; the result is valid in thread 0.
template <int NT> __device__ __forceinline__ void block_reduce(BatchAcc &a)
{
    constexpr int NW = NT / 32;
    __shared__ double r_s[NW][kSums], r_c[NW][kSums];
    __shared__ unsigned long long r_m[NW];
    __shared__ unsigned r_e[NW];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    unsigned long long mb = __double_as_longlong(a.vmax);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int q = 0; q < kSums; ++q) {
            const double s2 = __shfl_xor_sync(0xffffffffu, a.s[q], o);
            const double c2 = __shfl_xor_sync(0xffffffffu, a.c[q], o);
            merge_pair(a.s[q], a.c[q], s2, c2, up);
        }
        const unsigned long long om = __shfl_xor_sync(0xffffffffu, mb, o);
        mb = om > mb ? om : mb;
        a.err |= __shfl_xor_sync(0xffffffffu, a.err, o);
    }
    if (lane == 0) {
        for (int q = 0; q < kSums; ++q) {
            r_s[warp][q] = a.s[q];
            r_c[warp][q] = a.c[q];
        }
        r_m[warp] = mb;
        r_e[warp] = a.err;
    }
    __syncthreads();
    if (t == 0) {
        for (int w = 1; w < NW; ++w) {
            for (int q = 0; q < kSums; ++q) neumaier_merge(a.s[q], a.c[q], r_s[w][q], r_c[w][q]);
            mb = r_m[w] > mb ? r_m[w] : mb;
            a.err |= r_e[w];
        }
        a.vmax = __longlong_as_double((long long)mb);
    }
    __syncthreads();
}

// The signal-speed skip of the plain path, per instance: a cell computes its exact
// speed only when its FP32 upper bound reaches kSkipFrac x the previous step's max.
// skip_frac is kSkipFrac unless a caller set another fraction (0 turns the skip off;
// above 1 every cell skips and every step takes the exact pass).
template <class I> __device__ __forceinline__ float batch_threshold(const I *in, double skip_frac)
{
    return __double2float_rd(skip_frac * in->vmax_prev);
}

// Exact max signal speed over an instance's new state (the buffer the step wrote),
// whole block; valid in thread 0. Runs only when every cell skipped the exact speed.
template <int NT> __device__ __forceinline__ double block_max(double v, unsigned &err)
{
    __shared__ unsigned long long s_max[NT / 32];
    const unsigned long long mb = block_max_bits<NT>((unsigned long long)__double_as_longlong(v), s_max);
    if (__syncthreads_or(err != 0)) err = kErrNonPhysical;
    return __longlong_as_double((long long)mb);
}
template <int NT, class T, bool kF> __device__ double exact_max(const Inst2<T> *in, unsigned &err)
{
    const int b = in->parity ^ 1;
    const T *r = in->rhoE[b], *u = in->uv[b];
    const long long ny = in->nb_y, n = (long long)in->nb_x * ny;
    double vmax = 0.0;
    for (long long q = threadIdx.x; q < n; q += NT) {
        const long long c = (1 + q / ny) * in->ys + 1 + q % ny;
        const double sp = (double)speed2<T, kF>(__ldcg(r + 2 * c), __ldcg(u + 2 * c), __ldcg(u + 2 * c + 1),
                                                __ldcg(r + 2 * c + 1), in->ph);
        vmax = (sp > vmax) ? sp : vmax;
        if (!(sp <= 1.0e300)) err = kErrNonPhysical;
    }
    return block_max<NT>(vmax, err);
}
template <int NT, class T, bool kF> __device__ double exact_max(const Inst3<T> *in, unsigned &err)
{
    const int b = in->parity ^ 1;
    const T *r = in->rhoE[b], *u = in->uvw[b];
    const long long ncol = (long long)in->nb_y * in->nb_z, n = (long long)in->nb_x * ncol;
    double vmax = 0.0;
    for (long long q = threadIdx.x; q < n; q += NT) {
        const long long rr = q % ncol;
        const long long c = (1 + q / ncol) * in->zy + (1 + rr / in->nb_z) * in->zs + 1 + rr % in->nb_z;
        const double sp = (double)speed3<T, kF>(__ldcg(r + 2 * c), __ldcg(u + 3 * c), __ldcg(u + 3 * c + 1),
                                                __ldcg(u + 3 * c + 2), __ldcg(r + 2 * c + 1), in->ph);
        vmax = (sp > vmax) ? sp : vmax;
        if (!(sp <= 1.0e300)) err = kErrNonPhysical;
    }
    return block_max<NT>(vmax, err);
}

template <class T> __device__ __forceinline__ void set_dtdz(Inst2<T> *, T) {}
template <class T> __device__ __forceinline__ void set_dtdz(Inst3<T> *in, T Dt) { in->DtDz = Ar<T>::div(Dt, in->DZ); }

// Time-step bookkeeping of one instance after its step (thread 0 of the finalising block).
template <class T, class I> __device__ __forceinline__ void advance(I *in, double vmax, unsigned err, SlotStatus *st)
{
    using A = Ar<T>;
    const T big = T(1e20);
    const T dtn = A::div(in->ph.C_min, static_cast<T>(vmax));
    const T Dt = (dtn < big) ? dtn : big;
    in->steps += 1;
    in->t = __dadd_rn(in->t, (double)Dt);
    in->dt = Dt;
    in->DtDx = A::div(Dt, in->DX);
    in->DtDy = A::div(Dt, in->DY);
    set_dtdz<T>(in, Dt);
    in->parity ^= 1;
    in->vmax_prev = vmax;
    in->err |= err;
    in->active = (in->t < in->t_end) && (in->steps < in->max_steps) && !(in->err & kErrNonPhysical);
    if (st) {
        st->t = in->t;
        st->dt = (double)Dt;
        st->max_speed = vmax;
        st->steps = in->steps;
        st->exact_passes = in->exact_passes;
        st->active = in->active;
        st->err = in->err;
    }
    __threadfence();
    in->done_items = 0;
}

// Block-wide max of a non-negative double and OR of error bits; valid in thread 0.
template <int NT> __device__ __forceinline__ double block_max_err(double v, unsigned &err)
{
    __shared__ unsigned long long s_max[NT / 32];
    __shared__ unsigned s_err;
    if (threadIdx.x == 0) s_err = 0u;
    __syncthreads();
    if (err) atomicOr(&s_err, err);
    const unsigned long long mb = block_max_bits<NT>((unsigned long long)__double_as_longlong(v), s_max);
    err = s_err;
    __syncthreads(); // s_err / s_max free for the next use
    return __longlong_as_double((long long)mb);
}

// Merge an instance's item maxima, take the exact pass if no cell reached the skip
// threshold, and advance the instance (whole block).
template <int NT, class T, bool kF, class I>
__device__ void finalize_step(I *in, const ItemPart *parts, int nitems, SlotStatus *st, double skip_frac)
{
    unsigned long long mb = 0ull;
    unsigned err = 0;
    for (int i = threadIdx.x; i < nitems; i += NT) {
        const unsigned long long m = __ldcg(&parts[i].maxbits);
        mb = m > mb ? m : mb;
        err |= __ldcg(&parts[i].err);
    }
    double vmax = block_max_err<NT>(__longlong_as_double((long long)mb), err);
    // cells whose speed bound was under the threshold skipped the exact speed; if no
    // cell reached the threshold the skipped cells may hold the max: all cells again
    __shared__ int s_redo;
    if (threadIdx.x == 0) s_redo = (vmax < (double)batch_threshold(in, skip_frac)) ? 1 : 0;
    __syncthreads();
    if (s_redo) {
        unsigned e2 = 0;
        const double m = exact_max<NT, T, kF>(in, e2);
        if (threadIdx.x == 0) {
            vmax = m;
            err |= e2;
            in->exact_passes += 1;
        }
    }
    if (threadIdx.x == 0) advance<T>(in, vmax, err, st);
}

// Merge an instance's conservation-sum slots (fixed thread and lane order: the result
// depends only on the instance) and publish them (whole block).
template <int NT, class I>
__device__ void finalize_sums(I *in, const ItemPart *parts, int nitems, SlotStatus *st)
{
    BatchAcc a;
    for (int i = threadIdx.x; i < nitems; i += NT) {
        const ItemPart &p = parts[i];
        for (int q = 0; q < kSums; ++q) neumaier_merge(a.s[q], a.c[q], __ldcg(&p.s[q]), __ldcg(&p.c[q]));
        a.err |= __ldcg(&p.err);
    }
    block_reduce<NT>(a);
    if (threadIdx.x == 0) {
        if (st)
            for (int q = 0; q < kSums; ++q) st->sums[q] = __dadd_rn(a.s[q], a.c[q]);
        __threadfence();
        in->sum_items = 0;
    }
}

// A step item's max and error bits into its slot; returns (in every thread) whether this
// item completed its instance's step.
template <int NT>
__device__ __forceinline__ bool publish_step(const MaxAcc &acc, ItemPart *parts, int w, unsigned *done, int nitems,
                                             int *s_last)
{
    unsigned err = acc.err;
    const double vmax = block_max_err<NT>(acc.vmax, err);
    if (threadIdx.x == 0) {
        ItemPart &p = parts[w];
        p.maxbits = (unsigned long long)__double_as_longlong(vmax);
        p.err = err;
        __threadfence();
        *s_last = (atomicAdd(done, 1u) == (unsigned)nitems - 1u);
    }
    __syncthreads();
    const bool last = *s_last != 0;
    if (last) __threadfence();
    return last;
}

// The item's partial sums into its slot; returns (in every thread) whether this item
// completed its instance's step.
template <int NT>
__device__ __forceinline__ bool publish_item(BatchAcc &acc, ItemPart *parts, int w, unsigned *done, int nitems,
                                             int *s_last)
{
    block_reduce<NT>(acc);
    if (threadIdx.x == 0) {
        ItemPart &p = parts[w];
        for (int q = 0; q < kSums; ++q) {
            p.s[q] = acc.s[q];
            p.c[q] = acc.c[q];
        }
        p.maxbits = (unsigned long long)__double_as_longlong(acc.vmax);
        p.err = acc.err;
        __threadfence();
        *s_last = (atomicAdd(done, 1u) == (unsigned)nitems - 1u);
    }
    __syncthreads();
    const bool last = *s_last != 0;
    if (last) __threadfence();
    return last;
}

// resident blocks per SM the register budget of the 2D step aims at
template <class T> struct Batch2dOcc { static constexpr int value = sizeof(T) == 4 ? 6 : 4; };

// kF: fused arithmetic (hydro_math.cuh)
template <class T, bool kF>
__global__ void __launch_bounds__(kStripNT, Batch2dOcc<T>::value) batch2d(Inst2<T> *insts, const int2 *items, const int2 *ranges,
                                                      int nitems, unsigned *counter, ItemPart *parts,
                                                      SlotStatus *status, double skip_frac)
{
    __shared__ Smem2<T> S;
    __shared__ int s_item;
    __shared__ int s_last;
    march2d_init(S);
    unsigned ld = 0;
    for (;;) {
        __syncthreads(); // everyone has read s_item / finished the previous item
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int w = s_item;
        if (w >= nitems) break;
        const int2 it = items[w];
        Inst2<T> *I = insts + it.x;
        if (!I->active) continue;
        const int par = I->parity;
        const int strip = it.y % I->nstrips, ck = it.y / I->nstrips;
        const int i0 = 1 + ck * I->chunk;
        const March2 geo{kStripW * strip, i0, min(i0 + I->chunk - 1, I->nb_x), I->nb_x, I->nb_y, I->ys, 1};
        const Phys<T> ph = I->ph;
        if (threadIdx.x == 0) {
            prefetch_tensormap(&I->tm[par][0]);
            prefetch_tensormap(&I->tm[par][1]);
        }
        MaxAcc acc;
        const float tlo2 = skip_tlo2(batch_threshold(I, skip_frac)), ggm1 = I->ggm1;
        const bool ok = march2d<T, true, kF>(S, &I->tm[par][0], &I->tm[par][1], geo, I->rhoE[par ^ 1], I->uv[par ^ 1], ph,
                                   I->DtDx, I->DtDy, ld, [&](const Upd2<T> &o) {
                                       if (!(o.r > T(0))) acc.err |= kErrNonPhysical;
                                       if (!state_below(o, ggm1, tlo2))
                                           acc.add_speed((double)speed2<T, kF>(o.r, o.u, o.v, o.E, ph));
                                   });
        if (!ok) acc.err |= kErrWaitTimeout;
        const int2 rg = ranges[it.x];
        if (publish_step<kStripNT>(acc, parts, w, &I->done_items, rg.y, &s_last))
            finalize_step<kStripNT, T, kF>(I, parts + rg.x, rg.y, status ? status + it.x : nullptr, skip_frac);
    }
}

template <class T, bool kF>
__global__ void __launch_bounds__(k3NT<T>, k3MinBlocks<T>) batch3d(Inst3<T> *insts, const int2 *items, const int2 *ranges,
                                                  int nitems, unsigned *counter, ItemPart *parts,
                                                  SlotStatus *status, double skip_frac)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem3<T> &S = *reinterpret_cast<Smem3<T> *>(smem_raw);
    __shared__ int s_item;
    __shared__ int s_last;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int w = s_item;
        if (w >= nitems) break;
        const int2 it = items[w];
        Inst3<T> *I = insts + it.x;
        if (!I->active) continue;
        const int par = I->parity;
        const int tz = it.y % I->ntz, rem = it.y / I->ntz;
        const int ty = rem % I->nty, ck = rem / I->nty;
        const int i0 = 1 + ck * I->chunk;
        const March3 geo{k3TZ * tz, k3TY<T> * ty, i0, min(i0 + I->chunk - 1, I->nb_x), I->nb_x, I->nb_y, I->nb_z,
                         I->zs, I->zy, 1};
        const Phys<T> ph = I->ph;
        MaxAcc acc;
        const float tlo2 = skip_tlo2(batch_threshold(I, skip_frac)), ggm1 = I->ggm1;
        march3d<T, kF, false, k3Warps<T>, false>(
            S, I->rhoE[par], I->uvw[par], I->rhoE[par ^ 1], I->uvw[par ^ 1], geo, ph, I->DtDx, I->DtDy, I->DtDz,
            [&](const Upd3<T> &o) {
                if (!(o.r > T(0))) acc.err |= kErrNonPhysical;
                if (!state_below(o, ggm1, tlo2))
                    acc.add_speed((double)speed3<T, kF>(o.r, o.u, o.v, o.w, o.E, ph));
            });
        const int2 rg = ranges[it.x];
        if (publish_step<k3NT<T>>(acc, parts, w, &I->done_items, rg.y, &s_last))
            finalize_step<k3NT<T>, T, kF>(I, parts + rg.x, rg.y, status ? status + it.x : nullptr, skip_frac);
    }
}

// End-of-run conservation sums (compensated FP64 mass, momenta, energy) of every instance
// over the same work items: one pass over the current state after the run's last step.
template <int NT, class T> __device__ __forceinline__ void sum_item(const Inst2<T> *I, int y, BatchAcc &acc)
{
    using V2 = typename Vec2<T>::type;
    const int strip = y % I->nstrips, ck = y / I->nstrips;
    const int t = threadIdx.x, j = kStripW * strip + t;
    if (t < 1 || t > kStripW || j > I->nb_y) return;
    const int i0 = 1 + ck * I->chunk, i1 = min(i0 + I->chunk - 1, I->nb_x);
    const V2 *r = reinterpret_cast<const V2 *>(I->rhoE[I->parity]);
    const V2 *u = reinterpret_cast<const V2 *>(I->uv[I->parity]);
    for (int i = i0; i <= i1; ++i) {
        const long long c = (long long)i * I->ys + j;
        const V2 a = r[c], b = u[c];
        acc.add_sums<2>(a.x, b.x, b.y, T(0), a.y);
    }
}
template <int NT, class T> __device__ __forceinline__ void sum_item(const Inst3<T> *I, int y, BatchAcc &acc)
{
    const int tz = y % I->ntz, rem = y / I->ntz;
    const int ty = rem % I->nty, ck = rem / I->nty;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k = k3TZ * tz + lane, j = k3TY<T> * ty + w;
    if (w < 1 || w > k3TY<T> || lane < 1 || lane > k3TZ || j > I->nb_y || k > I->nb_z) return;
    const int i0 = 1 + ck * I->chunk, i1 = min(i0 + I->chunk - 1, I->nb_x);
    const T *r = I->rhoE[I->parity], *u = I->uvw[I->parity];
    for (int i = i0; i <= i1; ++i) {
        const long long c = (long long)i * I->zy + (long long)j * I->zs + k;
        acc.add_sums<3>(r[2 * c], u[3 * c], u[3 * c + 1], u[3 * c + 2], r[2 * c + 1]);
    }
}

template <int NT, class T, class I>
__global__ void __launch_bounds__(NT) batch_sums(I *insts, const int2 *items, const int2 *ranges, int nitems,
                                                 unsigned *counter, ItemPart *parts, SlotStatus *status)
{
    __shared__ int s_item;
    __shared__ int s_last;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int w = s_item;
        if (w >= nitems) break;
        const int2 it = items[w];
        I *in = insts + it.x;
        BatchAcc acc;
        sum_item<NT, T>(in, it.y, acc);
        const int2 rg = ranges[it.x];
        if (publish_item<NT>(acc, parts, w, &in->sum_items, rg.y, &s_last))
            finalize_sums<NT>(in, parts + rg.x, rg.y, status ? status + it.x : nullptr);
    }
}

// ----------------------------------------------------------------------- host engine ---
class BatchBase {
  public:
    virtual ~BatchBase() = default;
    virtual int add(const hydro_blast_t &spec) = 0;
    virtual int remove(int slot) = 0;
    virtual int run(int nsteps, bool sync) = 0;
    virtual int status(int slot, hydro_batch_status_t *out) = 0;
    virtual int state(int slot, const void **rhoE, const void **uvx, long long *row_stride) = 0;
    virtual size_t bytes(const hydro_blast_t &spec) const = 0;
    virtual int copy_state(int slot, void *rhoE, void *uvx, bool to_host) = 0;
    virtual int sync() = 0;
    virtual int prepare(int nsteps) = 0;
    virtual int set_skip_fraction(double f) = 0;
    virtual int set_arith(bool fused) = 0;
};

template <class T, int D> class BatchEngine final : public BatchBase {
    using Inst = typename std::conditional<D == 2, Inst2<T>, Inst3<T>>::type;

  public:
    BatchEngine(int chunk, int capacity, cudaStream_t stream, int *rc)
        : chunk_(chunk > 0 ? chunk : (D == 2 ? 32 : 64)), cap_(capacity)
    {
        own_stream_ = (stream == nullptr);
        cudaError_t e = cudaSuccess;
        if (own_stream_) e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
        else stream_ = stream;
        if (e == cudaSuccess) e = cudaMalloc(&insts_, sizeof(Inst) * cap_);
        if (e == cudaSuccess) e = cudaMalloc(&ranges_, sizeof(int2) * cap_);
        if (e == cudaSuccess) e = cudaMalloc(&counter_, 64);
        if (e == cudaSuccess) e = cudaMalloc(&scratch_bits_, 64);
        if (e == cudaSuccess) e = cudaMemset(scratch_bits_, 0, 64);
        if (e == cudaSuccess) e = cudaHostAlloc(&status_h_, sizeof(SlotStatus) * cap_, cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaHostGetDevicePointer(&status_d_, status_h_, 0);
        if (e == cudaSuccess) memset(status_h_, 0, sizeof(SlotStatus) * cap_);
        int dev = 0, nsm = 1, occ = 1;
        if (e == cudaSuccess) e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        // persistent grid: the resident blocks of the step kernel (the smaller of the
        // strict and fused variants' occupancy)
        int occ_f = 1;
        if constexpr (D == 2) {
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch2d<T, false>, kStripNT, 0);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, batch2d<T, true>, kStripNT, 0);
        } else {
            smem_ = (int)sizeof(Smem3<T>);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(batch3d<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(batch3d<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch3d<T, false>, k3NT<T>, smem_);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, batch3d<T, true>, k3NT<T>, smem_);
        }
        blocks_ = nsm * std::max(1, std::min(occ, occ_f));
        int occ_s = 0;
        if (e == cudaSuccess) {
            if constexpr (D == 2)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, batch_sums<kStripNT, T, Inst>, kStripNT, 0);
            else
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, batch_sums<k3NT<T>, T, Inst>, k3NT<T>, 0);
        }
        sum_blocks_ = nsm * std::max(1, occ_s);
        slots_.resize(cap_);
        host_ranges_.assign(cap_, make_int2(0, 0));
        *rc = (e == cudaSuccess) ? kOk : kErrCuda;
        if (e != cudaSuccess) set_error(kErrCuda, "batch create: %s", cudaGetErrorString(e));
    }

    ~BatchEngine() override
    {
        if (graph_) cudaGraphExecDestroy(graph_);
        for (auto &s : slots_)
            if (s.used) free_slot(s);
        cudaStreamSynchronize(stream_);
        cudaFree(insts_);
        cudaFree(ranges_);
        cudaFree(counter_);
        cudaFree(scratch_bits_);
        cudaFree(items_);
        cudaFree(parts_);
        cudaFreeHost(status_h_);
        if (own_stream_) cudaStreamDestroy(stream_);
    }

    // 2D rows are padded to a 16-byte multiple (one spare cell for odd NB_Y in FP32) so
    // that every instance can be fed by TMA; 3D keeps the reference strides.
    static size_t row_stride(size_t nb_y)
    {
        const size_t per = 16 / (2 * sizeof(T)); // cells per 16 bytes of one pair array
        return (nb_y + 2 + per - 1) / per * per;
    }

    size_t bytes(const hydro_blast_t &s) const override
    {
        if constexpr (D == 2) return 2 * 4 * sizeof(T) * (s.nb[0] + 2) * row_stride(s.nb[1]);
        else return 2 * 5 * sizeof(T) * (s.nb[0] + 2) * (s.nb[1] + 2) * (s.nb[2] + 2);
    }

    int add(const hydro_blast_t &s) override
    {
        const size_t nb_x = s.nb[0], nb_y = s.nb[1], nb_z = (D == 3) ? s.nb[2] : 0;
        const size_t lim = D == 2 ? (1u << 24) : (1u << 14);
        if (nb_x == 0 || nb_y == 0 || nb_x > lim || nb_y > lim || (D == 3 && (nb_z == 0 || nb_z > lim)) ||
            !(s.gamma > 1.0)) {
            set_error(kErrArg, "batch add: invalid %dD blast (grid %zu x %zu x %zu, gamma %g)", D, nb_x, nb_y, nb_z,
                      s.gamma);
            return kErrArg;
        }
        int slot = -1;
        for (int i = 0; i < cap_; ++i)
            if (!slots_[i].used) {
                slot = i;
                break;
            }
        if (slot < 0) {
            set_error(kErrArg, "batch add: all %d slots are in use", cap_);
            return kErrArg;
        }
        Slot &sl = slots_[slot];
        const size_t ys = (D == 2) ? row_stride(nb_y) : nb_y + 2;
        const size_t ncell = (D == 2) ? ys * (nb_x + 2) : (nb_x + 2) * (nb_y + 2) * (nb_z + 2);
        const size_t nv = (D == 2) ? 2 : 3;
        cudaError_t e = cudaSuccess;
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            e = cudaMallocAsync(&sl.rhoE[b], 2 * ncell * sizeof(T), stream_);
            if (e == cudaSuccess) e = cudaMallocAsync(&sl.uvx[b], nv * ncell * sizeof(T), stream_);
            if (e == cudaSuccess) e = cudaMemsetAsync(sl.rhoE[b], 0, 2 * ncell * sizeof(T), stream_);
            if (e == cudaSuccess) e = cudaMemsetAsync(sl.uvx[b], 0, nv * ncell * sizeof(T), stream_);
        }
        if (e != cudaSuccess) {
            set_error(kErrCuda, "batch add: allocation of %zu bytes failed: %s", bytes(s), cudaGetErrorString(e));
            free_slot(sl);
            return kErrCuda;
        }
        Inst I;
        memset(&I, 0, sizeof I);
        const T one = T(1);
        I.DX = one / T(nb_x + 1);
        I.DY = one / T(nb_y + 1);
        T ms = (I.DY < I.DX) ? I.DY : I.DX; // std::min({DX, DY[, DZ]}) (main.cxx:484)
        if constexpr (D == 3) {
            I.DZ = one / T(nb_z + 1);
            ms = (I.DZ < ms) ? I.DZ : ms;
        }
        {
            const T gamma = T(s.gamma), gm1 = T(gamma - one);
            I.ph = Phys<T>::make(T(T(s.C) * ms), gamma, gm1, T(one / gm1), T(s.K));
        }
        I.ggm1 = skip_ggm1(I.ph.gamma, I.ph.gm1);
        T first = 0;
        int rc;
        if constexpr (D == 2)
            rc = init2d_at<T>(sl.rhoE[0], sl.uvx[0], nb_x, nb_y, s.centre[0], s.centre[1], s.radius, T(s.rho_in),
                              T(s.rho_out), T(s.p_in), T(s.p_out), I.ph.C_min, I.ph.gamma, &first, stream_,
                              scratch_bits_, (long long)ys);
        else
            rc = init3d_at<T>(sl.rhoE[0], sl.uvx[0], nb_x, nb_y, nb_z, s.centre[0], s.centre[1], s.centre[2],
                              s.radius, T(s.rho_in), T(s.rho_out), T(s.p_in), T(s.p_out), I.ph.C_min, I.ph.gamma,
                              &first, stream_, scratch_bits_);
        if (rc != kOk) {
            free_slot(sl);
            return rc;
        }
        const T big = T(1e20);
        I.dt = (first < big) ? first : big; // first_Dt = min(1e20, IC min), main.cxx:618-660
        I.DtDx = I.dt / I.DX;
        I.DtDy = I.dt / I.DY;
        I.t = 0.0;
        I.t_end = s.t_end;
        I.max_steps = s.max_steps;
        I.steps = 0;
        I.nb_x = (int)nb_x;
        I.nb_y = (int)nb_y;
        I.chunk = chunk_;
        I.parity = 0;
        I.active = (0.0 < s.t_end) && (0 < s.max_steps);
        int nitems;
        if constexpr (D == 2) {
            I.ys = (long long)ys;
            I.nstrips = (int)((nb_y + kStripW - 1) / kStripW);
            const size_t rowbytes = 2 * sizeof(T) * ys;
            const CUtensorMapDataType dt =
                sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
            for (int b = 0; b < 2; ++b) {
                I.rhoE[b] = sl.rhoE[b];
                I.uv[b] = sl.uvx[b];
                if (!encode_tmap_2d(&I.tm[b][0], dt, sl.rhoE[b], 2 * (nb_y + 2), nb_x + 2, rowbytes, 2 * kStripNT, 1) ||
                    !encode_tmap_2d(&I.tm[b][1], dt, sl.uvx[b], 2 * (nb_y + 2), nb_x + 2, rowbytes, 2 * kStripNT, 1)) {
                    free_slot(sl);
                    set_error(kErrCuda, "batch add: tensor map encoding failed");
                    return kErrCuda;
                }
            }
            nitems = I.nstrips * (int)((nb_x + chunk_ - 1) / chunk_);
        } else {
            I.DtDz = I.dt / I.DZ;
            I.nb_z = (int)nb_z;
            I.zs = (long long)nb_z + 2;
            I.zy = (long long)(nb_y + 2) * I.zs;
            I.ntz = (int)((nb_z + k3TZ - 1) / k3TZ);
            I.nty = (int)((nb_y + k3TY<T> - 1) / k3TY<T>);
            for (int b = 0; b < 2; ++b) {
                I.rhoE[b] = sl.rhoE[b];
                I.uvw[b] = sl.uvx[b];
            }
            nitems = I.ntz * I.nty * (int)((nb_x + chunk_ - 1) / chunk_);
        }
        e = cudaMemcpyAsync(insts_ + slot, &I, sizeof I, cudaMemcpyHostToDevice, stream_);
        SlotStatus st0{};
        st0.dt = (double)I.dt;
        st0.active = I.active;
        status_h_[slot] = st0;
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) {
            free_slot(sl);
            set_error(kErrCuda, "batch add: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        sl.used = true;
        sl.nitems = nitems;
        sl.ys = ys;
        sl.nb[0] = nb_x;
        sl.nb[1] = nb_y;
        sl.nb[2] = nb_z;
        dirty_ = true;
        return slot;
    }

    int remove(int slot) override
    {
        if (slot < 0 || slot >= cap_ || !slots_[slot].used) {
            set_error(kErrArg, "batch remove: no instance in slot %d", slot);
            return kErrArg;
        }
        cudaError_t e = cudaStreamSynchronize(stream_);
        free_slot(slots_[slot]);
        dirty_ = true;
        if (e != cudaSuccess) {
            set_error(kErrCuda, "batch remove: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        return kOk;
    }

    int run(int nsteps, bool sync) override
    {
        if (nsteps < 0) {
            set_error(kErrArg, "batch run: negative step count");
            return kErrArg;
        }
        int rc = kOk;
        if (dirty_ || nsteps != graph_steps_) rc = rebuild(nsteps);
        if (rc != kOk) return rc;
        cudaError_t e = cudaSuccess;
        if (nitems_ > 0 && nsteps > 0) e = cudaGraphLaunch(graph_, stream_);
        if (e == cudaSuccess && sync) e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) {
            set_error(kErrCuda, "batch run: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        return kOk;
    }

    int status(int slot, hydro_batch_status_t *out) override
    {
        if (slot < 0 || slot >= cap_ || !slots_[slot].used || !out) {
            set_error(kErrArg, "batch status: no instance in slot %d", slot);
            return kErrArg;
        }
        const volatile SlotStatus *v = status_h_ + slot;
        out->t = v->t;
        out->dt = v->dt;
        out->mass = v->sums[0];
        out->mom[0] = v->sums[1];
        out->mom[1] = v->sums[2];
        out->mom[2] = v->sums[3];
        out->energy = v->sums[4];
        out->max_speed = v->max_speed;
        out->steps = v->steps;
        out->active = v->active;
        out->err = v->err;
        out->exact_passes = v->exact_passes;
        return kOk;
    }

    int state(int slot, const void **rhoE, const void **uvx, long long *row_stride) override
    {
        if (slot < 0 || slot >= cap_ || !slots_[slot].used) {
            set_error(kErrArg, "batch state: no instance in slot %d", slot);
            return kErrArg;
        }
        // the current buffer is the one the last completed step wrote: parity of steps
        const int par = (int)(status_h_[slot].steps & 1);
        *rhoE = slots_[slot].rhoE[par];
        *uvx = slots_[slot].uvx[par];
        if (row_stride) *row_stride = (long long)slots_[slot].ys;
        return kOk;
    }

    int copy_state(int slot, void *rhoE, void *uvx, bool to_host) override
    {
        const void *r, *u;
        long long ys;
        int rc = state(slot, &r, &u, &ys);
        if (rc != kOk) return rc;
        const Slot &sl = slots_[slot];
        const cudaMemcpyKind k = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        cudaError_t e;
        if constexpr (D == 2) {
            const size_t w = 2 * sizeof(T) * (sl.nb[1] + 2), sp = 2 * sizeof(T) * (size_t)ys;
            e = cudaMemcpy2DAsync(rhoE, w, r, sp, w, sl.nb[0] + 2, k, stream_);
            if (e == cudaSuccess) e = cudaMemcpy2DAsync(uvx, w, u, sp, w, sl.nb[0] + 2, k, stream_);
        } else {
            const size_t n = (sl.nb[0] + 2) * (sl.nb[1] + 2) * (sl.nb[2] + 2) * sizeof(T);
            e = cudaMemcpyAsync(rhoE, r, 2 * n, k, stream_);
            if (e == cudaSuccess) e = cudaMemcpyAsync(uvx, u, 3 * n, k, stream_);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) {
            set_error(kErrCuda, "batch copy_state: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        return kOk;
    }

    int set_skip_fraction(double f) override
    {
        if (!(f >= 0.0) || !(f <= 1e300)) {
            set_error(kErrArg, "batch skip fraction: %g is not a finite non-negative number", f);
            return kErrArg;
        }
        skip_frac_ = f;
        dirty_ = true; // the fraction is a kernel argument of the captured graph
        return kOk;
    }

    int set_arith(bool fused) override
    {
        fused_ = fused;
        dirty_ = true; // the step kernel of the captured graph changes
        return kOk;
    }

    int prepare(int nsteps) override
    {
        if (nsteps < 0) {
            set_error(kErrArg, "batch prepare: negative step count");
            return kErrArg;
        }
        return (dirty_ || nsteps != graph_steps_) ? rebuild(nsteps) : kOk;
    }

    int sync() override
    {
        const cudaError_t e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) {
            set_error(kErrCuda, "batch sync: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        return kOk;
    }

  private:
    struct Slot {
        bool used = false;
        T *rhoE[2] = {nullptr, nullptr}, *uvx[2] = {nullptr, nullptr};
        int nitems = 0;
        size_t ys = 0, nb[3] = {0, 0, 0};
    };

    void free_slot(Slot &s)
    {
        for (int b = 0; b < 2; ++b) {
            if (s.rhoE[b]) cudaFreeAsync(s.rhoE[b], stream_);
            if (s.uvx[b]) cudaFreeAsync(s.uvx[b], stream_);
            s.rhoE[b] = s.uvx[b] = nullptr;
        }
        s.used = false;
        s.nitems = 0;
    }

    void launch()
    {
        if constexpr (D == 2) {
            auto k = fused_ ? batch2d<T, true> : batch2d<T, false>;
            k<<<blocks_, kStripNT, 0, stream_>>>(insts_, items_, ranges_, nitems_, counter_, parts_, status_d_,
                                                 skip_frac_);
        } else {
            auto k = fused_ ? batch3d<T, true> : batch3d<T, false>;
            k<<<blocks_, k3NT<T>, smem_, stream_>>>(insts_, items_, ranges_, nitems_, counter_, parts_, status_d_,
                                                   skip_frac_);
        }
    }

    void launch_sums()
    {
        if constexpr (D == 2)
            batch_sums<kStripNT, T, Inst><<<sum_blocks_, kStripNT, 0, stream_>>>(insts_, items_, ranges_, nitems_,
                                                                                counter_ + 1, parts_, status_d_);
        else
            batch_sums<k3NT<T>, T, Inst><<<sum_blocks_, k3NT<T>, 0, stream_>>>(insts_, items_, ranges_, nitems_,
                                                                        counter_ + 1, parts_, status_d_);
    }

    // Work list and partial slots for the instances in use; the graph of `nsteps` steps
    // followed by the conservation sums.
    int rebuild(int nsteps)
    {
        std::vector<int2> items;
        for (int i = 0; i < cap_; ++i) {
            if (!slots_[i].used) {
                host_ranges_[i] = make_int2(0, 0);
                continue;
            }
            host_ranges_[i] = make_int2((int)items.size(), slots_[i].nitems);
            for (int k = 0; k < slots_[i].nitems; ++k) items.push_back(make_int2(i, k));
        }
        cudaError_t e = cudaStreamSynchronize(stream_);
        if (e == cudaSuccess && items.size() > items_cap_) {
            cudaFree(items_);
            cudaFree(parts_);
            items_ = nullptr;
            parts_ = nullptr;
            items_cap_ = std::max(items.size(), 2 * items_cap_);
            e = cudaMalloc(&items_, sizeof(int2) * items_cap_);
            if (e == cudaSuccess) e = cudaMalloc(&parts_, sizeof(ItemPart) * items_cap_);
            if (e != cudaSuccess) items_cap_ = 0;
        }
        nitems_ = (int)items.size();
        if (e == cudaSuccess && nitems_ > 0)
            e = cudaMemcpyAsync(items_, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ranges_, host_ranges_.data(), sizeof(int2) * cap_, cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        if (e == cudaSuccess && nitems_ > 0 && nsteps > 0) {
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
            for (int k = 0; k < nsteps && e == cudaSuccess; ++k) {
                e = cudaMemsetAsync(counter_, 0, sizeof(unsigned), stream_);
                if (e == cudaSuccess) {
                    launch();
                    e = cudaGetLastError();
                }
            }
            // the conservation sums of the state the run ends on
            if (e == cudaSuccess) e = cudaMemsetAsync(counter_ + 1, 0, sizeof(unsigned), stream_);
            if (e == cudaSuccess) {
                launch_sums();
                e = cudaGetLastError();
            }
            const cudaError_t e2 = cudaStreamEndCapture(stream_, &g);
            if (e == cudaSuccess) e = e2;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&graph_, g, 0);
            if (g) cudaGraphDestroy(g);
        }
        if (e != cudaSuccess) {
            set_error(kErrCuda, "batch rebuild: %s", cudaGetErrorString(e));
            return kErrCuda;
        }
        dirty_ = false;
        graph_steps_ = nsteps;
        return kOk;
    }

    int chunk_, cap_;
    double skip_frac_ = kSkipFrac;
    bool fused_ = false; // fused arithmetic of the step kernels (hydro_batch_set_arith)
    bool own_stream_ = false, dirty_ = true;
    cudaStream_t stream_ = nullptr;
    Inst *insts_ = nullptr;
    int2 *ranges_ = nullptr, *items_ = nullptr;
    size_t items_cap_ = 0;
    ItemPart *parts_ = nullptr;
    unsigned *counter_ = nullptr;
    unsigned long long *scratch_bits_ = nullptr;
    SlotStatus *status_h_ = nullptr, *status_d_ = nullptr;
    std::vector<Slot> slots_;
    std::vector<int2> host_ranges_;
    int nitems_ = 0, blocks_ = 1, sum_blocks_ = 1, graph_steps_ = -1, smem_ = 0;
    cudaGraphExec_t graph_ = nullptr;
};

} // namespace hydro

using namespace hydro;

extern "C" {

void *hydro_batch_create(int dim, int precision_bytes, int chunk, int capacity, void *stream)
{
    if ((dim != 2 && dim != 3) || (precision_bytes != 4 && precision_bytes != 8) || capacity <= 0 ||
        capacity > (1 << 20) || chunk < 0) {
        set_error(kErrArg, "hydro_batch_create: unsupported (dim %d, precision %d bytes, capacity %d)", dim,
                  precision_bytes, capacity);
        return nullptr;
    }
    int rc = kOk;
    BatchBase *b = nullptr;
    const cudaStream_t s = (cudaStream_t)stream;
    if (dim == 2 && precision_bytes == 8) b = new BatchEngine<double, 2>(chunk, capacity, s, &rc);
    else if (dim == 2) b = new BatchEngine<float, 2>(chunk, capacity, s, &rc);
    else if (precision_bytes == 8) b = new BatchEngine<double, 3>(chunk, capacity, s, &rc);
    else b = new BatchEngine<float, 3>(chunk, capacity, s, &rc);
    if (rc != kOk) {
        delete b;
        return nullptr;
    }
    return b;
}

int hydro_batch_add(void *b, const hydro_blast_t *spec)
{
    if (!b || !spec) {
        set_error(kErrArg, "hydro_batch_add: null argument");
        return kErrArg;
    }
    return static_cast<BatchBase *>(b)->add(*spec);
}

int hydro_batch_remove(void *b, int slot)
{
    if (!b) return kErrArg;
    return static_cast<BatchBase *>(b)->remove(slot);
}

int hydro_batch_run(void *b, int nsteps, int sync)
{
    if (!b) return kErrArg;
    return static_cast<BatchBase *>(b)->run(nsteps, sync != 0);
}

int hydro_batch_status(void *b, int slot, hydro_batch_status_t *out)
{
    if (!b) return kErrArg;
    return static_cast<BatchBase *>(b)->status(slot, out);
}

int hydro_batch_state(void *b, int slot, const void **rhoE, const void **uvx, long long *row_stride)
{
    if (!b || !rhoE || !uvx) return kErrArg;
    return static_cast<BatchBase *>(b)->state(slot, rhoE, uvx, row_stride);
}

int hydro_batch_copy_state(void *b, int slot, void *rhoE, void *uvx, int to_host)
{
    if (!b || !rhoE || !uvx) return kErrArg;
    return static_cast<BatchBase *>(b)->copy_state(slot, rhoE, uvx, to_host != 0);
}

long long hydro_batch_bytes(void *b, const hydro_blast_t *spec)
{
    if (!b || !spec) return kErrArg;
    return (long long)static_cast<BatchBase *>(b)->bytes(*spec);
}

int hydro_batch_prepare(void *b, int nsteps)
{
    if (!b) return kErrArg;
    return static_cast<BatchBase *>(b)->prepare(nsteps);
}

int hydro_batch_set_arith(void *b, int arith)
{
    if (!b || (arith & ~(HYDRO_ARITH_FUSED | HYDRO_ARITH_STRICT))) {
        set_error(kErrArg, "hydro_batch_set_arith: null batch or unknown bits 0x%x", arith);
        return kErrArg;
    }
    return static_cast<BatchBase *>(b)->set_arith((arith & HYDRO_ARITH_FUSED) && !(arith & HYDRO_ARITH_STRICT));
}

int hydro_batch_set_skip_fraction(void *b, double frac)
{
    if (!b) return kErrArg;
    return static_cast<BatchBase *>(b)->set_skip_fraction(frac);
}

int hydro_batch_sync(void *b)
{
    if (!b) return kErrArg;
    return static_cast<BatchBase *>(b)->sync();
}

void hydro_batch_destroy(void *b) { delete static_cast<BatchBase *>(b); }

int hydro2d_init_blast_at_f64(double *d_rhoE, double *d_uv, size_t NB_X, size_t NB_Y, double cx, double cy,
                              double radius, double rho_in, double rho_out, double p_in, double p_out, double C_min,
                              double gamma, double *min_dt, void *stream)
{
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    return init2d_at<double>(d_rhoE, d_uv, NB_X, NB_Y, cx, cy, radius, rho_in, rho_out, p_in, p_out, C_min, gamma,
                             min_dt, (cudaStream_t)stream, &ctx->scr->max_bits);
}
int hydro2d_init_blast_at_f32(float *d_rhoE, float *d_uv, size_t NB_X, size_t NB_Y, double cx, double cy,
                              double radius, float rho_in, float rho_out, float p_in, float p_out, float C_min,
                              float gamma, float *min_dt, void *stream)
{
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    return init2d_at<float>(d_rhoE, d_uv, NB_X, NB_Y, cx, cy, radius, rho_in, rho_out, p_in, p_out, C_min, gamma,
                            min_dt, (cudaStream_t)stream, &ctx->scr->max_bits);
}
int hydro3d_init_blast_at_f64(double *d_rhoE, double *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, double cx,
                              double cy, double cz, double radius, double rho_in, double rho_out, double p_in,
                              double p_out, double C_min, double gamma, double *min_dt, void *stream)
{
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    return init3d_at<double>(d_rhoE, d_uvw, NB_X, NB_Y, NB_Z, cx, cy, cz, radius, rho_in, rho_out, p_in, p_out,
                             C_min, gamma, min_dt, (cudaStream_t)stream, &ctx->scr->max_bits);
}
int hydro3d_init_blast_at_f32(float *d_rhoE, float *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, double cx,
                              double cy, double cz, double radius, float rho_in, float rho_out, float p_in,
                              float p_out, float C_min, float gamma, float *min_dt, void *stream)
{
    int err;
    DevCtx *ctx = ctx_current(&err);
    if (!ctx) return err;
    return init3d_at<float>(d_rhoE, d_uvw, NB_X, NB_Y, NB_Z, cx, cy, cz, radius, rho_in, rho_out, p_in, p_out,
                            C_min, gamma, min_dt, (cudaStream_t)stream, &ctx->scr->max_bits);
}

} // extern "C"
