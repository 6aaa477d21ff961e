// Device runtime pieces shared by the 2D and 3D kernels:
//  - mbarrier / TMA (cp.async.bulk.tensor) inline-PTX wrappers, every wait bounded, and
//    the per-thread cp.async copies used where TMA's alignment rules do not fit;
//  - the fused end-of-step reduction: the CFL maximum signal speed (the reference
//    folds it serially, hydro2d/kernel.cxx:313 and :318) and an FP64 compensated sum of
//    the new density (the mass the reference sums on the host in long double,
//    hydro2d/main.cxx:237-265), combined with warp shuffles, one partial per block and
//    one ticket atomic per block; the last block to finish writes Dt_next and the
//    status record and re-arms the scratch words for the next launch.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "hydro_math.cuh"

namespace hydro {

// error bits reported in StepStatus::err and by hydro_last_error()
enum : unsigned {
    kErrNonPhysical = 1u,  // a new cell with rho <= 0 or a non-finite signal speed
    kErrWaitTimeout = 2u,  // a bounded wait on a TMA barrier gave up
};

// Scratch words in device memory, one set per device context. max_bits, ticket and
// err are zero between launches (the last block of each launch resets them).
//
// Signal-speed skipping: a step reads the max signal speed of the previous completed
// step of the same problem (hist_max, matched by hist_key) and computes the exact speed
// only of cells whose cheap upper bound reaches skip_frac * hist_max. If the exact max
// found that way is below the threshold, a skipped cell might hold the true max: the
// step then sets `redo` and leaves Dt_next to the redo pass, which computes the exact
// speed of every cell. Dt_next is therefore always the exact reference value.
struct StepScratch {
    unsigned long long max_bits; // max signal speed as the bits of a non-negative double
    unsigned int ticket;         // blocks finished so far in this launch
    unsigned int err;            // error bits raised in this launch
    unsigned int redo;           // the last step left Dt_next to the redo pass
    unsigned int pad0;
    unsigned long long hist_key; // problem key of the last completed step
    double hist_max;             // its max signal speed
};

constexpr double kSkipFrac = 0.9;

// Result record of one launch, written by the last block (host-mapped memory).
struct StepStatus {
    double mass;       // sum of the new interior density (compensated FP64)
    double mass_comp;  // its compensation term
    double max_speed;  // max over interior cells of c_s + |u| of the new state
    unsigned int err;  // error bits
    unsigned int seq;  // launch sequence number, for the host to check completion
    unsigned int redo; // Dt_next still to be written by the redo pass
    unsigned int pad;
};

// Skip threshold of a step: the previous max of the same problem, scaled.
__device__ __forceinline__ double skip_threshold(const StepScratch *scr, unsigned long long key)
{
    const unsigned long long k = *reinterpret_cast<const volatile unsigned long long *>(&scr->hist_key);
    const double m = *reinterpret_cast<const volatile double *>(&scr->hist_max);
    return (key != 0ull && k == key) ? kSkipFrac * m : 0.0;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Wait for phase `parity` of a barrier, giving up after ~2^31 clock cycles (about a
// second). Returns false on time-out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 31)) return false;
    }
    return true;
}

// 2D tiled TMA load into shared memory, completion signalled on `bar`. The innermost
// coordinate x must be a multiple of 16 bytes / element size (asserted by the host).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int x, int y, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, int x, int y, int z, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                 : "memory");
}

// Per-thread asynchronous copy global -> shared of 4, 8 or 16 bytes (zero-filled when
// !valid); completion by commit groups, waited on by the issuing thread.
__device__ __forceinline__ void cp_async(void *dst, const void *src, int bytes, bool valid)
{
    const uint32_t d = smem_u32(dst);
    const int n = valid ? bytes : 0;
    if (bytes == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *tm)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

// Neumaier-compensated accumulation (s, c) += x, the FP64 counterpart of the
// reference's long-double loop (hydro2d/main.cxx:251-256).
__device__ __forceinline__ void neumaier_add(double &s, double &c, double x)
{
    const double t = __dadd_rn(s, x);
    if (fabs(s) >= fabs(x)) c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, t), x));
    else c = __dadd_rn(c, __dadd_rn(__dsub_rn(x, t), s));
    s = t;
}

__device__ __forceinline__ void neumaier_merge(double &s, double &c, double s2, double c2)
{
    neumaier_add(s, c, s2);
    c = __dadd_rn(c, c2);
}

// Per-thread accumulator of the fused reductions.
struct StepAcc {
    double vmax = 0.0; // running max of the signal speed (NaN never enters: flagged instead)
    double ms = 0.0, mc = 0.0;
    unsigned err = 0;

    template <class T> __device__ __forceinline__ void add_cell(T rho_new, T speed)
    {
        add_mass(rho_new);
        add_speed(speed);
    }
    template <class T> __device__ __forceinline__ void add_mass(T rho_new)
    {
        if (!(rho_new > T(0))) err |= kErrNonPhysical;
        // Kahan step, branch-free; mc carries the low part to add back (mass = ms + mc)
        const double y = __dadd_rn(static_cast<double>(rho_new), mc);
        const double tt = __dadd_rn(ms, y);
        mc = __dsub_rn(y, __dsub_rn(tt, ms));
        ms = tt;
    }
    template <class T> __device__ __forceinline__ void add_speed(T speed)
    {
        const double sp = static_cast<double>(speed);
        vmax = (sp > vmax) ? sp : vmax;
        if (!(sp <= 1.0e300)) err |= kErrNonPhysical;
    }
};

// Warp + block max of non-negative doubles held as bits; result valid in thread 0.
template <int NT> __device__ __forceinline__ unsigned long long block_max_bits(unsigned long long mb, unsigned long long *s_max)
{
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = t & 31, warp = t >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long om = __shfl_xor_sync(0xffffffffu, mb, o);
        mb = om > mb ? om : mb;
    }
    if (lane == 0) s_max[warp] = mb;
    __syncthreads();
    if (t == 0)
        for (int w = 1; w < NT / 32; ++w) mb = s_max[w] > mb ? s_max[w] : mb;
    return mb;
}

// The last block's common tail: Dt_next = C_min / max (in T, as the reference does at
// hydro2d/kernel.cxx:318) unless the max fell below the skip threshold, the history
// for the next step, and the re-arming of the scratch words. Thread 0 only.
template <class T>
__device__ __forceinline__ void finish_dt(StepScratch *scr, double vmax, double tlo, unsigned long long key, T C_min,
                                          T *Dt_next, StepStatus *status)
{
    const unsigned redo = (vmax < tlo) ? 1u : 0u;
    if (!redo) {
        // the max of values of type T, held exactly in a double, converts back exactly
        *Dt_next = Ar<T>::div(C_min, static_cast<T>(vmax));
        scr->hist_key = key;
        scr->hist_max = vmax;
    }
    scr->redo = redo;
    if (status) {
        status->max_speed = vmax;
        status->redo = redo;
    }
}

// Block-wide combination of the accumulators, one partial per block, one ticket atomic
// per block; the last block writes *Dt_next = C_min / max_speed (in T, as the
// reference does at hydro2d/kernel.cxx:318) and the status record. NT = threads/block.
template <int NT, class T>
__device__ __forceinline__ void step_epilogue(StepAcc acc, StepScratch *scr, double2 *partials, unsigned nblocks,
                                              unsigned bid, T C_min, T *Dt_next, StepStatus *status, unsigned seq,
                                              double tlo = 0.0, unsigned long long key = 0ull)
{
    static_assert(NT % 32 == 0 && NT <= 1024, "block size");
    constexpr int NW = NT / 32;
    __shared__ unsigned long long s_max[NW];
    __shared__ double s_ms[NW], s_mc[NW];
    __shared__ unsigned s_err[NW];
    __shared__ bool s_last;

    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = t & 31, warp = t >> 5;
    unsigned long long mb = __double_as_longlong(acc.vmax);
    double ms = acc.ms, mc = acc.mc;
    unsigned err = acc.err;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long om = __shfl_xor_sync(0xffffffffu, mb, o);
        mb = om > mb ? om : mb;
        const double s2 = __shfl_xor_sync(0xffffffffu, ms, o);
        const double c2 = __shfl_xor_sync(0xffffffffu, mc, o);
        if (lane & o) { // deterministic pairing: the higher lane folds into the lower
            double a = s2, b = c2;
            neumaier_merge(a, b, ms, mc);
            ms = a; mc = b;
        } else {
            neumaier_merge(ms, mc, s2, c2);
        }
        err |= __shfl_xor_sync(0xffffffffu, err, o);
    }
    if (lane == 0) {
        s_max[warp] = mb;
        s_ms[warp] = ms;
        s_mc[warp] = mc;
        s_err[warp] = err;
    }
    __syncthreads();
    if (t == 0) {
        for (int w = 1; w < NW; ++w) {
            mb = s_max[w] > mb ? s_max[w] : mb;
            neumaier_merge(ms, mc, s_ms[w], s_mc[w]);
            err |= s_err[w];
        }
        partials[bid] = make_double2(ms, mc);
        atomicMax(&scr->max_bits, mb);
        if (err) atomicOr(&scr->err, err);
        __threadfence();
        const unsigned prev = atomicAdd(&scr->ticket, 1u);
        s_last = (prev == nblocks - 1);
    }
    __syncthreads();
    if (!s_last) return;

    // last block: all partials and the max are visible after the fence
    __threadfence();
    double s = 0.0, c = 0.0;
    for (unsigned b = t; b < nblocks; b += NT) {
        const double2 p = __ldcg(&partials[b]);
        neumaier_merge(s, c, p.x, p.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double s2 = __shfl_xor_sync(0xffffffffu, s, o);
        const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
        if (lane & o) {
            double a = s2, b = c2;
            neumaier_merge(a, b, s, c);
            s = a; c = b;
        } else {
            neumaier_merge(s, c, s2, c2);
        }
    }
    if (lane == 0) {
        s_ms[warp] = s;
        s_mc[warp] = c;
    }
    __syncthreads();
    if (t == 0) {
        for (int w = 1; w < NW; ++w) neumaier_merge(s, c, s_ms[w], s_mc[w]);
        const unsigned long long gm = atomicAdd(&scr->max_bits, 0ull);
        const unsigned gerr = atomicAdd(&scr->err, 0u);
        const double vmax = __longlong_as_double(static_cast<long long>(gm));
        finish_dt(scr, vmax, tlo, key, C_min, Dt_next, status);
        if (status) {
            status->mass = s;
            status->mass_comp = c;
            status->err = gerr;
            __threadfence_system();
            status->seq = seq;
        }
        scr->max_bits = 0ull;
        scr->err = 0u;
        __threadfence();
        scr->ticket = 0u;
    }
}

// Epilogue of the redo pass: the exact max over every cell, then Dt_next.
template <int NT, class T>
__device__ __forceinline__ void redo_epilogue(double vmax, unsigned err, StepScratch *scr, unsigned nblocks, T C_min,
                                              T *Dt_next, StepStatus *status, unsigned long long key)
{
    __shared__ unsigned long long s_max[NT / 32];
    __shared__ bool s_last;
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    err = __reduce_or_sync(0xffffffffu, err);
    unsigned long long mb = block_max_bits<NT>(__double_as_longlong(vmax), s_max);
    if (t == 0) {
        atomicMax(&scr->max_bits, mb);
        if (err) atomicOr(&scr->err, err);
        __threadfence();
        s_last = (atomicAdd(&scr->ticket, 1u) == nblocks - 1);
    }
    __syncthreads();
    if (!s_last || t != 0) return;
    __threadfence();
    const unsigned long long gm = atomicAdd(&scr->max_bits, 0ull);
    const unsigned gerr = atomicAdd(&scr->err, 0u);
    finish_dt(scr, __longlong_as_double(static_cast<long long>(gm)), 0.0, key, C_min, Dt_next, status);
    if (status) {
        status->err |= gerr;
        __threadfence_system();
    }
    scr->max_bits = 0ull;
    scr->err = 0u;
    __threadfence();
    scr->ticket = 0u;
}

} // namespace hydro
