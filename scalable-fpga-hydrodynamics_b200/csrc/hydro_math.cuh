// Per-cell arithmetic of the first-order finite-volume update, device side.
//
// Every operation is an explicit round-to-nearest intrinsic (__dmul_rn, __dadd_rn,
// __drcp_rn, __dsqrt_rn, and the float forms), so the compiler can neither contract a
// multiply and an add into an FMA nor reassociate, whatever -fmad/-use_fast_math say.
// Each expression keeps the association of the reference source it restates, which
// makes the results bit-identical to the reference kernel compiled for an IEEE host
// without contraction (x86-64 SSE2, -ffp-contract=off).
//
// Faces are computed once per face instead of once per adjacent cell as the reference
// does (hydro2d/kernel.cxx:186-251 evaluates each face from both sides); the two
// evaluations there take identical arguments, so one evaluation gives the same bits.
// Quantities that depend on one cell only (primitives, the acoustic impedance
// sqrt(gamma*p*rho), the upwinded conservative values) are computed once per cell.
//
// Every per-cell function takes a template flag kF selecting the arithmetic:
//  kF = false (strict): the reference's operation order with one rounding per operation,
//    bit-identical to the reference kernel compiled without contraction;
//  kF = true (fused): the same formulas with each product that feeds a sum fused into one
//    rounding (fma), the reciprocal and square roots from the hardware approximations
//    refined by one third-order step (Fu below), and the energy of z faces taken from the
//    same sum of squares as x and y faces. Each result differs from the strict one by a few
//    units in the last place; not bit-identical.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hydro {

template <class T> struct Ar;

template <> struct Ar<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    // 1/x correctly rounded: the same value as ONE / x in IEEE double
    static __device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
    static constexpr double half = 0.5;
};

template <> struct Ar<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float rcp(float a) { return __frcp_rn(a); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
    static constexpr float half = 0.5f;
};

// Fused-mode primitives. Reciprocal and reciprocal square root start from the hardware
// approximations (PTX rcp.approx.ftz / rsqrt.approx.ftz) and take one third-order
// Householder step, which cubes the relative error of the start value:
//   1/a:       e = 1 - a y,          y' = y (1 + e + e^2)
//   1/sqrt(s): e = 1 - s y^2,        y' = y (1 + e/2 + 3 e^2 / 8)
// (the truncated binomial series of (1 - e)^-1 and (1 - e)^-1/2). The result is within a
// few ulp of the correctly rounded value. Inputs outside [2^-1000, 2^1000] (zero,
// subnormal, huge, negative, NaN), where the flush-to-zero approximations do not apply,
// take the correctly rounded intrinsic instead.
template <class T> struct Fu;

template <> struct Fu<double> {
    static __device__ __forceinline__ bool regular(double a)
    {
        const double m = fabs(a);
        return m >= 0x1p-1000 && m <= 0x1p1000;
    }
    // the refined reciprocal without the range check: equal to rcp(a) for regular a
    static __device__ __forceinline__ double rcp_reg(double a)
    {
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
        const double e = __fma_rn(-a, y, 1.0);
        return __fma_rn(y, __fma_rn(e, e, e), y);
    }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double rcp(double a)
    {
        if (!regular(a)) return __drcp_rn(a);
        return rcp_reg(a);
    }
    // 1/sqrt(s) for regular s > 0
    static __device__ __forceinline__ double rsqrt_pos(double s)
    {
        double y;
        asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(s));
        const double e = __fma_rn(-__dmul_rn(s, y), y, 1.0);
        return __fma_rn(y, __dmul_rn(e, __fma_rn(0.375, e, 0.5)), y);
    }
    static __device__ __forceinline__ double sqrt(double s)
    {
        if (!(s > 0.0 && regular(s))) return __dsqrt_rn(s);
        return __dmul_rn(s, rsqrt_pos(s));
    }
};

template <> struct Fu<float> {
    static __device__ __forceinline__ bool regular(float a)
    {
        const float m = fabsf(a);
        return m >= 0x1p-100f && m <= 0x1p100f;
    }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float rcp(float a)
    {
        if (!regular(a)) return __frcp_rn(a);
        float y;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
        const float e = __fmaf_rn(-a, y, 1.0f);
        return __fmaf_rn(y, __fmaf_rn(e, e, e), y);
    }
    static __device__ __forceinline__ float rsqrt_pos(float s)
    {
        float y;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(s));
        const float e = __fmaf_rn(-__fmul_rn(s, y), y, 1.0f);
        return __fmaf_rn(y, __fmul_rn(e, __fmaf_rn(0.375f, e, 0.5f)), y);
    }
    static __device__ __forceinline__ float sqrt(float s)
    {
        if (!(s > 0.0f && regular(s))) return __fsqrt_rn(s);
        return __fmul_rn(s, rsqrt_pos(s));
    }
};

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// std::max(a, b) as the reference calls it: a unless a < b
template <class T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }

// Physical constants of one launch (hydro2d/kernel.hpp:63-68 argument list).
template <class T> struct Phys {
    T C_min, gamma, gm1, divgamma, K;
    bool kneg; // K < 0
    T iK;      // 1 / K (fused arithmetic: 1/(K a) = (1/K)(1/a))

    static Phys make(T C_min, T gamma, T gm1, T divgamma, T K)
    {
        return Phys{C_min, gamma, gm1, divgamma, K, K < T(0), T(1) / K};
    }
};

// A cell seen by the face flux: everything compute_fluxes needs from one side
// (hydro2d/kernel.cxx:74-118), with the normal velocity and normal/tangential momenta
// already routed for the face direction.
//
// The face's acoustic impedance a = K * max(a_left, a_right) (kernel.cxx:95) is always
// one of the two per-cell products K*a_left, K*a_right (the same rounded product), and
// 1/a (kernel.cxx:97) is then one of the two per-cell reciprocals. Both are computed
// once per cell and the face only selects: a monotone rounding keeps the choice
// identical to comparing the unscaled a's (equal products are the same value).
template <class T> struct FaceIn {
    T r;   // density
    T un;  // normal velocity
    T p;   // pressure
    T Ka;  // K * sqrt(gamma * p * rho)
    T iKa; // 1 / (K * sqrt(gamma * p * rho))
    T mn;  // un * rho   (the reference's U_upwind_ux for this direction)
    T mt;  // ut * rho   (U_upwind_uy)
    T eup; // p * divgamma + (0.5 * rho) * |u|^2   (U_upwind_p)
};

template <class T> struct FaceIn3 {
    T r, un, p, Ka, iKa, mn, mt1, mt2, eup;
};

template <class T> struct Flux2 { T r, n, t, E; };
template <class T> struct Flux3 { T r, n, t1, t2, E; };

// Primitive variables of a 2D cell, hydro2d/kernel.cxx:5-29/31-53:
//   inv = 1/rho ; u = rho_u*inv ; v = rho_v*inv ; temp = u*u + v*v
//   p = (gm1*rho) * (E*inv - 0.5*temp)
// plus the per-cell face quantities (a, u*rho, v*rho, upwinded energy).
template <class T> struct Cell2 {
    T r, u, v, p, Ka, iKa, mu, mv, eup;
};

template <class T, bool kF = false>
__device__ __forceinline__ Cell2<T> make_cell2_checked(T ur, T uu, T uv, T uE, const Phys<T> &ph);

// FP64 fused arithmetic: one straight-line block (no branch inside the chain, so the
// scheduler can interleave it with the face evaluations around it), then one warp-uniform
// branch that recomputes the cells whose density or gamma p rho fell outside the range of
// the refined approximations; the values equal make_cell2_checked's in every lane (2D
// 88.2 -> 89.4 GCell/s fused at 40000 x 20000; the FP32 3D form measured slower and keeps
// the checked path).
template <class T, bool kF = false>
__device__ __forceinline__ Cell2<T> make_cell2(T ur, T uu, T uv, T uE, const Phys<T> &ph)
{
    if constexpr (kF && sizeof(T) == 8) {
        using A = Ar<T>;
        using F = Fu<T>;
        Cell2<T> c;
        const T inv = F::rcp_reg(ur);
        c.r = ur;
        c.u = A::mul(uu, inv);
        c.v = A::mul(uv, inv);
        const T temp = F::fma(c.v, c.v, A::mul(c.u, c.u));
        c.p = A::mul(A::mul(ph.gm1, ur), F::fma(-A::half, temp, A::mul(uE, inv)));
        const T s = A::mul(A::mul(ph.gamma, c.p), c.r);
        const T y = F::rsqrt_pos(s);
        c.Ka = A::mul(ph.K, A::mul(s, y));
        c.iKa = A::mul(ph.iK, y);
        c.mu = A::mul(c.u, c.r);
        c.mv = A::mul(c.v, c.r);
        c.eup = F::fma(A::mul(A::half, c.r), temp, A::mul(c.p, ph.divgamma));
        const bool bad = !F::regular(ur) || !(s > T(0) && F::regular(s));
        if (__any_sync(__activemask(), bad)) {
            if (bad) c = make_cell2_checked<T, true>(ur, uu, uv, uE, ph);
        }
        return c;
    } else {
        return make_cell2_checked<T, kF>(ur, uu, uv, uE, ph);
    }
}

// The per-cell conversion with the range checks inside the chain (both arithmetics).
template <class T, bool kF>
__device__ __forceinline__ Cell2<T> make_cell2_checked(T ur, T uu, T uv, T uE, const Phys<T> &ph)
{
    using A = Ar<T>;
    Cell2<T> c;
    if constexpr (kF) {
        using F = Fu<T>;
        const T inv = F::rcp(ur);
        c.r = ur;
        c.u = A::mul(uu, inv);
        c.v = A::mul(uv, inv);
        const T temp = F::fma(c.v, c.v, A::mul(c.u, c.u));
        c.p = A::mul(A::mul(ph.gm1, ur), F::fma(-A::half, temp, A::mul(uE, inv)));
        const T s = A::mul(A::mul(ph.gamma, c.p), c.r);
        if (s > T(0) && F::regular(s)) {
            const T y = F::rsqrt_pos(s);
            c.Ka = A::mul(ph.K, A::mul(s, y));
            c.iKa = A::mul(ph.iK, y);
        } else {
            c.Ka = A::mul(ph.K, A::sqrt(s));
            c.iKa = A::rcp(c.Ka);
        }
        c.mu = A::mul(c.u, c.r);
        c.mv = A::mul(c.v, c.r);
        c.eup = F::fma(A::mul(A::half, c.r), temp, A::mul(c.p, ph.divgamma));
        return c;
    }
    const T inv = A::rcp(ur);
    c.r = ur;
    c.u = A::mul(uu, inv);
    c.v = A::mul(uv, inv);
    const T temp = A::add(A::mul(c.u, c.u), A::mul(c.v, c.v));
    const T e_int = A::sub(A::mul(uE, inv), A::mul(A::half, temp));
    c.p = A::mul(A::mul(ph.gm1, ur), e_int);
    // a_left = SQRT(gamma * Q_p_left * Q_rho_left)   (kernel.cxx:92), scaled by K
    c.Ka = A::mul(ph.K, A::sqrt(A::mul(A::mul(ph.gamma, c.p), c.r)));
    c.iKa = A::rcp(c.Ka);
    // U_upwind_ux/uy = Q_upwind_u * Q_upwind_rho      (kernel.cxx:109-110)
    c.mu = A::mul(c.u, c.r);
    c.mv = A::mul(c.v, c.r);
    // U_upwind_p = Q_p*divgamma + (HALF*Q_rho)*(u*u + v*v)   (kernel.cxx:111); the sum
    // of two squares commutes exactly, so x and y faces share one value.
    c.eup = A::add(A::mul(c.p, ph.divgamma), A::mul(A::mul(A::half, c.r), temp));
    return c;
}

// x faces: normal = u
template <class T> __device__ __forceinline__ FaceIn<T> face_x(const Cell2<T> &c)
{
    return FaceIn<T>{c.r, c.u, c.p, c.Ka, c.iKa, c.mu, c.mv, c.eup};
}
// y faces: normal = v, the reference swaps (ux, uy) in the call (kernel.cxx:228-229)
template <class T> __device__ __forceinline__ FaceIn<T> face_y(const Cell2<T> &c)
{
    return FaceIn<T>{c.r, c.v, c.p, c.Ka, c.iKa, c.mv, c.mu, c.eup};
}
// reflective wall: mirror state with the normal velocity negated (kernel.cxx:222-225);
// -(v*rho) == (-v)*rho exactly, and the energy depends on v*v only.
template <class T> __device__ __forceinline__ FaceIn<T> mirror(const FaceIn<T> &f)
{
    return FaceIn<T>{f.r, -f.un, f.p, f.Ka, f.iKa, -f.mn, f.mt, f.eup};
}

// compute_fluxes, hydro2d/kernel.cxx:74-118, from cached per-cell quantities.
template <class T, bool kF = false>
__device__ __forceinline__ Flux2<T> face_flux(const FaceIn<T> &L, const FaceIn<T> &R, const Phys<T> &ph)
{
    using A = Ar<T>;
    // std::max(a_left, a_right) takes a_right iff a_left < a_right; with K < 0 the
    // products order the other way
    const bool right = ph.kneg ? (R.Ka < L.Ka) : (L.Ka < R.Ka);
    const T a = right ? R.Ka : L.Ka;
    const T diva = right ? R.iKa : L.iKa;
    if constexpr (kF) {
        using F = Fu<T>;
        const T us = A::mul(A::half, F::fma(-diva, A::sub(R.p, L.p), A::add(L.un, R.un)));
        const T ps = A::mul(A::half, F::fma(-a, A::sub(R.un, L.un), A::add(L.p, R.p)));
        const bool up = us >= T(0);
        Flux2<T> F2;
        F2.r = A::mul(up ? L.r : R.r, us);
        F2.n = F::fma(up ? L.mn : R.mn, us, ps);
        F2.t = A::mul(up ? L.mt : R.mt, us);
        F2.E = F::fma(up ? L.eup : R.eup, us, A::mul(ps, us));
        return F2;
    }
    const T us = A::mul(A::half, A::sub(A::add(L.un, R.un), A::mul(diva, A::sub(R.p, L.p))));
    const T ps = A::mul(A::half, A::sub(A::add(L.p, R.p), A::mul(a, A::sub(R.un, L.un))));
    const bool up = us >= T(0);
    const T r = up ? L.r : R.r;
    const T mn = up ? L.mn : R.mn;
    const T mt = up ? L.mt : R.mt;
    const T e = up ? L.eup : R.eup;
    Flux2<T> F;
    F.r = A::add(A::mul(r, us), T(0)); // "+ ZERO" kept: it turns -0 into +0
    F.n = A::add(A::mul(mn, us), ps);
    F.t = A::add(A::mul(mt, us), T(0));
    F.E = A::add(A::mul(e, us), A::mul(ps, us));
    return F;
}

// The 2D conservative update and the new state's signal speed,
// hydro2d/kernel.cxx:259-313. fx_lo/fx_hi are the faces at i-1/2 and i+1/2,
// fy_lo/fy_hi at j-1/2 and j+1/2 (y fluxes carry the y momentum in .n).
template <class T> struct Upd2 {
    T r, u, v, E, speed;
};

template <class T, bool kF = false>
__device__ __forceinline__ Upd2<T> update2(T ur, T uu, T uv, T uE, const Flux2<T> &fx_lo, const Flux2<T> &fx_hi,
                                           const Flux2<T> &fy_lo, const Flux2<T> &fy_hi, T DtDx, T DtDy,
                                           const Phys<T> &ph)
{
    using A = Ar<T>;
    if constexpr (kF) {
        using F = Fu<T>;
        Upd2<T> o;
        o.r = F::fma(DtDy, A::sub(fy_lo.r, fy_hi.r), F::fma(DtDx, A::sub(fx_lo.r, fx_hi.r), ur));
        o.u = F::fma(DtDy, A::sub(fy_lo.t, fy_hi.t), F::fma(DtDx, A::sub(fx_lo.n, fx_hi.n), uu));
        o.v = F::fma(DtDy, A::sub(fy_lo.n, fy_hi.n), F::fma(DtDx, A::sub(fx_lo.t, fx_hi.t), uv));
        o.E = F::fma(DtDy, A::sub(fy_lo.E, fy_hi.E), F::fma(DtDx, A::sub(fx_lo.E, fx_hi.E), uE));
        o.speed = T(0);
        return o;
    }
    const T x_r = A::mul(DtDx, A::sub(fx_lo.r, fx_hi.r));
    const T x_u = A::mul(DtDx, A::sub(fx_lo.n, fx_hi.n));
    const T x_v = A::mul(DtDx, A::sub(fx_lo.t, fx_hi.t));
    const T x_E = A::mul(DtDx, A::sub(fx_lo.E, fx_hi.E));
    const T y_r = A::mul(DtDy, A::sub(fy_lo.r, fy_hi.r));
    const T y_u = A::mul(DtDy, A::sub(fy_lo.t, fy_hi.t));
    const T y_v = A::mul(DtDy, A::sub(fy_lo.n, fy_hi.n));
    const T y_E = A::mul(DtDy, A::sub(fy_lo.E, fy_hi.E));
    Upd2<T> o;
    o.r = A::add(A::add(ur, x_r), y_r);
    o.u = A::add(A::add(uu, x_u), y_u);
    o.v = A::add(A::add(uv, x_v), y_v);
    o.E = A::add(A::add(uE, x_E), y_E);
    o.speed = T(0);
    return o;
}

// Signal speed c_s + |u| of a 2D state, hydro2d/kernel.cxx:287-309.
template <class T, bool kF = false> __device__ __forceinline__ T speed2(T r, T ru, T rv, T E, const Phys<T> &ph)
{
    using A = Ar<T>;
    if constexpr (kF) {
        using F = Fu<T>;
        const T inv = F::rcp(r);
        const T qu = A::mul(ru, inv), qv = A::mul(rv, inv);
        const T temp = F::fma(qv, qv, A::mul(qu, qu));
        const T p = A::mul(A::mul(ph.gm1, r), F::fma(-A::half, temp, A::mul(E, inv)));
        return A::add(F::sqrt(A::mul(A::mul(ph.gamma, p), inv)), F::sqrt(temp));
    }
    const T inv = A::rcp(r);
    const T qu = A::mul(ru, inv);
    const T qv = A::mul(rv, inv);
    const T temp = A::add(A::mul(qu, qu), A::mul(qv, qv));
    const T e_int = A::sub(A::mul(E, inv), A::mul(A::half, temp));
    const T p = A::mul(A::mul(ph.gm1, r), e_int);
    const T c_s = A::sqrt(A::mul(A::mul(ph.gamma, p), inv));
    const T Unorm = A::sqrt(temp);
    return A::add(c_s, Unorm);
}

// Whether the exact signal speed c_s + |u| of a new state is certainly below a threshold
// tlo, for skipping cells that cannot hold the maximum. With m2 = |rho u|^2 and
// ggm1 = gamma (gamma - 1): p = (gamma-1)(E - m2/(2 rho)) <= (gamma-1) E, so
//   c_s^2 = gamma p / rho <= ggm1 E / rho,   |u|^2 = m2 / rho^2,
// and with (a + b)^2 <= 2 (a^2 + b^2),
//   (c_s + |u|)^2 <= 2 (ggm1 E rho + m2) / rho^2.
// The speed is below tlo when 2 (ggm1 E rho + m2) < tlo^2 rho^2: no reciprocal and no
// square root. Evaluated in FP32 for either precision of the state (FP64 kernels keep
// their FP64 pipe for the update), with a relative margin of 2^-12, far above the
// roundings of the conversions, of this test and of the exact speed's own evaluation, on
// inputs in ranges where no product overflows or becomes subnormal; anything else (NaN,
// non-positive rho or E, out of range) answers false and takes the exact path.
__device__ __forceinline__ bool speed_below(float r, float E, float m2, float ggm1, float tlo2)
{
    if (!(r > 1e-6f) || !(r < 1e6f) || !(E > 1e-6f) || !(E < 1e12f) || !(m2 < 1e24f)) return false;
    return (ggm1 * E * r + m2) * (2.0f * (1.0f + 1.0f / 4096.0f)) < tlo2 * (r * r);
}
// The same test in FP64 for FP64 states (no conversions; the same bound, ranges and margin).
__device__ __forceinline__ bool speed_below(double r, double E, double m2, double ggm1, double tlo2)
{
    if (!(r > 1e-6) || !(r < 1e6) || !(E > 1e-6) || !(E < 1e12) || !(m2 < 1e24)) return false;
    return (ggm1 * E * r + m2) * (2.0 * (1.0 + 1.0 / 4096.0)) < tlo2 * (r * r);
}
// The skip test of a new 2D / 3D state in the state's own precision.
template <class T> __device__ __forceinline__ bool state_below(const Upd2<T> &o, float ggm1, float tlo2)
{
    return speed_below(o.r, o.E, o.u * o.u + o.v * o.v, (T)ggm1, (T)tlo2);
}
template <class T> struct Upd3;
template <class T> __device__ __forceinline__ bool state_below(const Upd3<T> &o, float ggm1, float tlo2)
{
    return speed_below(o.r, o.E, o.u * o.u + o.v * o.v + o.w * o.w, (T)ggm1, (T)tlo2);
}

// tlo^2 for speed_below; 0 (nothing skips) above the range the test is safe for
__device__ __forceinline__ float skip_tlo2(float tlof) { return (tlof <= 1e6f) ? tlof * tlof : 0.0f; }
// gamma (gamma - 1) in FP32 for speed_below; +inf (nothing skips) unless gamma > 1
template <class T> __host__ __device__ inline float skip_ggm1(T gamma, T gm1)
{
    const float v = (float)gamma * (float)gm1;
    return (gamma > T(1) && gm1 > T(0) && v > 0.0f) ? v : (float)(1.0 / 0.0);
}

// ---------------------------------------------------------------- 3D ----------------
// Primitive variables of a 3D cell, hydro3d/kernel.cxx:33-58:
//   temp = (u*u + v*v) + w*w
// The upwinded energy uses (un^2 + ut1^2) + ut2^2 with the per-direction order of the
// reference's calls (hydro3d/kernel.cxx:121): x (u,v,w) and y (v,u,w) give the same sum
// (the first addition commutes); z (w,v,u) is a different association, kept separately.
template <class T> struct Cell3 {
    T r, u, v, w, p, Ka, iKa, mu, mv, mw, eup_xy, eup_z;
};

template <class T, bool kF = false>
__device__ __forceinline__ Cell3<T> make_cell3_checked(T ur, T uu, T uv, T uw, T uE, const Phys<T> &ph);

// FP64 fused arithmetic: straight-line with a warp-uniform fix-up, as make_cell2 (3D 40.0 ->
// 41.2 GCell/s fused at 512^3; FP32 62.7 against 63.4 with it, so FP32 keeps the checked
// path).
template <class T, bool kF = false>
__device__ __forceinline__ Cell3<T> make_cell3(T ur, T uu, T uv, T uw, T uE, const Phys<T> &ph)
{
    if constexpr (kF && sizeof(T) == 8) {
        using A = Ar<T>;
        using F = Fu<T>;
        Cell3<T> c;
        const T inv = F::rcp_reg(ur);
        c.r = ur;
        c.u = A::mul(uu, inv);
        c.v = A::mul(uv, inv);
        c.w = A::mul(uw, inv);
        const T temp = F::fma(c.w, c.w, F::fma(c.v, c.v, A::mul(c.u, c.u)));
        c.p = A::mul(A::mul(ph.gm1, ur), F::fma(-A::half, temp, A::mul(uE, inv)));
        const T s = A::mul(A::mul(ph.gamma, c.p), c.r);
        const T y = F::rsqrt_pos(s);
        c.Ka = A::mul(ph.K, A::mul(s, y));
        c.iKa = A::mul(ph.iK, y);
        c.mu = A::mul(c.u, c.r);
        c.mv = A::mul(c.v, c.r);
        c.mw = A::mul(c.w, c.r);
        c.eup_xy = F::fma(A::mul(A::half, c.r), temp, A::mul(c.p, ph.divgamma));
        c.eup_z = c.eup_xy;
        const bool bad = !F::regular(ur) || !(s > T(0) && F::regular(s));
        if (__any_sync(__activemask(), bad)) {
            if (bad) c = make_cell3_checked<T, true>(ur, uu, uv, uw, uE, ph);
        }
        return c;
    } else {
        return make_cell3_checked<T, kF>(ur, uu, uv, uw, uE, ph);
    }
}

// The per-cell conversion with the range checks inside the chain (both arithmetics).
template <class T, bool kF>
__device__ __forceinline__ Cell3<T> make_cell3_checked(T ur, T uu, T uv, T uw, T uE, const Phys<T> &ph)
{
    using A = Ar<T>;
    Cell3<T> c;
    if constexpr (kF) {
        using F = Fu<T>;
        const T inv = F::rcp(ur);
        c.r = ur;
        c.u = A::mul(uu, inv);
        c.v = A::mul(uv, inv);
        c.w = A::mul(uw, inv);
        const T temp = F::fma(c.w, c.w, F::fma(c.v, c.v, A::mul(c.u, c.u)));
        c.p = A::mul(A::mul(ph.gm1, ur), F::fma(-A::half, temp, A::mul(uE, inv)));
        const T s = A::mul(A::mul(ph.gamma, c.p), c.r);
        if (s > T(0) && F::regular(s)) {
            const T y = F::rsqrt_pos(s);
            c.Ka = A::mul(ph.K, A::mul(s, y));
            c.iKa = A::mul(ph.iK, y);
        } else {
            c.Ka = A::mul(ph.K, A::sqrt(s));
            c.iKa = A::rcp(c.Ka);
        }
        c.mu = A::mul(c.u, c.r);
        c.mv = A::mul(c.v, c.r);
        c.mw = A::mul(c.w, c.r);
        c.eup_xy = F::fma(A::mul(A::half, c.r), temp, A::mul(c.p, ph.divgamma));
        c.eup_z = c.eup_xy;
        return c;
    }
    const T inv = A::rcp(ur);
    c.r = ur;
    c.u = A::mul(uu, inv);
    c.v = A::mul(uv, inv);
    c.w = A::mul(uw, inv);
    const T uu2 = A::mul(c.u, c.u), vv2 = A::mul(c.v, c.v), ww2 = A::mul(c.w, c.w);
    const T temp = A::add(A::add(uu2, vv2), ww2);
    const T e_int = A::sub(A::mul(uE, inv), A::mul(A::half, temp));
    c.p = A::mul(A::mul(ph.gm1, ur), e_int);
    c.Ka = A::mul(ph.K, A::sqrt(A::mul(A::mul(ph.gamma, c.p), c.r)));
    c.iKa = A::rcp(c.Ka);
    c.mu = A::mul(c.u, c.r);
    c.mv = A::mul(c.v, c.r);
    c.mw = A::mul(c.w, c.r);
    const T eint = A::mul(c.p, ph.divgamma);
    const T hr = A::mul(A::half, c.r);
    c.eup_xy = A::add(eint, A::mul(hr, temp));
    c.eup_z = A::add(eint, A::mul(hr, A::add(A::add(ww2, vv2), uu2)));
    return c;
}

// x faces: (u, v, w)
template <class T> __device__ __forceinline__ FaceIn3<T> face3_x(const Cell3<T> &c)
{
    return FaceIn3<T>{c.r, c.u, c.p, c.Ka, c.iKa, c.mu, c.mv, c.mw, c.eup_xy};
}
// y faces: (v, u, w)   hydro3d/kernel.cxx:254-256
template <class T> __device__ __forceinline__ FaceIn3<T> face3_y(const Cell3<T> &c)
{
    return FaceIn3<T>{c.r, c.v, c.p, c.Ka, c.iKa, c.mv, c.mu, c.mw, c.eup_xy};
}
// z faces: (w, v, u)   hydro3d/kernel.cxx:296-298
template <class T> __device__ __forceinline__ FaceIn3<T> face3_z(const Cell3<T> &c)
{
    return FaceIn3<T>{c.r, c.w, c.p, c.Ka, c.iKa, c.mw, c.mv, c.mu, c.eup_z};
}
template <class T> __device__ __forceinline__ FaceIn3<T> mirror3(const FaceIn3<T> &f)
{
    return FaceIn3<T>{f.r, -f.un, f.p, f.Ka, f.iKa, -f.mn, f.mt1, f.mt2, f.eup};
}

// compute_fluxes, hydro3d/kernel.cxx:79-130
template <class T, bool kF = false>
__device__ __forceinline__ Flux3<T> face_flux3(const FaceIn3<T> &L, const FaceIn3<T> &R, const Phys<T> &ph)
{
    using A = Ar<T>;
    const bool right = ph.kneg ? (R.Ka < L.Ka) : (L.Ka < R.Ka);
    const T a = right ? R.Ka : L.Ka;
    const T diva = right ? R.iKa : L.iKa;
    if constexpr (kF) {
        using F = Fu<T>;
        const T us = A::mul(A::half, F::fma(-diva, A::sub(R.p, L.p), A::add(L.un, R.un)));
        const T ps = A::mul(A::half, F::fma(-a, A::sub(R.un, L.un), A::add(L.p, R.p)));
        const bool up = us >= T(0);
        Flux3<T> F3;
        F3.r = A::mul(up ? L.r : R.r, us);
        F3.n = F::fma(up ? L.mn : R.mn, us, ps);
        F3.t1 = A::mul(up ? L.mt1 : R.mt1, us);
        F3.t2 = A::mul(up ? L.mt2 : R.mt2, us);
        F3.E = F::fma(up ? L.eup : R.eup, us, A::mul(ps, us));
        return F3;
    }
    const T us = A::mul(A::half, A::sub(A::add(L.un, R.un), A::mul(diva, A::sub(R.p, L.p))));
    const T ps = A::mul(A::half, A::sub(A::add(L.p, R.p), A::mul(a, A::sub(R.un, L.un))));
    const bool up = us >= T(0);
    const T r = up ? L.r : R.r;
    const T mn = up ? L.mn : R.mn;
    const T m1 = up ? L.mt1 : R.mt1;
    const T m2 = up ? L.mt2 : R.mt2;
    const T e = up ? L.eup : R.eup;
    Flux3<T> F;
    F.r = A::add(A::mul(r, us), T(0));
    F.n = A::add(A::mul(mn, us), ps);
    F.t1 = A::add(A::mul(m1, us), T(0));
    F.t2 = A::add(A::mul(m2, us), T(0));
    F.E = A::add(A::mul(e, us), A::mul(ps, us));
    return F;
}

template <class T> struct Upd3 {
    T r, u, v, w, E, speed;
};

// hydro3d/kernel.cxx:330-394. Slot routing per direction: x (n=u, t1=v, t2=w),
// y (n=v, t1=u, t2=w), z (n=w, t1=v, t2=u).
template <class T, bool kF = false>
__device__ __forceinline__ Upd3<T> update3(T ur, T uu, T uv, T uw, T uE, const Flux3<T> &fx_lo,
                                           const Flux3<T> &fx_hi, const Flux3<T> &fy_lo, const Flux3<T> &fy_hi,
                                           const Flux3<T> &fz_lo, const Flux3<T> &fz_hi, T DtDx, T DtDy, T DtDz,
                                           const Phys<T> &ph)
{
    using A = Ar<T>;
    if constexpr (kF) {
        using F = Fu<T>;
        Upd3<T> o;
        o.r = F::fma(DtDz, A::sub(fz_lo.r, fz_hi.r),
                     F::fma(DtDy, A::sub(fy_lo.r, fy_hi.r), F::fma(DtDx, A::sub(fx_lo.r, fx_hi.r), ur)));
        o.u = F::fma(DtDz, A::sub(fz_lo.t2, fz_hi.t2),
                     F::fma(DtDy, A::sub(fy_lo.t1, fy_hi.t1), F::fma(DtDx, A::sub(fx_lo.n, fx_hi.n), uu)));
        o.v = F::fma(DtDz, A::sub(fz_lo.t1, fz_hi.t1),
                     F::fma(DtDy, A::sub(fy_lo.n, fy_hi.n), F::fma(DtDx, A::sub(fx_lo.t1, fx_hi.t1), uv)));
        o.w = F::fma(DtDz, A::sub(fz_lo.n, fz_hi.n),
                     F::fma(DtDy, A::sub(fy_lo.t2, fy_hi.t2), F::fma(DtDx, A::sub(fx_lo.t2, fx_hi.t2), uw)));
        o.E = F::fma(DtDz, A::sub(fz_lo.E, fz_hi.E),
                     F::fma(DtDy, A::sub(fy_lo.E, fy_hi.E), F::fma(DtDx, A::sub(fx_lo.E, fx_hi.E), uE)));
        o.speed = T(0);
        return o;
    }
    const T x_r = A::mul(DtDx, A::sub(fx_lo.r, fx_hi.r));
    const T x_u = A::mul(DtDx, A::sub(fx_lo.n, fx_hi.n));
    const T x_v = A::mul(DtDx, A::sub(fx_lo.t1, fx_hi.t1));
    const T x_w = A::mul(DtDx, A::sub(fx_lo.t2, fx_hi.t2));
    const T x_E = A::mul(DtDx, A::sub(fx_lo.E, fx_hi.E));
    const T y_r = A::mul(DtDy, A::sub(fy_lo.r, fy_hi.r));
    const T y_u = A::mul(DtDy, A::sub(fy_lo.t1, fy_hi.t1));
    const T y_v = A::mul(DtDy, A::sub(fy_lo.n, fy_hi.n));
    const T y_w = A::mul(DtDy, A::sub(fy_lo.t2, fy_hi.t2));
    const T y_E = A::mul(DtDy, A::sub(fy_lo.E, fy_hi.E));
    const T z_r = A::mul(DtDz, A::sub(fz_lo.r, fz_hi.r));
    const T z_u = A::mul(DtDz, A::sub(fz_lo.t2, fz_hi.t2));
    const T z_v = A::mul(DtDz, A::sub(fz_lo.t1, fz_hi.t1));
    const T z_w = A::mul(DtDz, A::sub(fz_lo.n, fz_hi.n));
    const T z_E = A::mul(DtDz, A::sub(fz_lo.E, fz_hi.E));
    Upd3<T> o;
    o.r = A::add(A::add(A::add(ur, x_r), y_r), z_r);
    o.u = A::add(A::add(A::add(uu, x_u), y_u), z_u);
    o.v = A::add(A::add(A::add(uv, x_v), y_v), z_v);
    o.w = A::add(A::add(A::add(uw, x_w), y_w), z_w);
    o.E = A::add(A::add(A::add(uE, x_E), y_E), z_E);
    o.speed = T(0);
    return o;
}

// Signal speed c_s + |u| of a 3D state, hydro3d/kernel.cxx:367-390.
template <class T, bool kF = false>
__device__ __forceinline__ T speed3(T r, T ru, T rv, T rw, T E, const Phys<T> &ph)
{
    using A = Ar<T>;
    if constexpr (kF) {
        using F = Fu<T>;
        const T inv = F::rcp(r);
        const T qu = A::mul(ru, inv), qv = A::mul(rv, inv), qw = A::mul(rw, inv);
        const T temp = F::fma(qw, qw, F::fma(qv, qv, A::mul(qu, qu)));
        const T p = A::mul(A::mul(ph.gm1, r), F::fma(-A::half, temp, A::mul(E, inv)));
        return A::add(F::sqrt(A::mul(A::mul(ph.gamma, p), inv)), F::sqrt(temp));
    }
    const T inv = A::rcp(r);
    const T qu = A::mul(ru, inv), qv = A::mul(rv, inv), qw = A::mul(rw, inv);
    const T temp = A::add(A::add(A::mul(qu, qu), A::mul(qv, qv)), A::mul(qw, qw));
    const T e_int = A::sub(A::mul(E, inv), A::mul(A::half, temp));
    const T p = A::mul(A::mul(ph.gm1, r), e_int);
    const T c_s = A::sqrt(A::mul(A::mul(ph.gamma, p), inv));
    const T Unorm = A::sqrt(temp);
    return A::add(c_s, Unorm);
}

} // namespace hydro
