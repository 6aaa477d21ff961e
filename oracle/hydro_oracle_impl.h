/*
 * Oracle (test infrastructure only): a direct-indexed CPU restatement of the
 * reference's first-order finite-volume update, host time-step chain and blast
 * initial condition. Included twice by hydro_oracle.c, once per precision, with
 *   T     the arithmetic type (the reference's DATATYPE, hydro2d/kernel.hpp:9-39)
 *   SUF   the symbol suffix (_f64 / _f32)
 *   TSQRT the square root for T (the reference's SQRT macro)
 *   L(x)  the literal for T (the reference's LITERAL macro)
 * It must be compiled with -ffp-contract=off: every expression below keeps the
 * reference's operation order and association, so that with IEEE arithmetic and no
 * contraction the results are bit-for-bit those of the reference kernel.
 *
 * What differs from the reference, on purpose and without changing any result:
 *  - cells are addressed directly instead of through the FPGA line buffer
 *    (hydro2d/kernel.cxx:142-159); the buffer is exact whenever the reference's
 *    cache-size check (hydro2d/main.cxx:503-516) passes;
 *  - at a reflective wall the mirrored state is selected directly, where the reference
 *    first converts the zero ghost cell (1/0 -> inf/NaN) and then discards it with a
 *    select (hydro2d/kernel.cxx:219-225); the selected values are identical.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)

/* std::max(a, b) as the reference calls it (MMAX): returns a unless a < b */
static inline T FN(smax)(T a, T b) { return (a < b) ? b : a; }
/* std::min(a, b): returns a unless b < a */
static inline T FN(smin)(T a, T b) { return (b < a) ? b : a; }

/* hydro2d/kernel.cxx:31-53 (and :5-29, the same arithmetic) */
static inline void FN(prim2)(T ur, T uu, T uv, T uE, T gm1, T *qr, T *qu, T *qv, T *qp)
{
    T inv = L(1.0) / ur;
    *qr = ur;
    *qu = uu * inv;
    *qv = uv * inv;
    T temp = *qu * *qu + *qv * *qv;
    T e_int = uE * inv - L(0.5) * temp;
    *qp = gm1 * ur * e_int;
}

/* hydro2d/kernel.cxx:74-118. Argument order is (rho, normal velocity, tangential
 * velocity, p) for the left then the right state. */
static inline void FN(flux2)(T rl, T ul, T vl, T pl, T rr, T urr, T vr, T pr, T K, T gamma, T divgamma, T *Fr,
                             T *Fu, T *Fv, T *FE)
{
    T a_left = TSQRT(gamma * pl * rl);
    T a_right = TSQRT(gamma * pr * rr);
    T a = K * FN(smax)(a_left, a_right);
    const T diva = L(1.0) / a;
    T us = L(0.5) * ((ul + urr) - diva * (pr - pl));
    T ps = L(0.5) * ((pl + pr) - a * (urr - ul));
    const int up = us >= L(0.0);
    T r = up ? rl : rr;
    T u = up ? ul : urr;
    T v = up ? vl : vr;
    T p = up ? pl : pr;
    T Ur = r;
    T Uu = u * r;
    T Uv = v * r;
    T UE = p * divgamma + L(0.5) * r * (u * u + v * v);
    *Fr = Ur * us + L(0.0);
    *Fu = Uu * us + ps;
    *Fv = Uv * us + L(0.0);
    *FE = UE * us + ps * us;
}

/* One time step of the 2D kernel, hydro2d/kernel.cxx:132-319. State arrays hold
 * (NB_X+2)*(NB_Y+2) cells as interleaved pairs: rhoE[2c]=rho, rhoE[2c+1]=E,
 * uv[2c]=rho*u, uv[2c+1]=rho*v, with c = i*(NB_Y+2)+j. The X ghost rows i=0 and
 * i=NB_X+1 are read from the input arrays, as the reference kernel does; only
 * interior cells of the outputs are written. */
void FN(oracle2d_step)(const T *rhoE, const T *uv, T *rhoE_next, T *uv_next, T *Dt_next, T C_min, T gamma, T gm1,
                       T divgamma, T K, size_t NB_X, size_t NB_Y, T DtDx, T DtDy)
{
    const size_t ys = NB_Y + 2;
    T max_speed = L(0.0);
    for (size_t i = 1; i <= NB_X; ++i) {
        for (size_t j = 1; j <= NB_Y; ++j) {
            const size_t c = i * ys + j;
            const T U_r = rhoE[2 * c], U_E = rhoE[2 * c + 1], U_u = uv[2 * c], U_v = uv[2 * c + 1];
            T qr, qu, qv, qp;
            FN(prim2)(U_r, U_u, U_v, U_E, gm1, &qr, &qu, &qv, &qp);

            T fx1r, fx1u, fx1v, fx1E, fx2r, fx2u, fx2v, fx2E;
            T fy1r, fy1u, fy1v, fy1E, fy2r, fy2u, fy2v, fy2E;
            {
                const size_t n = c - ys;
                T lr, lu, lv, lp;
                FN(prim2)(rhoE[2 * n], uv[2 * n], uv[2 * n + 1], rhoE[2 * n + 1], gm1, &lr, &lu, &lv, &lp);
                FN(flux2)(lr, lu, lv, lp, qr, qu, qv, qp, K, gamma, divgamma, &fx1r, &fx1u, &fx1v, &fx1E);
            }
            {
                const size_t n = c + ys;
                T rr, ru, rv, rp;
                FN(prim2)(rhoE[2 * n], uv[2 * n], uv[2 * n + 1], rhoE[2 * n + 1], gm1, &rr, &ru, &rv, &rp);
                FN(flux2)(qr, qu, qv, qp, rr, ru, rv, rp, K, gamma, divgamma, &fx2r, &fx2u, &fx2v, &fx2E);
            }
            {
                T lr, lu, lv, lp;
                if (j == 1) {
                    lr = qr; lu = qu; lv = -qv; lp = qp;
                } else {
                    const size_t n = c - 1;
                    FN(prim2)(rhoE[2 * n], uv[2 * n], uv[2 * n + 1], rhoE[2 * n + 1], gm1, &lr, &lu, &lv, &lp);
                }
                FN(flux2)(lr, lv, lu, lp, qr, qv, qu, qp, K, gamma, divgamma, &fy1r, &fy1u, &fy1v, &fy1E);
            }
            {
                T rr, ru, rv, rp;
                if (j == NB_Y) {
                    rr = qr; ru = qu; rv = -qv; rp = qp;
                } else {
                    const size_t n = c + 1;
                    FN(prim2)(rhoE[2 * n], uv[2 * n], uv[2 * n + 1], rhoE[2 * n + 1], gm1, &rr, &ru, &rv, &rp);
                }
                FN(flux2)(qr, qv, qu, qp, rr, rv, ru, rp, K, gamma, divgamma, &fy2r, &fy2u, &fy2v, &fy2E);
            }

            /* hydro2d/kernel.cxx:259-273: the y fluxes come back with the velocity
             * slots swapped */
            const T x_r = DtDx * (fx1r - fx2r), x_u = DtDx * (fx1u - fx2u);
            const T x_v = DtDx * (fx1v - fx2v), x_E = DtDx * (fx1E - fx2E);
            const T y_r = DtDy * (fy1r - fy2r), y_u = DtDy * (fy1v - fy2v);
            const T y_v = DtDy * (fy1u - fy2u), y_E = DtDy * (fy1E - fy2E);
            const T nr = U_r + x_r + y_r;
            const T nu = U_u + x_u + y_u;
            const T nv = U_v + x_v + y_v;
            const T nE = U_E + x_E + y_E;
            rhoE_next[2 * c] = nr;
            uv_next[2 * c] = nu;
            uv_next[2 * c + 1] = nv;
            rhoE_next[2 * c + 1] = nE;

            /* hydro2d/kernel.cxx:281-314 */
            const T inv = L(1.0) / nr;
            const T u = nu * inv, v = nv * inv;
            const T temp = u * u + v * v;
            const T e_int = nE * inv - L(0.5) * temp;
            const T p = gm1 * nr * e_int;
            const T c_s = TSQRT(gamma * p * inv);
            const T Unorm = TSQRT(temp);
            const T speed = c_s + Unorm;
            max_speed = FN(smax)(speed, max_speed);
        }
    }
    *Dt_next = C_min / max_speed;
}

/* hydro3d/kernel.cxx:33-58 */
static inline void FN(prim3)(T ur, T uu, T uv, T uw, T uE, T gm1, T *qr, T *qu, T *qv, T *qw, T *qp)
{
    T inv = L(1.0) / ur;
    *qr = ur;
    *qu = uu * inv;
    *qv = uv * inv;
    *qw = uw * inv;
    T temp = *qu * *qu + *qv * *qv + *qw * *qw;
    T e_int = uE * inv - L(0.5) * temp;
    *qp = gm1 * ur * e_int;
}

/* hydro3d/kernel.cxx:79-130. Order (rho, normal, tangential 1, tangential 2, p). */
static inline void FN(flux3)(T rl, T al, T bl, T cl, T pl, T rr, T ar, T br, T cr, T pr, T K, T gamma, T divgamma,
                             T *Fr, T *Fa, T *Fb, T *Fc, T *FE)
{
    T a_left = TSQRT(gamma * pl * rl);
    T a_right = TSQRT(gamma * pr * rr);
    T a = K * FN(smax)(a_left, a_right);
    const T diva = L(1.0) / a;
    T us = L(0.5) * ((al + ar) - diva * (pr - pl));
    T ps = L(0.5) * ((pl + pr) - a * (ar - al));
    const int up = us >= L(0.0);
    T r = up ? rl : rr;
    T ua = up ? al : ar;
    T ub = up ? bl : br;
    T uc = up ? cl : cr;
    T p = up ? pl : pr;
    T Ur = r;
    T Ua = ua * r;
    T Ub = ub * r;
    T Uc = uc * r;
    T eint = p * divgamma;
    T ekin = L(0.5) * r * (ua * ua + ub * ub + uc * uc);
    T UE = eint + ekin;
    *Fr = Ur * us + L(0.0);
    *Fa = Ua * us + ps;
    *Fb = Ub * us + L(0.0);
    *Fc = Uc * us + L(0.0);
    *FE = UE * us + ps * us;
}

#define PRIM3_AT(n, r, u, v, w, p)                                                                                 \
    FN(prim3)(rhoE[2 * (n)], uvw[3 * (n)], uvw[3 * (n) + 1], uvw[3 * (n) + 2], rhoE[2 * (n) + 1], gm1, &r, &u, &v, \
              &w, &p)

/* One time step of the 3D kernel, hydro3d/kernel.cxx:145-407. rhoE holds (rho, E)
 * pairs and uvw (rho*u, rho*v, rho*w) triples; c = i*(NB_Y+2)*(NB_Z+2) + j*(NB_Z+2) + k. */
void FN(oracle3d_step)(const T *rhoE, const T *uvw, T *rhoE_next, T *uvw_next, T *Dt_next, T C_min, T gamma, T gm1,
                       T divgamma, T K, size_t NB_X, size_t NB_Y, size_t NB_Z, T DtDx, T DtDy, T DtDz)
{
    const size_t zs = NB_Z + 2;
    const size_t zy = (NB_Y + 2) * zs;
    T max_speed = L(0.0);
    for (size_t i = 1; i <= NB_X; ++i) {
        for (size_t j = 1; j <= NB_Y; ++j) {
            for (size_t k = 1; k <= NB_Z; ++k) {
                const size_t c = i * zy + j * zs + k;
                const T U_r = rhoE[2 * c], U_E = rhoE[2 * c + 1];
                const T U_u = uvw[3 * c], U_v = uvw[3 * c + 1], U_w = uvw[3 * c + 2];
                T qr, qu, qv, qw, qp;
                FN(prim3)(U_r, U_u, U_v, U_w, U_E, gm1, &qr, &qu, &qv, &qw, &qp);

                T fx1[5], fx2[5], fy1[5], fy2[5], fz1[5], fz2[5];
                {
                    T r, u, v, w, p;
                    PRIM3_AT(c - zy, r, u, v, w, p);
                    FN(flux3)(r, u, v, w, p, qr, qu, qv, qw, qp, K, gamma, divgamma, &fx1[0], &fx1[1], &fx1[2],
                              &fx1[3], &fx1[4]);
                }
                {
                    T r, u, v, w, p;
                    PRIM3_AT(c + zy, r, u, v, w, p);
                    FN(flux3)(qr, qu, qv, qw, qp, r, u, v, w, p, K, gamma, divgamma, &fx2[0], &fx2[1], &fx2[2],
                              &fx2[3], &fx2[4]);
                }
                {
                    T r, u, v, w, p;
                    if (j == 1) { r = qr; u = qu; v = -qv; w = qw; p = qp; }
                    else PRIM3_AT(c - zs, r, u, v, w, p);
                    FN(flux3)(r, v, u, w, p, qr, qv, qu, qw, qp, K, gamma, divgamma, &fy1[0], &fy1[1], &fy1[2],
                              &fy1[3], &fy1[4]);
                }
                {
                    T r, u, v, w, p;
                    if (j == NB_Y) { r = qr; u = qu; v = -qv; w = qw; p = qp; }
                    else PRIM3_AT(c + zs, r, u, v, w, p);
                    FN(flux3)(qr, qv, qu, qw, qp, r, v, u, w, p, K, gamma, divgamma, &fy2[0], &fy2[1], &fy2[2],
                              &fy2[3], &fy2[4]);
                }
                {
                    T r, u, v, w, p;
                    if (k == 1) { r = qr; u = qu; v = qv; w = -qw; p = qp; }
                    else PRIM3_AT(c - 1, r, u, v, w, p);
                    FN(flux3)(r, w, v, u, p, qr, qw, qv, qu, qp, K, gamma, divgamma, &fz1[0], &fz1[1], &fz1[2],
                              &fz1[3], &fz1[4]);
                }
                {
                    T r, u, v, w, p;
                    if (k == NB_Z) { r = qr; u = qu; v = qv; w = -qw; p = qp; }
                    else PRIM3_AT(c + 1, r, u, v, w, p);
                    FN(flux3)(qr, qw, qv, qu, qp, r, w, v, u, p, K, gamma, divgamma, &fz2[0], &fz2[1], &fz2[2],
                              &fz2[3], &fz2[4]);
                }

                /* hydro3d/kernel.cxx:330-352 (component slots permuted per direction) */
                const T x_r = DtDx * (fx1[0] - fx2[0]), x_u = DtDx * (fx1[1] - fx2[1]);
                const T x_v = DtDx * (fx1[2] - fx2[2]), x_w = DtDx * (fx1[3] - fx2[3]);
                const T x_E = DtDx * (fx1[4] - fx2[4]);
                const T y_r = DtDy * (fy1[0] - fy2[0]), y_u = DtDy * (fy1[2] - fy2[2]);
                const T y_v = DtDy * (fy1[1] - fy2[1]), y_w = DtDy * (fy1[3] - fy2[3]);
                const T y_E = DtDy * (fy1[4] - fy2[4]);
                const T z_r = DtDz * (fz1[0] - fz2[0]), z_u = DtDz * (fz1[3] - fz2[3]);
                const T z_v = DtDz * (fz1[2] - fz2[2]), z_w = DtDz * (fz1[1] - fz2[1]);
                const T z_E = DtDz * (fz1[4] - fz2[4]);
                const T nr = U_r + x_r + y_r + z_r;
                const T nu = U_u + x_u + y_u + z_u;
                const T nv = U_v + x_v + y_v + z_v;
                const T nw = U_w + x_w + y_w + z_w;
                const T nE = U_E + x_E + y_E + z_E;
                rhoE_next[2 * c] = nr;
                uvw_next[3 * c] = nu;
                uvw_next[3 * c + 1] = nv;
                uvw_next[3 * c + 2] = nw;
                rhoE_next[2 * c + 1] = nE;

                /* hydro3d/kernel.cxx:361-394 */
                const T inv = L(1.0) / nr;
                const T u = nu * inv, v = nv * inv, w = nw * inv;
                const T temp = u * u + v * v + w * w;
                const T e_int = nE * inv - L(0.5) * temp;
                const T p = gm1 * nr * e_int;
                const T c_s = TSQRT(gamma * p * inv);
                const T Unorm = TSQRT(temp);
                const T speed = c_s + Unorm;
                max_speed = FN(smax)(speed, max_speed);
            }
        }
    }
    *Dt_next = C_min / max_speed;
}
#undef PRIM3_AT

/* One cell of the blast initial condition, hydro2d/main.cxx:296-335 (3D:
 * hydro3d/main.cxx:314-358 with dz != 0): inside/outside by the double distance to the
 * centre, E = p/(gamma-1), zero momentum; returns C_min/(c_s+|u|) of the cell. */
static inline T FN(ic_cell)(double dx, double dy, double dz, int is3d, double radius, T u_in, T u_out, T p_in,
                            T p_out, T C_min, T gamma, T gm1, T *U_r, T *U_p)
{
    const double d = is3d ? sqrt(dx * dx + dy * dy + dz * dz) : sqrt(dx * dx + dy * dy);
    *U_r = (d <= radius ? u_in : u_out);
    *U_p = (d <= radius ? p_in : p_out) / gm1;
    const T zero = L(0.0);
    const T inv = L(1.0) / *U_r;
    const T qu = zero * inv, qv = zero * inv, qw = zero * inv;
    const T temp = is3d ? qu * qu + qv * qv + qw * qw : qu * qu + qv * qv;
    const T e_int = *U_p * inv - L(0.5) * temp;
    const T qp = gm1 * *U_r * e_int;
    const T c_s = TSQRT(gamma * qp * inv);
    const T Unorm = TSQRT(temp);
    return C_min / (c_s + Unorm);
}

/* Blast initial condition and first time step for the whole domain as one
 * subdomain, hydro2d/main.cxx:280-338 (base_i = base_j = 0). Writes the interior
 * of rhoE/uv (ghosts untouched) and returns min over cells of C_min/(c_s+|u|). */
T FN(oracle2d_init)(T *rhoE, T *uv, size_t NB_X, size_t NB_Y, T u_in, T u_out, T p_in, T p_out, T C_min, T gamma)
{
    T min_Dt = L(1e20);
    const T gm1 = gamma - L(1.0);
    const double cx = (double)(NB_X + 1) / 2.0;
    const double cy = (double)(NB_Y + 1) / 2.0;
    const double radius = (cy < cx ? cy : cx) / 3;
    const size_t ys = NB_Y + 2;
    for (size_t i = 1; i <= NB_X; ++i) {
        for (size_t j = 1; j <= NB_Y; ++j) {
            const size_t c = i * ys + j;
            T U_r, U_p;
            const T local = FN(ic_cell)((double)i - cx, (double)j - cy, 0.0, 0, radius, u_in, u_out, p_in, p_out,
                                        C_min, gamma, gm1, &U_r, &U_p);
            rhoE[2 * c] = U_r;
            rhoE[2 * c + 1] = U_p;
            uv[2 * c] = L(0.0);
            uv[2 * c + 1] = L(0.0);
            min_Dt = FN(smin)(min_Dt, local);
        }
    }
    return min_Dt;
}

/* hydro3d/main.cxx:296-363 for one subdomain covering the domain */
T FN(oracle3d_init)(T *rhoE, T *uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, T u_in, T u_out, T p_in, T p_out,
                    T C_min, T gamma)
{
    T min_Dt = L(1e20);
    const T gm1 = gamma - L(1.0);
    const double cx = (double)(NB_X + 1) / 2.0;
    const double cy = (double)(NB_Y + 1) / 2.0;
    const double cz = (double)(NB_Z + 1) / 2.0;
    double m = cx;
    if (cy < m) m = cy;
    if (cz < m) m = cz;
    const double radius = m / 3;
    const size_t zs = NB_Z + 2, zy = (NB_Y + 2) * zs;
    for (size_t i = 1; i <= NB_X; ++i) {
        for (size_t j = 1; j <= NB_Y; ++j) {
            for (size_t k = 1; k <= NB_Z; ++k) {
                const size_t c = i * zy + j * zs + k;
                T U_r, U_p;
                const T local = FN(ic_cell)((double)i - cx, (double)j - cy, (double)k - cz, 1, radius, u_in, u_out,
                                            p_in, p_out, C_min, gamma, gm1, &U_r, &U_p);
                rhoE[2 * c] = U_r;
                rhoE[2 * c + 1] = U_p;
                uvw[3 * c] = L(0.0);
                uvw[3 * c + 1] = L(0.0);
                uvw[3 * c + 2] = L(0.0);
                min_Dt = FN(smin)(min_Dt, local);
            }
        }
    }
    return min_Dt;
}

/* The blast IC's initial total mass (row-major Neumaier in long double, as
 * hydro2d/main.cxx:237-265 sums it) and first Dt, computed cell by cell without
 * storing the grid (NB_Z = 0 for 2D). */
double FN(oracle_blast_stats)(size_t NB_X, size_t NB_Y, size_t NB_Z, T u_in, T u_out, T p_in, T p_out, T C_min,
                              T gamma, T *min_dt)
{
    const int is3d = NB_Z > 0;
    const T gm1 = gamma - L(1.0);
    const double cx = (double)(NB_X + 1) / 2.0, cy = (double)(NB_Y + 1) / 2.0, cz = (double)(NB_Z + 1) / 2.0;
    double m = cy < cx ? cy : cx;
    if (is3d && cz < m) m = cz;
    const double radius = m / 3;
    long double total = 0.0L, comp = 0.0L;
    T mn = L(1e20);
    const size_t k1 = is3d ? NB_Z : 1;
    for (size_t i = 1; i <= NB_X; ++i)
        for (size_t j = 1; j <= NB_Y; ++j)
            for (size_t k = 1; k <= k1; ++k) {
                T U_r, U_p;
                const T local = FN(ic_cell)((double)i - cx, (double)j - cy, is3d ? (double)k - cz : 0.0, is3d,
                                            radius, u_in, u_out, p_in, p_out, C_min, gamma, gm1, &U_r, &U_p);
                mn = FN(smin)(mn, local);
                long double var = (long double)U_r;
                long double t = total + var;
                if (fabsl(total) >= var) comp += (total - t) + var;
                else comp += (var - t) + total;
                total = t;
            }
    *min_dt = mn;
    return (double)(total + comp);
}

/* Periodic X ghost rows, hydro2d/main.cxx:349-378 (the 2D "row" is one X index). */
void FN(oracle2d_ghost_x)(T *rhoE, T *uv, size_t NB_X, size_t NB_Y)
{
    const size_t ys = NB_Y + 2;
    memcpy(&rhoE[0], &rhoE[2 * NB_X * ys], 2 * ys * sizeof(T));
    memcpy(&uv[0], &uv[2 * NB_X * ys], 2 * ys * sizeof(T));
    memcpy(&rhoE[2 * (NB_X + 1) * ys], &rhoE[2 * ys], 2 * ys * sizeof(T));
    memcpy(&uv[2 * (NB_X + 1) * ys], &uv[2 * ys], 2 * ys * sizeof(T));
}

/* hydro3d/main.cxx:374-403: periodic X ghost planes */
void FN(oracle3d_ghost_x)(T *rhoE, T *uvw, size_t NB_X, size_t NB_Y, size_t NB_Z)
{
    const size_t zy = (NB_Y + 2) * (NB_Z + 2);
    memcpy(&rhoE[0], &rhoE[2 * NB_X * zy], 2 * zy * sizeof(T));
    memcpy(&uvw[0], &uvw[3 * NB_X * zy], 3 * zy * sizeof(T));
    memcpy(&rhoE[2 * (NB_X + 1) * zy], &rhoE[2 * zy], 2 * zy * sizeof(T));
    memcpy(&uvw[3 * (NB_X + 1) * zy], &uvw[3 * zy], 3 * zy * sizeof(T));
}

/* Interior density sum in long double with Neumaier compensation,
 * hydro2d/main.cxx:237-265 / hydro3d/main.cxx:249-281 (ncell_inner = NB_Z+2 for 3D,
 * 1 with NB_Z = 0 for 2D). */
double FN(oracle_mass)(const T *rhoE, size_t NB_X, size_t NB_Y, size_t NB_Z)
{
    long double total = 0.0L, comp = 0.0L;
    const int is3d = NB_Z > 0;
    const size_t zs = is3d ? NB_Z + 2 : 1;
    const size_t zy = (NB_Y + 2) * zs;
    const size_t k0 = is3d ? 1 : 0, k1 = is3d ? NB_Z : 0;
    for (size_t i = 1; i <= NB_X; ++i)
        for (size_t j = 1; j <= NB_Y; ++j)
            for (size_t k = k0; k <= k1; ++k) {
                const size_t c = i * zy + j * zs + k;
                long double var = (long double)rhoE[2 * c];
                long double t = total + var;
                if (fabsl(total) >= var) comp += (total - t) + var;
                else comp += (var - t) + total;
                total = t;
            }
    return (double)(total + comp);
}

/* The reference host loop for one rank and one subdomain, hydro2d/main.cxx:595-836
 * (3D: hydro3d/main.cxx:642-900 with NB_Z > 0). Runs the blast from its initial
 * condition and records, per iteration, the printed t and the newly reduced Dt
 * (quirk kept: t advances by the new Dt, main.cxx:813-814). Final state is left in
 * rhoE/uvx (each of (NB_X+2)(NB_Y+2)[(NB_Z+2)] cells, zero-initialised by the
 * caller). Returns the number of iterations run. */
size_t FN(oracle_run)(size_t NB_X, size_t NB_Y, size_t NB_Z, double max_t, size_t max_it, T *rhoE, T *uvx,
                      double *t_log, T *dt_log, T *first_dt, double *mass0, double *mass1)
{
    const int is3d = NB_Z > 0;
    const size_t nv = is3d ? 3 : 2;
    const size_t ncell = (NB_X + 2) * (NB_Y + 2) * (is3d ? NB_Z + 2 : 1);
    const T DX = L(1.0) / (T)(NB_X + 1);
    const T DY = L(1.0) / (T)(NB_Y + 1);
    const T DZ = is3d ? L(1.0) / (T)(NB_Z + 1) : L(0.0);
    T min_spacing = FN(smin)(DX, DY);
    if (is3d) min_spacing = FN(smin)(min_spacing, DZ);
    const T C = is3d ? L(0.4) : L(0.5);
    const T gamma = L(1.4), K = L(1.1);
    const T gm1 = gamma - L(1.0);
    const T divgamma = L(1.0) / gm1;
    const T C_min = C * min_spacing;

    T *rhoE_n = (T *)calloc(2 * ncell, sizeof(T));
    T *uvx_n = (T *)calloc(nv * ncell, sizeof(T));
    if (!rhoE_n || !uvx_n) { free(rhoE_n); free(uvx_n); return (size_t)-1; }

    const T min_Dt = is3d ? FN(oracle3d_init)(rhoE, uvx, NB_X, NB_Y, NB_Z, L(1.0), L(1.2), L(10.0), L(0.1), C_min,
                                              gamma)
                          : FN(oracle2d_init)(rhoE, uvx, NB_X, NB_Y, L(1.0), L(1.2), L(10.0), L(0.1), C_min, gamma);
    /* first_Dt starts at 1e20 and takes the min with each subdomain's value (main.cxx:618,654) */
    T Dt_local = FN(smin)(L(1e20), min_Dt);
    if (first_dt) *first_dt = Dt_local;
    if (mass0) *mass0 = FN(oracle_mass)(rhoE, NB_X, NB_Y, NB_Z);

    double t = 0.0;
    size_t it = 0;
    T *cur_r = rhoE, *cur_x = uvx, *nxt_r = rhoE_n, *nxt_x = uvx_n;
    while (t < max_t && it < max_it) {
        if (is3d) FN(oracle3d_ghost_x)(cur_r, cur_x, NB_X, NB_Y, NB_Z);
        else FN(oracle2d_ghost_x)(cur_r, cur_x, NB_X, NB_Y);
        const T DtDx = Dt_local / DX;
        const T DtDy = Dt_local / DY;
        const T DtDz = is3d ? Dt_local / DZ : L(0.0);
        T dtn;
        if (is3d)
            FN(oracle3d_step)(cur_r, cur_x, nxt_r, nxt_x, &dtn, C_min, gamma, gm1, divgamma, K, NB_X, NB_Y, NB_Z,
                              DtDx, DtDy, DtDz);
        else
            FN(oracle2d_step)(cur_r, cur_x, nxt_r, nxt_x, &dtn, C_min, gamma, gm1, divgamma, K, NB_X, NB_Y, DtDx,
                              DtDy);
        T *s = cur_r; cur_r = nxt_r; nxt_r = s;
        s = cur_x; cur_x = nxt_x; nxt_x = s;
        Dt_local = FN(smin)(L(1e20), dtn);
        if (t_log) t_log[it] = t;
        if (dt_log) dt_log[it] = Dt_local;
        ++it;
        t += Dt_local;
    }
    if (cur_r != rhoE) {
        memcpy(rhoE, cur_r, 2 * ncell * sizeof(T));
        memcpy(uvx, cur_x, nv * ncell * sizeof(T));
    }
    if (mass1) *mass1 = FN(oracle_mass)(rhoE, NB_X, NB_Y, NB_Z);
    free(rhoE_n);
    free(uvx_n);
    return it;
}

#undef FN
#undef CAT
#undef CAT2
