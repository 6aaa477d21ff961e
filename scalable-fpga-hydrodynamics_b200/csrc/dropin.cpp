// The reference's `launcher` symbol for one (dimension, precision) variant, compiled
// four times into libhydro2d.so, libhydro2d_float.so, libhydro3d.so and
// libhydro3d_float.so. The reference's host program links one of them in place of its
// SYCL kernel object (hydro2d/kernel.hpp:63-68, hydro3d/kernel.hpp:64-69).
#include "../../include/hydro_b200.h"

#ifdef USE_FLOAT
#define DATATYPE float
#define SUF(name) name##_f32
#else
#define DATATYPE double
#define SUF(name) name##_f64
#endif

extern "C" {
#if HYDRO_DIM == 2
double launcher(const DATATYPE *d_rhoE, const DATATYPE *d_uv, DATATYPE *d_rhoE_next, DATATYPE *d_uv_next,
                DATATYPE *Dt_next, const DATATYPE C_min, const DATATYPE gamma, const DATATYPE gamma_minus_one,
                const DATATYPE divgamma, const DATATYPE K, const size_t NB_X, const size_t NB_Y,
                const DATATYPE *DtDx, const DATATYPE *DtDy, hydro_queue_t queue)
{
    return SUF(hydro2d_launcher)(d_rhoE, d_uv, d_rhoE_next, d_uv_next, Dt_next, C_min, gamma, gamma_minus_one,
                                 divgamma, K, NB_X, NB_Y, DtDx, DtDy, queue);
}
#else
double launcher(const DATATYPE *d_rhoE, const DATATYPE *d_uvw, DATATYPE *d_rhoE_next, DATATYPE *d_uvw_next,
                DATATYPE *Dt_next, const DATATYPE C_min, const DATATYPE gamma, const DATATYPE gamma_minus_one,
                const DATATYPE divgamma, const DATATYPE K, const size_t NB_X, const size_t NB_Y, const size_t NB_Z,
                const DATATYPE *DtDx, const DATATYPE *DtDy, const DATATYPE *DtDz, hydro_queue_t queue)
{
    return SUF(hydro3d_launcher)(d_rhoE, d_uvw, d_rhoE_next, d_uvw_next, Dt_next, C_min, gamma, gamma_minus_one,
                                 divgamma, K, NB_X, NB_Y, NB_Z, DtDx, DtDy, DtDz, queue);
}
#endif
}
