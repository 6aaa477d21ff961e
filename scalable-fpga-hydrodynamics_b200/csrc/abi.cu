// extern "C" entry points declared in include/hydro_b200.h.
#include <algorithm>
#include <stdio.h>
#include <time.h>

#include "../../include/hydro_b200.h"
#include "hydro_host.h"

using namespace hydro;

namespace {

double now_us()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e6 + ts.tv_nsec / 1e3;
}

// Select the queue's device for the duration of a call.
struct DeviceScope {
    int prev = -1;
    bool ok = true;
    explicit DeviceScope(int dev)
    {
        if (dev < 0) return;
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
            set_error(kErrCuda, "cudaSetDevice(%d) failed", dev);
            ok = false;
        }
    }
    ~DeviceScope()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// The reference never reports a status; the drop-in prints each distinct failure once
// per call to stderr and returns a negative time for hard errors only.
double finish_launcher(int rc, double t0, const char *what)
{
    const double dt = now_us() - t0;
    if (rc == kOk) return dt;
    fprintf(stderr, "[hydro_b200] %s: %s\n", what, last_error_string());
    if (rc == kErrPhys) return dt; // outputs were written, as the reference would
    return -1.0;
}

template <class T> Phys<T> phys(T C_min, T gamma, T gm1, T divgamma, T K)
{
    return Phys<T>::make(C_min, gamma, gm1, divgamma, K);
}

// The arithmetic a step runs in, from the HYDRO_ARITH_* bits of the flags.
bool fused_of(int flags)
{
    if (flags & HYDRO_ARITH_STRICT) return false;
    return (flags & HYDRO_ARITH_FUSED) != 0;
}

void fill(hydro_step_info_t *out, const StepInfo &in)
{
    if (!out) return;
    out->mass = in.mass;
    out->max_speed = in.max_speed;
    out->err = in.err;
    out->kernel = in.kernel;
}

// Fused-mode reciprocal and square root of each value (diagnostics: the tests compare them
// with the correctly rounded values).
template <class T> __global__ void fused_math_kernel(const T *x, long long n, T *rcp, T *sq)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        rcp[i] = Fu<T>::rcp(x[i]);
        sq[i] = Fu<T>::sqrt(x[i]);
    }
}

template <class T> int fused_math(const T *x, size_t n, T *rcp, T *sq, void *stream)
{
    if (!x || !rcp || !sq) {
        set_error(kErrArg, "hydro_fused_math: null argument");
        return kErrArg;
    }
    if (n == 0) return kOk;
    const cudaStream_t st = (cudaStream_t)stream;
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)device_sms() * 8);
    fused_math_kernel<T><<<blocks, 256, 0, st>>>(x, (long long)n, rcp, sq);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "hydro_fused_math: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    return kOk;
}

} // namespace

extern "C" {

int hydro_fused_math_f64(const double *d_x, size_t n, double *d_rcp, double *d_sqrt, void *stream)
{
    return fused_math<double>(d_x, n, d_rcp, d_sqrt, stream);
}
int hydro_fused_math_f32(const float *d_x, size_t n, float *d_rcp, float *d_sqrt, void *stream)
{
    return fused_math<float>(d_x, n, d_rcp, d_sqrt, stream);
}

double hydro2d_launcher_f64(const double *d_rhoE, const double *d_uv, double *d_rhoE_next, double *d_uv_next,
                            double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma,
                            double K, size_t NB_X, size_t NB_Y, const double *DtDx, const double *DtDy,
                            hydro_queue_t queue)
{
    const double t0 = now_us();
    DeviceScope ds(queue.device);
    if (!ds.ok) return finish_launcher(kErrCuda, t0, "launcher");
    if (!DtDx || !DtDy) {
        set_error(kErrArg, "launcher: DtDx/DtDy must not be null");
        return finish_launcher(kErrArg, t0, "launcher");
    }
    const int rc = step2d<double>(d_rhoE, d_uv, d_rhoE_next, d_uv_next, Dt_next,
                                  phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, *DtDx, *DtDy,
                                  (cudaStream_t)queue.stream, Kernel::Auto, true, nullptr,
                                  (queue.flags & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(queue.flags));
    return finish_launcher(rc, t0, "launcher");
}

double hydro2d_launcher_f32(const float *d_rhoE, const float *d_uv, float *d_rhoE_next, float *d_uv_next,
                            float *Dt_next, float C_min, float gamma, float gamma_minus_one, float divgamma, float K,
                            size_t NB_X, size_t NB_Y, const float *DtDx, const float *DtDy, hydro_queue_t queue)
{
    const double t0 = now_us();
    DeviceScope ds(queue.device);
    if (!ds.ok) return finish_launcher(kErrCuda, t0, "launcher");
    if (!DtDx || !DtDy) {
        set_error(kErrArg, "launcher: DtDx/DtDy must not be null");
        return finish_launcher(kErrArg, t0, "launcher");
    }
    const int rc = step2d<float>(d_rhoE, d_uv, d_rhoE_next, d_uv_next, Dt_next,
                                 phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, *DtDx, *DtDy,
                                 (cudaStream_t)queue.stream, Kernel::Auto, true, nullptr,
                                  (queue.flags & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(queue.flags));
    return finish_launcher(rc, t0, "launcher");
}

double hydro3d_launcher_f64(const double *d_rhoE, const double *d_uvw, double *d_rhoE_next, double *d_uvw_next,
                            double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma,
                            double K, size_t NB_X, size_t NB_Y, size_t NB_Z, const double *DtDx, const double *DtDy,
                            const double *DtDz, hydro_queue_t queue)
{
    const double t0 = now_us();
    DeviceScope ds(queue.device);
    if (!ds.ok) return finish_launcher(kErrCuda, t0, "launcher");
    if (!DtDx || !DtDy || !DtDz) {
        set_error(kErrArg, "launcher: DtDx/DtDy/DtDz must not be null");
        return finish_launcher(kErrArg, t0, "launcher");
    }
    const int rc = step3d<double>(d_rhoE, d_uvw, d_rhoE_next, d_uvw_next, Dt_next,
                                  phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, NB_Z, *DtDx, *DtDy,
                                  *DtDz, (cudaStream_t)queue.stream, Kernel::Auto, true, nullptr,
                                  (queue.flags & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(queue.flags));
    return finish_launcher(rc, t0, "launcher");
}

double hydro3d_launcher_f32(const float *d_rhoE, const float *d_uvw, float *d_rhoE_next, float *d_uvw_next,
                            float *Dt_next, float C_min, float gamma, float gamma_minus_one, float divgamma, float K,
                            size_t NB_X, size_t NB_Y, size_t NB_Z, const float *DtDx, const float *DtDy,
                            const float *DtDz, hydro_queue_t queue)
{
    const double t0 = now_us();
    DeviceScope ds(queue.device);
    if (!ds.ok) return finish_launcher(kErrCuda, t0, "launcher");
    if (!DtDx || !DtDy || !DtDz) {
        set_error(kErrArg, "launcher: DtDx/DtDy/DtDz must not be null");
        return finish_launcher(kErrArg, t0, "launcher");
    }
    const int rc = step3d<float>(d_rhoE, d_uvw, d_rhoE_next, d_uvw_next, Dt_next,
                                 phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, NB_Z, *DtDx, *DtDy,
                                 *DtDz, (cudaStream_t)queue.stream, Kernel::Auto, true, nullptr,
                                  (queue.flags & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(queue.flags));
    return finish_launcher(rc, t0, "launcher");
}

int hydro2d_step_f64(const double *d_rhoE, const double *d_uv, double *d_rhoE_next, double *d_uv_next,
                     double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma, double K,
                     size_t NB_X, size_t NB_Y, double DtDx, double DtDy, void *stream, int kernel, int sync,
                     hydro_step_info_t *info)
{
    StepInfo si;
    const int rc = step2d<double>(d_rhoE, d_uv, d_rhoE_next, d_uv_next, Dt_next,
                                  phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, DtDx, DtDy,
                                  (cudaStream_t)stream, (Kernel)(kernel & 0xff), sync != 0, &si,
                                  (kernel & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(kernel));
    fill(info, si);
    return rc;
}

int hydro2d_step_f32(const float *d_rhoE, const float *d_uv, float *d_rhoE_next, float *d_uv_next, float *Dt_next,
                     float C_min, float gamma, float gamma_minus_one, float divgamma, float K, size_t NB_X,
                     size_t NB_Y, float DtDx, float DtDy, void *stream, int kernel, int sync,
                     hydro_step_info_t *info)
{
    StepInfo si;
    const int rc = step2d<float>(d_rhoE, d_uv, d_rhoE_next, d_uv_next, Dt_next,
                                 phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, DtDx, DtDy,
                                 (cudaStream_t)stream, (Kernel)(kernel & 0xff), sync != 0, &si,
                                  (kernel & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(kernel));
    fill(info, si);
    return rc;
}

int hydro3d_step_f64(const double *d_rhoE, const double *d_uvw, double *d_rhoE_next, double *d_uvw_next,
                     double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma, double K,
                     size_t NB_X, size_t NB_Y, size_t NB_Z, double DtDx, double DtDy, double DtDz, void *stream,
                     int kernel, int sync, hydro_step_info_t *info)
{
    StepInfo si;
    const int rc = step3d<double>(d_rhoE, d_uvw, d_rhoE_next, d_uvw_next, Dt_next,
                                  phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, NB_Z, DtDx, DtDy,
                                  DtDz, (cudaStream_t)stream, (Kernel)(kernel & 0xff), sync != 0, &si,
                                  (kernel & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(kernel));
    fill(info, si);
    return rc;
}

int hydro3d_step_f32(const float *d_rhoE, const float *d_uvw, float *d_rhoE_next, float *d_uvw_next,
                     float *Dt_next, float C_min, float gamma, float gamma_minus_one, float divgamma, float K,
                     size_t NB_X, size_t NB_Y, size_t NB_Z, float DtDx, float DtDy, float DtDz, void *stream,
                     int kernel, int sync, hydro_step_info_t *info)
{
    StepInfo si;
    const int rc = step3d<float>(d_rhoE, d_uvw, d_rhoE_next, d_uvw_next, Dt_next,
                                 phys(C_min, gamma, gamma_minus_one, divgamma, K), NB_X, NB_Y, NB_Z, DtDx, DtDy, DtDz,
                                 (cudaStream_t)stream, (Kernel)(kernel & 0xff), sync != 0, &si,
                                  (kernel & HYDRO_X_GHOSTS_FROM_MEMORY) == 0, fused_of(kernel));
    fill(info, si);
    return rc;
}

int hydro2d_init_blast_f64(double *d_rhoE, double *d_uv, size_t NB_X, size_t NB_Y, double rho_in, double rho_out,
                           double p_in, double p_out, double C_min, double gamma, double *min_dt, void *stream)
{
    return init2d<double>(d_rhoE, d_uv, NB_X, NB_Y, rho_in, rho_out, p_in, p_out, C_min, gamma, min_dt,
                          (cudaStream_t)stream);
}
int hydro2d_init_blast_f32(float *d_rhoE, float *d_uv, size_t NB_X, size_t NB_Y, float rho_in, float rho_out,
                           float p_in, float p_out, float C_min, float gamma, float *min_dt, void *stream)
{
    return init2d<float>(d_rhoE, d_uv, NB_X, NB_Y, rho_in, rho_out, p_in, p_out, C_min, gamma, min_dt,
                         (cudaStream_t)stream);
}
int hydro3d_init_blast_f64(double *d_rhoE, double *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, double rho_in,
                           double rho_out, double p_in, double p_out, double C_min, double gamma, double *min_dt,
                           void *stream)
{
    return init3d<double>(d_rhoE, d_uvw, NB_X, NB_Y, NB_Z, rho_in, rho_out, p_in, p_out, C_min, gamma, min_dt,
                          (cudaStream_t)stream);
}
int hydro3d_init_blast_f32(float *d_rhoE, float *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, float rho_in,
                           float rho_out, float p_in, float p_out, float C_min, float gamma, float *min_dt,
                           void *stream)
{
    return init3d<float>(d_rhoE, d_uvw, NB_X, NB_Y, NB_Z, rho_in, rho_out, p_in, p_out, C_min, gamma, min_dt,
                         (cudaStream_t)stream);
}

int hydro_mass_f64(const double *d_rhoE, size_t NB_X, size_t NB_Y, size_t NB_Z, double *out, void *stream)
{
    return mass_sum<double>(d_rhoE, NB_X, NB_Y, NB_Z, out, (cudaStream_t)stream);
}
int hydro_mass_f32(const float *d_rhoE, size_t NB_X, size_t NB_Y, size_t NB_Z, double *out, void *stream)
{
    return mass_sum<float>(d_rhoE, NB_X, NB_Y, NB_Z, out, (cudaStream_t)stream);
}

int hydro_last_step_info(hydro_step_info_t *info)
{
    int err;
    DevCtx *c = ctx_current(&err);
    if (!c) return err;
    if (!info) return kErrArg;
    const StepStatus st = read_status(c->status_h);
    info->mass = st.mass + st.mass_comp;
    info->max_speed = st.max_speed;
    info->err = st.err;
    info->kernel = c->last_kernel;
    if (st.err & kErrWaitTimeout) {
        c->dirty = true;
        return kErrTimeout;
    }
    return (st.err & kErrNonPhysical) ? kErrPhys : kOk;
}

int hydro_device_contexts(void) { return ctx_count(); }

int hydro_set_launch_shape(int dim, int precision_bytes, int warps, int chunk, int blocks_per_sm)
{
    return set_launch_shape(dim, (size_t)precision_bytes, warps, chunk, blocks_per_sm);
}

int hydro_last_launch_shape(int *warps, int *chunk, int *blocks_per_sm, int *tma)
{
    int err;
    DevCtx *c = ctx_current(&err);
    if (!c) return err;
    if (warps) *warps = c->last_warps;
    if (chunk) *chunk = c->last_chunk;
    if (blocks_per_sm) *blocks_per_sm = c->last_blocks;
    if (tma) *tma = c->last_tma ? 1 : 0;
    return kOk;
}

int hydro_last_error(void) { return last_error(); }
const char *hydro_last_error_string(void) { return last_error_string(); }
void hydro_clear_error(void) { clear_error(); }
const char *hydro_version(void) { return "hydro_b200 0.1 (sm_100a)"; }

} // extern "C"
