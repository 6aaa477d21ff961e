/*
 * C ABI of the B200 finite-volume library (libhydro_b200.so).
 *
 * The reference exposes one device entry point per program, the C-linkage
 *   extern "C" double launcher(...)
 * declared in hydro2d/kernel.hpp:63-68 (2D) and hydro3d/kernel.hpp:64-69 (3D), once
 * per precision (DATATYPE = double, or float under USE_FLOAT, kernel.hpp:9-39).
 * Because all four share the symbol name `launcher`, this library exports them under
 * distinct names; four thin drop-in libraries re-export each one as `launcher`:
 *
 *   libhydro2d.so        launcher == hydro2d_launcher_f64
 *   libhydro2d_float.so  launcher == hydro2d_launcher_f32
 *   libhydro3d.so        launcher == hydro3d_launcher_f64
 *   libhydro3d_float.so  launcher == hydro3d_launcher_f32
 *
 * Conventions shared by every launcher (the reference's, hydro2d/kernel.cxx:331-367):
 *  - device pointers are owned by the caller (hydro2d/main.cxx:125-129);
 *  - NB_X/NB_Y[/NB_Z] are interior sizes, arrays hold NB+2 cells per axis;
 *  - DtDx/DtDy[/DtDz] arrive by const reference in the reference, i.e. as pointers to
 *    host memory at the ABI; they are read on the host before the launch;
 *  - the call is synchronous and returns the elapsed microseconds measured on the host
 *    around launch and completion (feeds T->total_compute, hydro2d/main.cxx:767);
 *  - on a CUDA or argument error it returns a negative value, prints one line to
 *    stderr and latches the error for hydro_last_error(); it never aborts;
 *  - X is periodic by in-kernel wrap over the whole domain: the ghost rows/planes of
 *    the input are not read, so the host's ghost copies (hydro2d/main.cxx:720-729) are
 *    harmless but unnecessary; Y (and Z) walls are reflective.
 *  - the sycl::queue by-value argument becomes hydro_queue_t, a trivially copyable
 *    struct holding the CUDA stream; include/compat/sycl/sycl.hpp defines sycl::queue
 *    with exactly this layout so an unchanged main.cxx calls these entry points.
 */
#ifndef HYDRO_B200_H
#define HYDRO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The queue a launcher runs on: a CUDA stream (NULL = legacy default stream) and the
 * device it belongs to (-1 = the current device); flags: 0 or HYDRO_X_GHOSTS_FROM_MEMORY. */
typedef struct hydro_queue {
    void *stream;
    int device;
    int flags;
} hydro_queue_t;

/* X boundary of a step. By default the kernels take the X neighbours of the first and
 * last interior rows (planes) by periodic wrap inside the kernel: the whole domain is on
 * one device and the input's X ghost rows are never read. With this bit set in
 * hydro_queue_t.flags (launchers) or in the `kernel` argument (step entry points), they
 * read the ghost rows 0 and NB_X+1 of the input instead, as the reference kernel does
 * (hydro2d/kernel.cxx:152-170): the caller fills them, e.g. the reference's multi-rank
 * host loop exchanging subdomain edges (hydro2d/main.cxx:349-424, --sdx N). */
#define HYDRO_X_GHOSTS_FROM_MEMORY 0x100

/* Arithmetic of a step, as bits of hydro_queue_t.flags (launchers) or of the `kernel`
 * argument (step entry points).
 * HYDRO_ARITH_STRICT: every operation rounded once, in the reference's order, no
 *   contraction: bit-identical to the reference kernel compiled with -ffp-contract=off.
 * HYDRO_ARITH_FUSED: the same formulas with products that feed sums fused (one rounding),
 *   and reciprocals / square roots from the hardware approximations refined by one
 *   third-order step; results differ from strict by a few units in the last place per
 *   operation (not bit-identical), as the reference's own contracting build (-march=native)
 *   differs from its strict one.
 * With neither bit the step is strict. STRICT wins if both are set. The direct kernel
 * (HYDRO_KERNEL_DIRECT, and the fallback for misaligned arrays) is always strict. */
#define HYDRO_ARITH_FUSED 0x200
#define HYDRO_ARITH_STRICT 0x400

/* Extra results of one step, beyond what the reference's launcher returns. */
typedef struct hydro_step_info {
    double mass;      /* compensated FP64 sum of the new interior density */
    double max_speed; /* max over interior cells of c_s + |u| (Dt_next = C_min / this) */
    unsigned err;     /* bit 0: non-physical state; bit 1: a bounded wait timed out */
    int kernel;       /* 1 = strip kernel (rows by TMA, or per-lane cp.async where TMA rejects the
                         row pitch), 2 = direct kernel */
} hydro_step_info_t;

/* Kernel selection for the *_step entry points. AUTO takes the strip kernel whenever the
 * input and output arrays are aligned to their cell size, else the direct kernel; STRIP
 * on arrays that are not returns HYDRO_ERR_ARG. */
#define HYDRO_KERNEL_AUTO 0
#define HYDRO_KERNEL_STRIP 1
#define HYDRO_KERNEL_DIRECT 2

/* Return codes */
#define HYDRO_OK 0
#define HYDRO_ERR_ARG (-1)
#define HYDRO_ERR_CUDA (-2)
#define HYDRO_ERR_NONPHYSICAL (-3)
#define HYDRO_ERR_TIMEOUT (-4)

/* ---- drop-in launchers ---------------------------------------------------------- */

/* Replaces `launcher` of hydro2d/kernel.hpp:63-68 with DATATYPE = double. */
double hydro2d_launcher_f64(const double *d_rhoE, const double *d_uv, double *d_rhoE_next, double *d_uv_next,
                            double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma,
                            double K, size_t NB_X, size_t NB_Y, const double *DtDx, const double *DtDy,
                            hydro_queue_t queue);

/* Replaces `launcher` of hydro2d/kernel.hpp:63-68 with DATATYPE = float (USE_FLOAT). */
double hydro2d_launcher_f32(const float *d_rhoE, const float *d_uv, float *d_rhoE_next, float *d_uv_next,
                            float *Dt_next, float C_min, float gamma, float gamma_minus_one, float divgamma, float K,
                            size_t NB_X, size_t NB_Y, const float *DtDx, const float *DtDy, hydro_queue_t queue);

/* Replaces `launcher` of hydro3d/kernel.hpp:64-69 with DATATYPE = double. */
double hydro3d_launcher_f64(const double *d_rhoE, const double *d_uvw, double *d_rhoE_next, double *d_uvw_next,
                            double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma,
                            double K, size_t NB_X, size_t NB_Y, size_t NB_Z, const double *DtDx, const double *DtDy,
                            const double *DtDz, hydro_queue_t queue);

/* Replaces `launcher` of hydro3d/kernel.hpp:64-69 with DATATYPE = float (USE_FLOAT). */
double hydro3d_launcher_f32(const float *d_rhoE, const float *d_uvw, float *d_rhoE_next, float *d_uvw_next,
                            float *Dt_next, float C_min, float gamma, float gamma_minus_one, float divgamma, float K,
                            size_t NB_X, size_t NB_Y, size_t NB_Z, const float *DtDx, const float *DtDy,
                            const float *DtDz, hydro_queue_t queue);

/* ---- CSV output formatted on the GPU --------------------------------------------- */
/* Write a state (device arrays, reference layout) as the reference's write_results does
 * (hydro2d/main.cxx:166-235, hydro3d/main.cxx:172-247): the header "x,y,rho,p,u,v"
 * ("x,y,z,rho,p,u,v,w"), then one line "i,j[,k],rho,E,rho_u,rho_v[,rho_w]" per interior
 * cell in row-major order, i = i_offset + row - 1, each value as std::ostream writes it
 * (printf %g: 6 significant digits, correctly rounded). Byte-identical to the reference's
 * files. Returns the bytes written, or a negative error code. */
long long hydro2d_write_csv_f64(const double *d_rhoE, const double *d_uv, size_t NB_X, size_t NB_Y, size_t i_offset,
                                const char *path, void *stream);
long long hydro2d_write_csv_f32(const float *d_rhoE, const float *d_uv, size_t NB_X, size_t NB_Y, size_t i_offset,
                                const char *path, void *stream);
long long hydro3d_write_csv_f64(const double *d_rhoE, const double *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z,
                                size_t i_offset, const char *path, void *stream);
long long hydro3d_write_csv_f32(const float *d_rhoE, const float *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z,
                                size_t i_offset, const char *path, void *stream);
/* printf("%g") of n device doubles into d_out, 16 NUL-padded bytes per value. */
int hydro_format_g(const double *d_values, size_t n, char *d_out, void *stream);

/* ---- step entry points with explicit stream, kernel choice and results ------------ */
/* Same arithmetic as the launchers (hydro2d/kernel.cxx:132-319, hydro3d/kernel.cxx:
 * 145-407) with DtDx.. by value. sync = 0 only enqueues on `stream` (info->kernel is
 * still set); sync = 1 waits and fills *info (may be NULL). */
int hydro2d_step_f64(const double *d_rhoE, const double *d_uv, double *d_rhoE_next, double *d_uv_next,
                     double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma, double K,
                     size_t NB_X, size_t NB_Y, double DtDx, double DtDy, void *stream, int kernel, int sync,
                     hydro_step_info_t *info);
int hydro2d_step_f32(const float *d_rhoE, const float *d_uv, float *d_rhoE_next, float *d_uv_next, float *Dt_next,
                     float C_min, float gamma, float gamma_minus_one, float divgamma, float K, size_t NB_X,
                     size_t NB_Y, float DtDx, float DtDy, void *stream, int kernel, int sync,
                     hydro_step_info_t *info);
int hydro3d_step_f64(const double *d_rhoE, const double *d_uvw, double *d_rhoE_next, double *d_uvw_next,
                     double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma, double K,
                     size_t NB_X, size_t NB_Y, size_t NB_Z, double DtDx, double DtDy, double DtDz, void *stream,
                     int kernel, int sync, hydro_step_info_t *info);
int hydro3d_step_f32(const float *d_rhoE, const float *d_uvw, float *d_rhoE_next, float *d_uvw_next,
                     float *Dt_next, float C_min, float gamma, float gamma_minus_one, float divgamma, float K,
                     size_t NB_X, size_t NB_Y, size_t NB_Z, float DtDx, float DtDy, float DtDz, void *stream,
                     int kernel, int sync, hydro_step_info_t *info);

/* The 2D FP64 step of hydro2d_step_f64 for callers that cannot allocate memory.
 * No counterpart in the reference (whose kernel needs no scratch). Some callers own all
 * of a GPU's memory through their own pool or caching allocator, so a second allocator's
 * cudaMalloc may fail or fragment it; others step inside a latency-critical loop where
 * cudaMalloc/cudaFree, which can synchronise the whole device, must not run; others are
 * built to allocate nothing after start-up. The regular entry points allocate their
 * scratch (a few words, one partial sum per block, a pinned status record) on first use;
 * this one allocates nothing: its scratch is a fixed array of about 1 MiB compiled into
 * the library, which every GPU that loads the library holds until the process exits.
 * Limit: at most 65536 blocks of partial sums per launch, i.e. NB_Y <= 8257536 (larger
 * grids are rejected with HYDRO_ERR_ARG and a message); NB_X is handled by longer chunks.
 * The first call in a CUDA context performs a one-time set-up (it looks up the array's
 * address in that context); make that first call before any stream capture begins. All
 * calls share the array and it keeps the last call's contents: calls that overlap on the
 * GPU (two streams, two threads) race and must be serialised by the caller.
 * Arguments as hydro2d_step_f64 except that there is no `kernel` argument: the kernel is
 * chosen as HYDRO_KERNEL_AUTO does, and the X ghost rows are always the in-kernel periodic
 * wrap (HYDRO_X_GHOSTS_FROM_MEMORY is not available). With sync = 1 it waits and returns
 * results and codes as hydro2d_step_f64; with sync = 0 it only enqueues, and the step's
 * results and error codes come from hydro2d_noalloc_last_info. */
int hydro2d_step_f64_noalloc(const double *d_rhoE, const double *d_uv, double *d_rhoE_next, double *d_uv_next,
                             double *Dt_next, double C_min, double gamma, double gamma_minus_one, double divgamma,
                             double K, size_t NB_X, size_t NB_Y, double DtDx, double DtDy, void *stream, int sync,
                             hydro_step_info_t *info);

/* Results of the last hydro2d_step_f64_noalloc call in the current CUDA context, read from
 * the fixed array without allocating: the copy is ordered on `stream` (the step's stream),
 * which it synchronises. Returns HYDRO_OK, HYDRO_ERR_NONPHYSICAL or HYDRO_ERR_TIMEOUT from
 * the step's error bits. No counterpart in the reference. */
int hydro2d_noalloc_last_info(void *stream, hydro_step_info_t *info);

/* The launch shape hydro2d_step_f64_noalloc uses on a GPU with `sms` multiprocessors, for
 * the strip kernel (strip = 1) or the direct kernel (0): rows per block (*chunk, 0 for the
 * direct kernel) and the grid. Returns the number of blocks (at most 65536), or 0 when the
 * grid does not fit the fixed scratch. Host only. No counterpart in the reference. */
unsigned hydro2d_noalloc_launch_shape(size_t NB_X, size_t NB_Y, int strip, int sms, int *chunk, unsigned *grid_x,
                                      unsigned *grid_y);

/* Launch shape of the plain strip kernels for (dim 2 or 3, precision 4 or 8 bytes), as an
 * autotuner picks it. 0 keeps the built-in choice for any field.
 *  warps: 3D only, the tile height in rows with the one-row halo (8, 16, and in FP64 also
 *    9 and 12). Tiles of 8, 12 and 16 rows run one warp per row; a 9-row tile runs on 8
 *    warps, warp 0 holding both halo rows, and needs the tensor-map staging (FP64 with an
 *    even NB_Z and 16-byte aligned arrays; elsewhere 8 rows run). Built-in: 9 where the
 *    tensor maps apply, else 8;
 *  chunk: the most rows (2D) or planes (3D) one block marches (built-in 256); blocks take
 *    fewer on grids too small to fill the GPU with that many (sized from the grid and the
 *    SM count);
 *  blocks_per_sm: 2D only, the resident blocks per SM the kernel's registers are budgeted
 *    for (4, or 5 in FP64 / 8 in FP32; built-in 4).
 * Process-wide; the results do not depend on the shape. No counterpart in the reference,
 * whose single-task kernel has no launch shape. */
int hydro_set_launch_shape(int dim, int precision_bytes, int warps, int chunk, int blocks_per_sm);
/* The shape the last strip-kernel step on the current device used (warps: the 3D tile
 * height in rows as above, 0 in 2D), and
 * whether its rows / planes were staged by tensor-map loads (1) or per-lane copies (0). */
int hydro_last_launch_shape(int *warps, int *chunk, int *blocks_per_sm, int *tma);

/* Diagnostics: the number of per-device contexts (scratch words, partial sums, a pinned
 * status record) the regular entry points have created in this process. The
 * allocation-free entry points create none. No counterpart in the reference. */
int hydro_device_contexts(void);

/* Results of the last step launched on the current device, for steps enqueued with
 * sync = 0: valid once the caller has synchronised that step's stream. Returns
 * HYDRO_OK, HYDRO_ERR_NONPHYSICAL or HYDRO_ERR_TIMEOUT from the step's error bits.
 * No counterpart in the reference (its launcher is synchronous and reports nothing). */
int hydro_last_step_info(hydro_step_info_t *info);

/* ---- initial condition and mass on the device -------------------------------------- */
/* Blast initial condition of set_init_conditions_diffusion for one subdomain covering
 * the domain (hydro2d/main.cxx:280-338, hydro3d/main.cxx:296-363): writes the interior
 * (ghosts untouched) and returns the first Dt = min C_min/(c_s+|u|) in *min_dt (host).
 * Synchronous. */
int hydro2d_init_blast_f64(double *d_rhoE, double *d_uv, size_t NB_X, size_t NB_Y, double rho_in, double rho_out,
                           double p_in, double p_out, double C_min, double gamma, double *min_dt, void *stream);
int hydro2d_init_blast_f32(float *d_rhoE, float *d_uv, size_t NB_X, size_t NB_Y, float rho_in, float rho_out,
                           float p_in, float p_out, float C_min, float gamma, float *min_dt, void *stream);
int hydro3d_init_blast_f64(double *d_rhoE, double *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, double rho_in,
                           double rho_out, double p_in, double p_out, double C_min, double gamma, double *min_dt,
                           void *stream);
int hydro3d_init_blast_f32(float *d_rhoE, float *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, float rho_in,
                           float rho_out, float p_in, float p_out, float C_min, float gamma, float *min_dt,
                           void *stream);

/* Interior density sum (the quantity of compute_total_mass, hydro2d/main.cxx:237-265,
 * hydro3d/main.cxx:249-281) as a compensated FP64 sum on the device; NB_Z = 0 for 2D.
 * Synchronous; *out is host memory. */
int hydro_mass_f64(const double *d_rhoE, size_t NB_X, size_t NB_Y, size_t NB_Z, double *out, void *stream);
int hydro_mass_f32(const float *d_rhoE, size_t NB_X, size_t NB_Y, size_t NB_Z, double *out, void *stream);

/* ---- batched step ----------------------------------------------------------------------- */
/* No counterpart in the reference, whose host loop advances one domain per rank
 * (hydro2d/main.cxx:689-815): many independent blast instances of uneven sizes advanced by
 * one persistent kernel per step, each with its own Dt, simulated time (FP64), end time
 * and conservation sums; n steps run as one CUDA graph with no host round trip. An
 * instance's state is bit-identical to the same blast advanced alone (or through the plain
 * path) in the same precision. */

/* One blast problem. Cell-index coordinates as the reference's initial condition uses them
 * (interior cells 1..NB per axis, hydro2d/main.cxx:290-306): density rho_in / pressure
 * p_in inside the circle (sphere) of `radius` around `centre`, rho_out / p_out outside,
 * at rest; gamma, K and the CFL number C as hydro2d/main.cxx:601-607. The instance runs
 * while t < t_end and steps < max_steps (the reference loop condition, main.cxx:689). */
typedef struct hydro_blast {
    size_t nb[3]; /* NB_X, NB_Y, NB_Z (NB_Z = 0 in 2D) */
    double centre[3];
    double radius;
    double rho_in, rho_out, p_in, p_out;
    double gamma, K, C;
    double t_end;
    long long max_steps;
} hydro_blast_t;

typedef struct hydro_batch_status {
    double t, dt;      /* simulated time reached; the Dt of the next step */
    double mass;       /* compensated FP64 sums over the interior after the last step */
    double mom[3];
    double energy;
    double max_speed;
    long long steps;
    int active;        /* 0 once t >= t_end, steps >= max_steps or an error */
    unsigned err;      /* bit 0: non-physical state; bit 1: a bounded wait timed out */
    long long exact_passes; /* steps whose max signal speed needed the exact pass over all
                               cells (no cell reached the skip threshold) */
} hydro_batch_status_t;

/* A batch of `dim`-D (2) instances in FP32 (precision_bytes 4) or FP64 (8), rows per work
 * item `chunk` (0: 32 rows in 2D, 64 planes in 3D), at most `capacity` instances, on `stream`
 * (NULL: its own). */
void *hydro_batch_create(int dim, int precision_bytes, int chunk, int capacity, void *stream);
/* Allocate, initialise and admit one instance; returns its slot (>= 0) or an error code. */
int hydro_batch_add(void *batch, const hydro_blast_t *spec);
/* Device bytes one instance of `spec` holds (state, double-buffered). */
long long hydro_batch_bytes(void *batch, const hydro_blast_t *spec);
/* Release an instance's slot and memory (waits for the batch's stream). */
int hydro_batch_remove(void *batch, int slot);
/* Enqueue `nsteps` batched steps (one CUDA graph); sync = 1 waits for them. */
int hydro_batch_run(void *batch, int nsteps, int sync);
/* An instance's status after the last completed step (valid once the batch is synced). */
int hydro_batch_status(void *batch, int slot, hydro_batch_status_t *out);
/* Device pointers to an instance's current (rho,E) and momentum arrays and their row
 * stride in cells (rows may be padded past NB_Y + 2). Valid until the next run. */
int hydro_batch_state(void *batch, int slot, const void **rhoE, const void **uvx, long long *row_stride);
/* Copy an instance's current state into caller buffers in the reference layout
 * ((NB_X+2)(NB_Y+2) cells, no row padding); `to_host` selects host or device buffers. */
int hydro_batch_copy_state(void *batch, int slot, void *rhoE, void *uvx, int to_host);
/* Wait for every step enqueued on the batch. */
int hydro_batch_sync(void *batch);
/* Build (capture and instantiate) the graph of `nsteps` steps for the current instance set
 * without running it, so that the next hydro_batch_run(nsteps) only launches. */
int hydro_batch_prepare(void *batch, int nsteps);
/* The signal-speed skip of the batched step: a cell computes its exact signal speed only
 * when an FP32 upper bound of it reaches `frac` x the previous step's max of its instance;
 * a step where no cell does takes an exact pass over all the instance's cells. Dt is the
 * exact value whatever `frac` is (default 0.9; 0 computes every cell exactly). */
int hydro_batch_set_skip_fraction(void *batch, double frac);
/* Arithmetic of the batch's step kernels: HYDRO_ARITH_STRICT (default) or
 * HYDRO_ARITH_FUSED, as for the plain steps; an instance's state stays bit-identical to the
 * plain path in the same precision and arithmetic. Takes effect at the next run. */
int hydro_batch_set_arith(void *batch, int arith);
void hydro_batch_destroy(void *batch);

/* The blast initial condition of hydro2d/main.cxx:280-338 (hydro3d/main.cxx:296-363) with
 * an explicit centre and radius (cell-index units) and densities/pressures inside and
 * outside, for the plain path; first Dt in *min_dt (host). Synchronous. */
int hydro2d_init_blast_at_f64(double *d_rhoE, double *d_uv, size_t NB_X, size_t NB_Y, double cx, double cy,
                              double radius, double rho_in, double rho_out, double p_in, double p_out, double C_min,
                              double gamma, double *min_dt, void *stream);
int hydro2d_init_blast_at_f32(float *d_rhoE, float *d_uv, size_t NB_X, size_t NB_Y, double cx, double cy,
                              double radius, float rho_in, float rho_out, float p_in, float p_out, float C_min,
                              float gamma, float *min_dt, void *stream);
int hydro3d_init_blast_at_f64(double *d_rhoE, double *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, double cx,
                              double cy, double cz, double radius, double rho_in, double rho_out, double p_in,
                              double p_out, double C_min, double gamma, double *min_dt, void *stream);
int hydro3d_init_blast_at_f32(float *d_rhoE, float *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z, double cx,
                              double cy, double cz, double radius, float rho_in, float rho_out, float p_in,
                              float p_out, float C_min, float gamma, float *min_dt, void *stream);

/* Diagnostics: the reciprocal and square root of n device values as the fused arithmetic
 * (HYDRO_ARITH_FUSED) computes them, for comparison with the correctly rounded values.
 * Synchronous. No counterpart in the reference. */
int hydro_fused_math_f64(const double *d_x, size_t n, double *d_rcp, double *d_sqrt, void *stream);
int hydro_fused_math_f32(const float *d_x, size_t n, float *d_rcp, float *d_sqrt, void *stream);

/* ---- errors -------------------------------------------------------------------------- */
/* No counterpart in the reference (it has no status return): last error code latched
 * by any entry point (0 = none), its message, and a reset. */
int hydro_last_error(void);
const char *hydro_last_error_string(void);
void hydro_clear_error(void);
const char *hydro_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HYDRO_B200_H */
