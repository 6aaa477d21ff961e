// Host-side runtime of the CUDA library: per-device contexts (scratch words, the
// host-mapped status record), the error latch behind hydro_last_error(), TMA
// descriptor encoding, and the typed step entry points the C ABI forwards to.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "hydro_rt.cuh"

namespace hydro {

// Which kernel a step runs.
enum class Kernel : int {
    Auto = 0,   // strip kernel when its alignment rules hold, else the direct kernel
    Strip = 1,  // TMA-fed strip march (faces computed once)
    Direct = 2, // one thread per cell, neighbours loaded directly (faces computed twice)
};

struct DevCtx {
    int device = -1;
    StepScratch *scr = nullptr;   // device
    double2 *partials = nullptr;  // device, one per block
    size_t partial_cap = 0;
    StepStatus *status_h = nullptr; // host-mapped
    StepStatus *status_d = nullptr; // device alias of status_h
    unsigned seq = 0;
    int last_kernel = 0; // Kernel run by the last step launch
    int last_warps = 0;  // its launch shape (strip kernels): warps per block, rows/planes per block
    int last_chunk = 0;
    int last_blocks = 0;   // 2D: its register budget in blocks per SM
    bool last_tma = false; // its rows/planes staged by tensor-map loads
    bool dirty = false; // a launch failed: scratch words must be re-zeroed
};

// Copy of the host-mapped status record, read field by field through volatile loads.
inline StepStatus read_status(const StepStatus *p)
{
    const volatile StepStatus *v = p;
    StepStatus s;
    s.mass = v->mass;
    s.mass_comp = v->mass_comp;
    s.max_speed = v->max_speed;
    s.err = v->err;
    s.seq = v->seq;
    s.redo = v->redo;
    s.pad = 0;
    return s;
}

// a / 0 evaluated at run time (the reference's Dt_next when no cell exists)
template <class T> inline T div_zero(T a)
{
    volatile T z = T(0);
    return a / z;
}

// Key of a problem for the signal-speed skip history: the Dt_next address, the grid and
// the precision. 0 (never skip) when the speed bound's premise gamma > 1 fails.
template <class T>
inline unsigned long long problem_key(const void *dt_next, size_t a, size_t b, size_t c, size_t tsize,
                                      const Phys<T> &ph)
{
    if (!(ph.gamma > T(1))) return 0ull;
    unsigned long long k = reinterpret_cast<uintptr_t>(dt_next);
    k ^= (a + 0x9E3779B97F4A7C15ull) * 0xBF58476D1CE4E5B9ull;
    k ^= (b + 0x632BE59BD9B4E019ull) * 0x94D049BB133111EBull;
    k ^= (c + 0x2545F4914F6CDD1Dull) * 0xD6E8FEB86659FD93ull;
    k ^= tsize << 56;
    return k ? k : 1ull;
}

// Launch shape of the plain strip kernels per (dimensionality, precision), set by
// hydro_set_launch_shape (an autotuner); 0 fields keep the built-in choice.
struct LaunchShape {
    int warps = 0;  // 3D: warps per block (tile rows with halo)
    int chunk = 0;  // rows (2D) or planes (3D) each block marches
    int blocks = 0; // 2D: resident blocks per SM the registers are budgeted for (4, or 5 in FP64 / 8 in FP32)
};
LaunchShape launch_shape(int dim, size_t tsize);
int set_launch_shape(int dim, size_t tsize, int warps, int chunk, int blocks);

// Context of the current device (created on first use; never freed before exit).
DevCtx *ctx_current(int *err);
// Number of device contexts created so far in this process.
int ctx_count();
// Streaming multiprocessors of the current device, queried once per device (launch
// shapes are sized in multiples of it); 1 if the query fails.
int device_sms();
// Grow the partials array to at least n entries (synchronises the device on growth).
int ctx_reserve(DevCtx *c, size_t n);

// error latch (process-wide, last error wins)
void set_error(int code, const char *fmt, ...);
int last_error();
const char *last_error_string();
void clear_error();

// return codes of the typed entry points
enum : int {
    kOk = 0,
    kErrArg = -1,   // invalid argument (sizes, null pointers)
    kErrCuda = -2,  // a CUDA runtime call failed
    kErrPhys = -3,  // the step produced a non-physical state (flag only; outputs written)
    kErrTimeout = -4,
};

// Encode a 2D tiled tensor map (no swizzle, zero OOB fill). Returns false when the
// driver entry point is missing or encoding fails.
bool encode_tmap_2d(CUtensorMap *tm, CUtensorMapDataType dt, const void *base, uint64_t dim0, uint64_t dim1,
                    uint64_t stride1_bytes, uint32_t box0, uint32_t box1);
bool encode_tmap_3d(CUtensorMap *tm, CUtensorMapDataType dt, const void *base, uint64_t dim0, uint64_t dim1,
                    uint64_t dim2, uint64_t stride1_bytes, uint64_t stride2_bytes, uint32_t box0, uint32_t box1,
                    uint32_t box2);

// Result of one step beyond the outputs the reference writes.
struct StepInfo {
    double mass = 0.0;      // compensated sum of the new interior density
    double max_speed = 0.0; // max signal speed of the new state
    unsigned err = 0;       // error bits of the launch
    int kernel = 0;         // Kernel actually run
};

// One FVM step on the whole domain (periodic X by in-kernel wrap, reflective Y[/Z]).
// Launches on `stream`, and when `sync` is true waits for it and fills *info. xwrap:
// X neighbours of the first and last interior rows (planes) by periodic wrap inside the
// kernel (the whole domain on one device); false: from the ghost rows 0 and NB_X+1 of the
// input, filled by the caller (a subdomain of a multi-rank run).
// fused: the strip kernels in fused arithmetic (hydro_math.cuh); the direct kernel is
// always strict.
template <class T>
int step2d(const T *rhoE, const T *uv, T *rhoE_next, T *uv_next, T *Dt_next, const Phys<T> &ph, size_t nb_x,
           size_t nb_y, T DtDx, T DtDy, cudaStream_t stream, Kernel which, bool sync, StepInfo *info,
           bool xwrap = true, bool fused = false);

template <class T>
int step3d(const T *rhoE, const T *uvw, T *rhoE_next, T *uvw_next, T *Dt_next, const Phys<T> &ph, size_t nb_x,
           size_t nb_y, size_t nb_z, T DtDx, T DtDy, T DtDz, cudaStream_t stream, Kernel which, bool sync,
           StepInfo *info, bool xwrap = true, bool fused = false);

// Blast initial condition and first Dt on the device (hydro2d/main.cxx:280-338).
template <class T>
int init2d(T *rhoE, T *uv, size_t nb_x, size_t nb_y, T u_in, T u_out, T p_in, T p_out, T C_min, T gamma,
           T *min_dt, cudaStream_t stream);
// The same blast with an explicit centre (cx, cy) and radius in cell-index units (the
// reference's coordinates: interior cells are 1..NB), densities rho_in/rho_out and
// pressures p_in/p_out. `bits` is one device word of scratch; `ys` the row stride in
// cells (0: NB_Y + 2, the reference layout).
template <class T>
int init2d_at(T *rhoE, T *uv, size_t nb_x, size_t nb_y, double cx, double cy, double radius, T u_in, T u_out, T p_in,
              T p_out, T C_min, T gamma, T *min_dt, cudaStream_t stream, unsigned long long *bits, long long ys = 0);
template <class T>
int init3d_at(T *rhoE, T *uvw, size_t nb_x, size_t nb_y, size_t nb_z, double cx, double cy, double cz, double radius,
              T u_in, T u_out, T p_in, T p_out, T C_min, T gamma, T *min_dt, cudaStream_t stream,
              unsigned long long *bits);
template <class T>
int init3d(T *rhoE, T *uvw, size_t nb_x, size_t nb_y, size_t nb_z, T u_in, T u_out, T p_in, T p_out, T C_min,
           T gamma, T *min_dt, cudaStream_t stream);

// Compensated interior density sum on the device (hydro2d/main.cxx:237-265).
template <class T> int mass_sum(const T *rhoE, size_t nb_x, size_t nb_y, size_t nb_z, double *out, cudaStream_t s);

} // namespace hydro
