// Per-device contexts, error latch and TMA descriptor encoding.
#include <atomic>
#include <cudaTypedefs.h>
#include <mutex>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "hydro_host.h"

namespace hydro {

namespace {
std::mutex g_mu;
DevCtx *g_ctx[64] = {};
int g_err = 0;
char g_msg[512] = "";
} // namespace

void set_error(int code, const char *fmt, ...)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_err = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
}

int last_error()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_err;
}

const char *last_error_string()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_msg;
}

void clear_error()
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_err = 0;
    g_msg[0] = 0;
}

DevCtx *ctx_current(int *err)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        set_error(kErrCuda, "cudaGetDevice failed: %s", cudaGetErrorString(e));
        *err = kErrCuda;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_ctx[dev]) {
        *err = kOk;
        return g_ctx[dev];
    }
    DevCtx *c = new DevCtx;
    c->device = dev;
    e = cudaMalloc(&c->scr, sizeof(StepScratch));
    if (e == cudaSuccess) e = cudaMemset(c->scr, 0, sizeof(StepScratch));
    if (e == cudaSuccess) e = cudaHostAlloc(&c->status_h, sizeof(StepStatus), cudaHostAllocMapped);
    if (e == cudaSuccess) {
        memset(c->status_h, 0, sizeof(StepStatus));
        e = cudaHostGetDevicePointer(&c->status_d, c->status_h, 0);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        snprintf(g_msg, sizeof g_msg, "device context set-up failed: %s", cudaGetErrorString(e));
        g_err = kErrCuda;
        *err = kErrCuda;
        if (c->scr) cudaFree(c->scr);
        if (c->status_h) cudaFreeHost(c->status_h);
        delete c;
        return nullptr;
    }
    g_ctx[dev] = c;
    *err = kOk;
    return c;
}

int device_sms()
{
    static std::atomic<int> cache[64];
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 1;
    cache[dev].store(n, std::memory_order_relaxed);
    return n;
}

namespace {
LaunchShape g_shape[2][2]; // [dim - 2][FP64]
} // namespace

LaunchShape launch_shape(int dim, size_t tsize)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_shape[dim == 3][tsize == 8];
}

int set_launch_shape(int dim, size_t tsize, int warps, int chunk, int blocks)
{
    const int alt_blocks = tsize == 8 ? 5 : 8;
    if ((dim != 2 && dim != 3) || (tsize != 4 && tsize != 8) || chunk < 0 || chunk > (1 << 20) ||
        (dim == 2 && (warps != 0 || (blocks != 0 && blocks != 4 && blocks != alt_blocks))) ||
        (dim == 3 && (blocks != 0 || (warps != 0 && warps != 8 && warps != 16 &&
                                          !(tsize == 8 && (warps == 9 || warps == 12)))))) {
        set_error(kErrArg,
                  "hydro_set_launch_shape: unsupported shape (dim %d, %zu-byte values, %d warps, chunk %d, %d blocks)",
                  dim, tsize, warps, chunk, blocks);
        return kErrArg;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_shape[dim == 3][tsize == 8] = LaunchShape{warps, chunk, blocks};
    return kOk;
}

int ctx_count()
{
    std::lock_guard<std::mutex> lk(g_mu);
    int n = 0;
    for (DevCtx *c : g_ctx) n += (c != nullptr);
    return n;
}

int ctx_reserve(DevCtx *c, size_t n)
{
    if (n <= c->partial_cap) return kOk;
    size_t cap = c->partial_cap ? c->partial_cap : 1024;
    while (cap < n) cap *= 2;
    cudaError_t e = cudaDeviceSynchronize();
    if (c->partials) cudaFree(c->partials);
    c->partials = nullptr;
    c->partial_cap = 0;
    if (e == cudaSuccess) e = cudaMalloc(&c->partials, cap * sizeof(double2));
    if (e != cudaSuccess) {
        set_error(kErrCuda, "scratch allocation of %zu partials failed: %s", cap, cudaGetErrorString(e));
        return kErrCuda;
    }
    c->partial_cap = cap;
    return kOk;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}
} // namespace

bool encode_tmap_2d(CUtensorMap *tm, CUtensorMapDataType dt, const void *base, uint64_t dim0, uint64_t dim1,
                    uint64_t stride1_bytes, uint32_t box0, uint32_t box1)
{
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {dim0, dim1};
    cuuint64_t strides[1] = {stride1_bytes};
    cuuint32_t box[2] = {box0, box1};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(tm, dt, 2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool encode_tmap_3d(CUtensorMap *tm, CUtensorMapDataType dt, const void *base, uint64_t dim0, uint64_t dim1,
                    uint64_t dim2, uint64_t stride1_bytes, uint64_t stride2_bytes, uint32_t box0, uint32_t box1,
                    uint32_t box2)
{
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {dim0, dim1, dim2};
    cuuint64_t strides[2] = {stride1_bytes, stride2_bytes};
    cuuint32_t box[3] = {box0, box1, box2};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(tm, dt, 3, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

} // namespace hydro
