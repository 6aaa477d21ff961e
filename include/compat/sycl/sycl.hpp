// The SYCL subset used by the reference host programs (hydro2d/main.cxx,
// hydro3d/main.cxx), implemented on the CUDA runtime, so that those programs compile
// unchanged and drive this project's CUDA launcher instead of the SYCL single_task.
//
//   sycl::queue            a CUDA stream on the current device; trivially copyable with
//                          the layout of hydro_queue_t, because the reference passes it
//                          by value to `launcher` (hydro2d/kernel.hpp:63-68)
//   queue.memcpy / wait    cudaMemcpyAsync on the stream / cudaStreamSynchronize
//   malloc_device / free   cudaMalloc / cudaFree  (hydro2d/main.cxx:125-141)
//   device::get_info       the six queries of hydro2d/main.cxx:534-560 from
//                          cudaDeviceProp
//   handler::single_task   not provided: only the reference's kernel.cxx uses it, and
//                          that file is what this project replaces.
#ifndef HYDRO_COMPAT_SYCL_HPP
#define HYDRO_COMPAT_SYCL_HPP

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>
#include <string>
#include <type_traits>

#include "../../hydro_b200.h"

using std::sqrt;

namespace sycl {

namespace detail {
inline void check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[sycl-on-cuda] %s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}
} // namespace detail

namespace info {
namespace device {
struct max_work_group_size { using return_type = size_t; };
struct max_compute_units { using return_type = size_t; };
struct global_mem_size { using return_type = size_t; };
struct mem_base_addr_align { using return_type = size_t; };
struct global_mem_cache_line_size { using return_type = size_t; };
struct name { using return_type = std::string; };
} // namespace device
} // namespace info

class device {
  public:
    explicit device(int id = 0) : id_(id) {}
    template <class Q> typename Q::return_type get_info() const
    {
        cudaDeviceProp p;
        detail::check(cudaGetDeviceProperties(&p, id_), "cudaGetDeviceProperties");
        return answer(Q{}, p);
    }

  private:
    int id_;
    static size_t answer(info::device::max_work_group_size, const cudaDeviceProp &p) { return p.maxThreadsPerBlock; }
    static size_t answer(info::device::max_compute_units, const cudaDeviceProp &p) { return p.multiProcessorCount; }
    static size_t answer(info::device::global_mem_size, const cudaDeviceProp &p) { return p.totalGlobalMem; }
    static size_t answer(info::device::mem_base_addr_align, const cudaDeviceProp &) { return 256 * 8; }
    static size_t answer(info::device::global_mem_cache_line_size, const cudaDeviceProp &) { return 128; }
    static std::string answer(info::device::name, const cudaDeviceProp &p) { return std::string(p.name); }
};

class event {
  public:
    explicit event(cudaStream_t s = nullptr) : s_(s) {}
    void wait() { detail::check(cudaStreamSynchronize(s_), "cudaStreamSynchronize"); }

  private:
    cudaStream_t s_;
};

struct default_selector_t {};
inline constexpr default_selector_t default_selector_v{};

// Trivially copyable: its only data member is the C ABI's hydro_queue_t.
class queue {
  public:
    queue()
    {
        int dev = 0;
        detail::check(cudaGetDevice(&dev), "cudaGetDevice");
        cudaStream_t s = nullptr;
        detail::check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        q_.stream = s;
        q_.device = dev;
        // HYDRO_B200_X_GHOSTS=memory: the kernels read the X ghost rows the host loop fills
        // (a multi-rank --sdx run) instead of wrapping periodically in-kernel (one rank)
        const char *xg = std::getenv("HYDRO_B200_X_GHOSTS");
        q_.flags = (xg && std::strcmp(xg, "memory") == 0) ? HYDRO_X_GHOSTS_FROM_MEMORY : 0;
        // HYDRO_B200_ARITH=fused / strict: the arithmetic of every step (the library's
        // default when unset)
        const char *ar = std::getenv("HYDRO_B200_ARITH");
        if (ar && std::strcmp(ar, "fused") == 0) q_.flags |= HYDRO_ARITH_FUSED;
        if (ar && std::strcmp(ar, "strict") == 0) q_.flags |= HYDRO_ARITH_STRICT;
    }
    template <class S> explicit queue(const S &) : queue() {}

    void wait() { detail::check(cudaStreamSynchronize(stream()), "cudaStreamSynchronize"); }
    event memcpy(void *dst, const void *src, size_t bytes)
    {
        detail::check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, stream()), "cudaMemcpyAsync");
        return event(stream());
    }
    device get_device() const { return device(q_.device); }
    cudaStream_t stream() const { return static_cast<cudaStream_t>(q_.stream); }

  private:
    hydro_queue_t q_;
};

static_assert(std::is_trivially_copyable<queue>::value, "queue is passed by value through a C ABI");
static_assert(sizeof(queue) == sizeof(hydro_queue_t), "queue must have the layout of hydro_queue_t");

template <class T> T *malloc_device(size_t n, queue &)
{
    void *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    return static_cast<T *>(p);
}
inline void free(void *p, queue &) { cudaFree(p); }

} // namespace sycl

#endif
