// Test infrastructure (oracle): a host-only stand-in for the SYCL subset used by
// hydro2d/{main,kernel}.cxx and hydro3d/{main,kernel}.cxx, so that the reference's
// unchanged sources compile with g++ and run their kernel on one CPU core.
//
// - handler::single_task runs the kernel lambda inline (the reference launches a
//   single work-item, hydro2d/kernel.cxx:354-359), so the CPU build executes the
//   reference's own per-cell loop in the reference's own order.
// - malloc_device is calloc: device memory starts zeroed like a fresh allocation that
//   the reference host then fills with a full-array copy (hydro2d/main.cxx:650-652).
// - device::get_info answers the six queries of hydro2d/main.cxx:534-560.
// It also pulls in <cmath>/<ctime> and puts sqrt in the global namespace, which the real
// header does transitively (hydro2d/kernel.hpp:33 uses unqualified sqrt).
#ifndef HYDRO_ORACLE_SYCL_SHIM_HPP
#define HYDRO_ORACLE_SYCL_SHIM_HPP

#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <math.h>
#include <string>
#include <time.h>
#include <algorithm>

using std::sqrt;

namespace sycl {

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
    template <class Q> typename Q::return_type get_info() const { return answer(Q{}); }

  private:
    static size_t answer(info::device::max_work_group_size) { return 1; }
    static size_t answer(info::device::max_compute_units) { return 1; }
    static size_t answer(info::device::global_mem_size) { return size_t(1) << 40; }
    static size_t answer(info::device::mem_base_addr_align) { return 1024; }
    static size_t answer(info::device::global_mem_cache_line_size) { return 64; }
    static std::string answer(info::device::name) { return "host CPU (single_task inline)"; }
};

class event {
  public:
    void wait() {}
};

class handler {
  public:
    template <class F> void single_task(F f) { f(); }
};

struct default_selector_t {};
inline constexpr default_selector_t default_selector_v{};

class queue {
  public:
    queue() = default;
    template <class S> explicit queue(const S &) {}
    template <class F> event submit(F f)
    {
        handler h;
        f(h);
        return {};
    }
    void wait() {}
    event memcpy(void *dst, const void *src, size_t bytes)
    {
        std::memcpy(dst, src, bytes);
        return {};
    }
    device get_device() const { return {}; }
};

template <class T> T *malloc_device(size_t n, queue &) { return static_cast<T *>(std::calloc(n, sizeof(T))); }
inline void free(void *p, queue &) { std::free(p); }

} // namespace sycl

#endif
