// CSV output of a state, formatted on the GPU, byte-identical to the reference's
// write_results (hydro2d/main.cxx:166-235, hydro3d/main.cxx:172-247): a header, then one
// line "i,j[,k],rho,E,rho_u,rho_v[,rho_w]" per interior cell in row-major order, each value
// as std::ostream writes a double by default, i.e. printf("%g"): 6 significant digits,
// correctly rounded (ties to even) from the exact binary value, fixed notation for decimal
// exponents -4..5 and "d.ddddde+XX" otherwise, trailing zeros removed. FP32 states are
// formatted through their exact double value, as the stream does.
//
// Decimal conversion (every double, subnormals included): an estimate of the decimal
// exponent X and of the 6-digit integer N with |v| ~ N * 10^(X-5), from log10/exp10 in
// double (N off by at most one), then exact comparisons of |v| = m * 2^q with the rounding
// midpoints (N +- 1/2) * 10^(X-5) in fixed-size integer arithmetic (m * 5^k or
// (2N+1) * 5^k, shifted by powers of two; 5^k from a table built once per device), which
// move N to the correctly rounded value.
//
// Pipeline, per chunk of rows: one thread formats one cell's line into a fixed-size slot,
// a device scan of the line lengths gives each line's offset, a compaction writes the
// lines back to back, and the chunk goes to pinned host memory while the next chunk is
// formatted; the host writes the bytes to the file.
#include <cub/device/device_scan.cuh>

#include <math.h>
#include <mutex>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/hydro_b200.h"
#include "hydro_host.h"

namespace hydro {
namespace {

constexpr int kLimbs = 14;     // 896-bit integers: enough for m*5^330*2^s and (2N+1)*5^310
constexpr int kPow5Max = 340;  // 5^k for the decimal exponents of every finite double
constexpr int kSlot = 112;     // bytes reserved per line (longest 3D line: 103)

__device__ unsigned long long g_pow5[kPow5Max + 1][kLimbs];

// 5^k, k = 0..kPow5Max, by repeated multiplication (one thread, once per device)
__global__ void pow5_init_kernel()
{
    unsigned long long p[kLimbs] = {1ull};
    for (int k = 0; k <= kPow5Max; ++k) {
        for (int l = 0; l < kLimbs; ++l) g_pow5[k][l] = p[l];
        unsigned long long carry = 0;
        for (int l = 0; l < kLimbs; ++l) {
            const unsigned long long lo = p[l] * 5ull, hi = __umul64hi(p[l], 5ull);
            const unsigned long long s = lo + carry;
            carry = hi + (s < lo ? 1ull : 0ull);
            p[l] = s;
        }
    }
}

struct Big {
    unsigned long long w[kLimbs];
};

// r = a * m (a a table entry, m < 2^64)
__device__ __forceinline__ void big_mul_small(Big &r, const unsigned long long *a, unsigned long long m)
{
    unsigned long long carry = 0;
#pragma unroll
    for (int l = 0; l < kLimbs; ++l) {
        const unsigned long long lo = a[l] * m, hi = __umul64hi(a[l], m);
        const unsigned long long s = lo + carry;
        carry = hi + (s < lo ? 1ull : 0ull);
        r.w[l] = s;
    }
}
__device__ __forceinline__ void big_set(Big &r, unsigned long long v)
{
    r.w[0] = v;
#pragma unroll
    for (int l = 1; l < kLimbs; ++l) r.w[l] = 0;
}
// r <<= s (the operands here never lose bits: sizes checked in the header comment)
__device__ __forceinline__ void big_shl(Big &r, int s)
{
    const int q = s >> 6, b = s & 63;
    for (int l = kLimbs - 1; l >= 0; --l) {
        const int src = l - q;
        unsigned long long v = src >= 0 ? r.w[src] << b : 0ull;
        if (b && src - 1 >= 0) v |= r.w[src - 1] >> (64 - b);
        r.w[l] = v;
    }
}
__device__ __forceinline__ int big_cmp(const Big &a, const Big &b)
{
    for (int l = kLimbs - 1; l >= 0; --l)
        if (a.w[l] != b.w[l]) return a.w[l] < b.w[l] ? -1 : 1;
    return 0;
}

// sign of m*2^q - (2N+1) * 10^t / 2, exactly
__device__ int cmp_midpoint(unsigned long long m, int q, unsigned long long n2p1, int t)
{
    Big A, B;
    int ea, eb;
    if (t >= 0) {
        big_set(A, m);
        ea = q;
        big_mul_small(B, g_pow5[t], n2p1);
        eb = t - 1;
    } else {
        big_mul_small(A, g_pow5[-t], m);
        ea = q;
        big_set(B, n2p1);
        eb = t - 1;
    }
    const int d = ea - eb;
    if (d >= 0)
        big_shl(A, d);
    else
        big_shl(B, -d);
    return big_cmp(A, B);
}

__device__ __forceinline__ int put_uint(char *s, unsigned long long v)
{
    char tmp[20];
    int n = 0;
    do {
        tmp[n++] = char('0' + v % 10);
        v /= 10;
    } while (v);
    for (int i = 0; i < n; ++i) s[i] = tmp[n - 1 - i];
    return n;
}

// printf("%g", v); returns the length (at most 13)
__device__ int format_g(double v, char *s)
{
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    const bool neg = bits >> 63;
    const int bexp = (int)((bits >> 52) & 0x7ff);
    const unsigned long long frac = bits & ((1ull << 52) - 1);
    int n = 0;
    if (neg) s[n++] = '-';
    if (bexp == 0x7ff) {
        const char *w = frac ? "nan" : "inf";
        for (int i = 0; i < 3; ++i) s[n++] = w[i];
        return n;
    }
    if (bexp == 0 && frac == 0) {
        s[n++] = '0';
        return n;
    }
    const unsigned long long m = bexp ? (frac | (1ull << 52)) : frac;
    const int q = bexp ? bexp - 1075 : -1074;
    const double a = fabs(v);
    // estimate: X = floor(log10 a), N = round(a * 10^(5-X)) within one unit
    const double lg = log10(a);
    int X = (int)floor(lg);
    long long N = llrint(exp10(lg - (double)X + 5.0));
    for (int guard = 0; guard < 8; ++guard) {
        const int t = X - 5;
        if (N < 99999) N = 99999;
        if (N > 1000000) N = 1000000;
        // move N until a lies within [N - 1/2, N + 1/2] * 10^t, ties to even
        bool moved = true;
        for (int it = 0; it < 4 && moved; ++it) {
            moved = false;
            const int hi = cmp_midpoint(m, q, 2ull * (unsigned long long)N + 1ull, t);
            if (hi > 0 || (hi == 0 && (N & 1))) {
                ++N;
                moved = true;
                continue;
            }
            const int lo = cmp_midpoint(m, q, 2ull * (unsigned long long)N - 1ull, t);
            if (lo < 0 || (lo == 0 && (N & 1))) {
                --N;
                moved = true;
            }
        }
        if (N >= 1000000) { // rounds up to the next decade
            ++X;
            N = 100000;
            break;
        }
        if (N < 100000) { // the decade was overestimated
            --X;
            N = llrint(exp10(lg - (double)X + 5.0));
            continue;
        }
        break;
    }
    char d[6];
    for (int i = 5; i >= 0; --i) {
        d[i] = char('0' + N % 10);
        N /= 10;
    }
    int last = 5; // last significant digit kept after removing trailing zeros
    while (last > 0 && d[last] == '0') --last;
    if (X < -4 || X >= 6) {
        s[n++] = d[0];
        if (last > 0) {
            s[n++] = '.';
            for (int i = 1; i <= last; ++i) s[n++] = d[i];
        }
        s[n++] = 'e';
        s[n++] = X < 0 ? '-' : '+';
        const int ax = X < 0 ? -X : X;
        if (ax < 10) s[n++] = '0';
        n += put_uint(s + n, (unsigned long long)ax);
    } else if (X >= 0) {
        for (int i = 0; i <= X; ++i) s[n++] = d[i];
        if (last > X) {
            s[n++] = '.';
            for (int i = X + 1; i <= last; ++i) s[n++] = d[i];
        }
    } else {
        s[n++] = '0';
        s[n++] = '.';
        for (int i = 0; i < -X - 1; ++i) s[n++] = '0';
        for (int i = 0; i <= last; ++i) s[n++] = d[i];
    }
    return n;
}

// One line per cell of rows [row0, row0 + rows) (interior rows, 1-based) into fixed slots.
template <class T, int D>
__global__ void format_lines(const T *rhoE, const T *uvx, int nb_y, int nb_z, long long row0, int rows,
                             long long i_offset, char *slots, unsigned *lens)
{
    const long long per_row = (long long)nb_y * (D == 3 ? nb_z : 1);
    const long long ncell = per_row * rows;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell;
         q += (long long)gridDim.x * blockDim.x) {
        const long long r = q / per_row, rem = q % per_row;
        const long long i = row0 + r; // 1-based interior row
        long long j, k = 0, c;
        if (D == 2) {
            j = rem;
            c = i * (nb_y + 2) + j + 1;
        } else {
            j = rem / nb_z;
            k = rem % nb_z;
            c = (i * (long long)(nb_y + 2) + j + 1) * (nb_z + 2) + k + 1;
        }
        uint4 buf[kSlot / 16];
        char *s = reinterpret_cast<char *>(buf);
        int n = put_uint(s, (unsigned long long)(i_offset + i - 1));
        s[n++] = ',';
        n += put_uint(s + n, (unsigned long long)j);
        s[n++] = ',';
        if (D == 3) {
            n += put_uint(s + n, (unsigned long long)k);
            s[n++] = ',';
        }
        n += format_g((double)rhoE[2 * c], s + n);
        s[n++] = ',';
        n += format_g((double)rhoE[2 * c + 1], s + n);
        for (int v = 0; v < D; ++v) {
            s[n++] = ',';
            n += format_g((double)uvx[D * c + v], s + n);
        }
        s[n++] = '\n';
        uint4 *dst = reinterpret_cast<uint4 *>(slots + q * kSlot);
#pragma unroll
        for (int w = 0; w < kSlot / 16; ++w)
            if (16 * w < n) dst[w] = buf[w];
        lens[q] = (unsigned)n;
    }
}

// Lines back to back at their scanned offsets.
__global__ void compact_lines(const char *slots, const unsigned *lens, const unsigned long long *offs, long long n,
                              char *out)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const char *src = slots + q * kSlot;
        char *dst = out + offs[q];
        const unsigned len = lens[q];
        for (unsigned b = 0; b < len; ++b) dst[b] = src[b];
    }
}

// g_values formatted as %g into 16-byte records (for tests)
__global__ void format_values(const double *v, long long n, char *out)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        char s[16];
        const int len = format_g(v[q], s);
        for (int b = 0; b < 16; ++b) out[q * 16 + b] = b < len ? s[b] : '\0';
    }
}

std::mutex g_pow5_mu;
bool g_pow5_done[64];

int ensure_pow5(cudaStream_t st)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error(kErrCuda, "csv: no current device");
        return kErrCuda;
    }
    std::lock_guard<std::mutex> lk(g_pow5_mu);
    if (g_pow5_done[dev]) return kOk;
    pow5_init_kernel<<<1, 1, 0, st>>>();
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "csv: power table: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    g_pow5_done[dev] = true;
    return kOk;
}

template <class T, int D>
long long write_csv(const T *rhoE, const T *uvx, size_t nb_x, size_t nb_y, size_t nb_z, size_t i_offset,
                    const char *path, cudaStream_t st)
{
    if (!rhoE || !uvx || !path) {
        set_error(kErrArg, "write_csv: null argument");
        return kErrArg;
    }
    if (nb_x > (1u << 30) || nb_y > (1u << 30) || (D == 3 && nb_z > (1u << 30)) || i_offset > (1ull << 40)) {
        set_error(kErrArg, "write_csv: grid or row offset too large");
        return kErrArg;
    }
    int rc = ensure_pow5(st);
    if (rc != kOk) return rc;
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error(kErrArg, "write_csv: cannot open %s", path);
        return kErrArg;
    }
    const char *header = D == 2 ? "x,y,rho,p,u,v\n" : "x,y,z,rho,p,u,v,w\n";
    long long total = (long long)fwrite(header, 1, strlen(header), f);
    const long long per_row = (long long)nb_y * (D == 3 ? (long long)nb_z : 1);
    if (nb_x == 0 || per_row == 0) {
        fclose(f);
        return total;
    }
    // cells per chunk (HYDRO_B200_CSV_CHUNK_CELLS overrides, e.g. to exercise many chunks)
    long long target = 4ll << 20;
    if (const char *env = getenv("HYDRO_B200_CSV_CHUNK_CELLS")) {
        const long long v = atoll(env);
        if (v > 0) target = v;
    }
    const int rows = (int)std::max<long long>(1, std::min<long long>((long long)nb_x, target / per_row));
    const long long cap = per_row * rows;
    char *slots = nullptr, *out = nullptr, *host[2] = {nullptr, nullptr};
    unsigned *lens = nullptr;
    unsigned long long *offs = nullptr, *h_tot = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaEvent_t done[2] = {nullptr, nullptr};
    long long pending[2] = {0, 0};
    cudaError_t e = cudaMalloc(&slots, (size_t)cap * kSlot);
    if (e == cudaSuccess) e = cudaMalloc(&out, (size_t)cap * kSlot);
    if (e == cudaSuccess) e = cudaMalloc(&lens, (size_t)cap * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&offs, (size_t)(cap + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&host[0], (size_t)cap * kSlot);
    if (e == cudaSuccess) e = cudaMallocHost(&host[1], (size_t)cap * kSlot);
    if (e == cudaSuccess) e = cudaMallocHost(&h_tot, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, lens, offs, (int)cap, st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    int chunk = 0;
    for (long long row0 = 1; e == cudaSuccess && row0 <= (long long)nb_x; row0 += rows, ++chunk) {
        const int nr = (int)std::min<long long>(rows, (long long)nb_x - row0 + 1);
        const long long n = per_row * nr;
        const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)device_sms() * 16);
        format_lines<T, D><<<blocks, 256, 0, st>>>(rhoE, uvx, (int)nb_y, (int)nb_z, row0, nr, (long long)i_offset,
                                                    slots, lens);
        e = cudaGetLastError();
        // offsets of the n lines; offs[n] = the chunk's byte count
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, lens, offs, (int)n, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&h_tot[0], offs + (n - 1), sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        unsigned last_len = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_tot[1], lens + (n - 1), sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) break;
        memcpy(&last_len, &h_tot[1], sizeof(unsigned));
        const long long bytes = (long long)h_tot[0] + last_len;
        compact_lines<<<blocks, 256, 0, st>>>(slots, lens, offs, n, out);
        e = cudaGetLastError();
        const int b = chunk & 1;
        // the previous use of this pinned buffer has been written out below
        if (e == cudaSuccess) e = cudaMemcpyAsync(host[b], out, (size_t)bytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(done[b], st);
        pending[b] = bytes;
        // write the other buffer (the previous chunk) while this one is in flight
        const int o = b ^ 1;
        if (e == cudaSuccess && pending[o] > 0 && chunk > 0) {
            e = cudaEventSynchronize(done[o]);
            if (e == cudaSuccess) {
                if ((long long)fwrite(host[o], 1, (size_t)pending[o], f) != pending[o]) {
                    set_error(kErrArg, "write_csv: short write to %s", path);
                    rc = kErrArg;
                    break;
                }
                total += pending[o];
                pending[o] = 0;
            }
        }
    }
    // the last chunk
    if (e == cudaSuccess && rc == kOk) {
        const int b = (chunk - 1) & 1;
        if (pending[b] > 0) {
            e = cudaEventSynchronize(done[b]);
            if (e == cudaSuccess) {
                if ((long long)fwrite(host[b], 1, (size_t)pending[b], f) != pending[b]) {
                    set_error(kErrArg, "write_csv: short write to %s", path);
                    rc = kErrArg;
                } else {
                    total += pending[b];
                }
            }
        }
    }
    if (e != cudaSuccess) cudaStreamSynchronize(st);
    cudaFree(slots);
    cudaFree(out);
    cudaFree(lens);
    cudaFree(offs);
    cudaFree(tmp);
    if (host[0]) cudaFreeHost(host[0]);
    if (host[1]) cudaFreeHost(host[1]);
    if (h_tot) cudaFreeHost(h_tot);
    for (auto ev : done)
        if (ev) cudaEventDestroy(ev);
    if (fclose(f) != 0 && rc == kOk) {
        set_error(kErrArg, "write_csv: closing %s failed", path);
        rc = kErrArg;
    }
    if (e != cudaSuccess) {
        set_error(kErrCuda, "write_csv: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    return rc == kOk ? total : rc;
}

} // namespace
} // namespace hydro

using namespace hydro;

extern "C" {

long long hydro2d_write_csv_f64(const double *d_rhoE, const double *d_uv, size_t NB_X, size_t NB_Y, size_t i_offset,
                                const char *path, void *stream)
{
    return write_csv<double, 2>(d_rhoE, d_uv, NB_X, NB_Y, 0, i_offset, path, (cudaStream_t)stream);
}
long long hydro2d_write_csv_f32(const float *d_rhoE, const float *d_uv, size_t NB_X, size_t NB_Y, size_t i_offset,
                                const char *path, void *stream)
{
    return write_csv<float, 2>(d_rhoE, d_uv, NB_X, NB_Y, 0, i_offset, path, (cudaStream_t)stream);
}
long long hydro3d_write_csv_f64(const double *d_rhoE, const double *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z,
                                size_t i_offset, const char *path, void *stream)
{
    return write_csv<double, 3>(d_rhoE, d_uvw, NB_X, NB_Y, NB_Z, i_offset, path, (cudaStream_t)stream);
}
long long hydro3d_write_csv_f32(const float *d_rhoE, const float *d_uvw, size_t NB_X, size_t NB_Y, size_t NB_Z,
                                size_t i_offset, const char *path, void *stream)
{
    return write_csv<float, 3>(d_rhoE, d_uvw, NB_X, NB_Y, NB_Z, i_offset, path, (cudaStream_t)stream);
}

int hydro_format_g(const double *d_values, size_t n, char *d_out, void *stream)
{
    if (!d_values || !d_out) {
        set_error(kErrArg, "hydro_format_g: null argument");
        return kErrArg;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_pow5(st);
    if (rc != kOk) return rc;
    if (n == 0) return kOk;
    format_values<<<(int)std::min<size_t>((n + 255) / 256, (size_t)device_sms() * 16), 256, 0, st>>>(d_values, (long long)n, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(kErrCuda, "hydro_format_g: %s", cudaGetErrorString(e));
        return kErrCuda;
    }
    return kOk;
}

} // extern "C"
