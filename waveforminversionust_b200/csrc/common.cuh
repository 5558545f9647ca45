// Shared device/host helpers for the sm_100a Helmholtz kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/wust_b200.h"

namespace wust {

// ---------------------------------------------------------------------------
// Errors: every internal failure throws WustError(status, message); the C ABI
// converts it to a status code and a thread-local message.
// ---------------------------------------------------------------------------
struct WustError {
    int status;
    std::string message;
};

[[noreturn]] void fail(int status, const char *fmt, ...);
void set_last_error(const std::string &msg);

#define WUST_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t wust_e_ = (call);                                                        \
        if (wust_e_ != cudaSuccess)                                                          \
            ::wust::fail(WUST_ERR_CUDA, "%s failed: %s (%d)", #call, cudaGetErrorString(wust_e_), \
                         (int)wust_e_);                                                      \
    } while (0)

#define WUST_LAUNCH_CHECK() WUST_CUDA(cudaPeekAtLastError())

// ---------------------------------------------------------------------------
// Complex arithmetic (interleaved float2 / double2).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// acc += a * b
__device__ __forceinline__ void cfma(float2 &acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfma_conj(float2 &acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(-a.y, b.x, acc.y);
}

__host__ __device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 zscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
    // Smith's algorithm for a / b.
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    } else {
        double r = b.x / b.y, den = b.x * r + b.y;
        return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
    }
}
__host__ __device__ __forceinline__ double2 z_from(float2 a) { return make_double2((double)a.x, (double)a.y); }
__host__ __device__ __forceinline__ float2 c_from(double2 a) { return make_float2((float)a.x, (float)a.y); }
__host__ __device__ __forceinline__ double zabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// %globaltimer in nanoseconds: the clock of every bounded device-side wait.
__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Coefficient views: the nine block arrays in the reference layout
// (ninePointCoefficients.m:16-24): Dd Ny x Nx, Dl/Du (Ny-1) x Nx,
// Ld/Ud Ny x (Nx-1), Ll/Lu/Ul/Uu (Ny-1) x (Nx-1), all column-major.
// ---------------------------------------------------------------------------
template <typename T>
struct Coefs {
    const T *Dd, *Dl, *Du, *Ld, *Ll, *Lu, *Ud, *Ul, *Uu;
    int ny, nx;
    __host__ __device__ __forceinline__ T dd(int y, int x) const { return Dd[y + (size_t)ny * x]; }
    __host__ __device__ __forceinline__ T dl(int y, int x) const { return Dl[y + (size_t)(ny - 1) * x]; }
    __host__ __device__ __forceinline__ T du(int y, int x) const { return Du[y + (size_t)(ny - 1) * x]; }
    __host__ __device__ __forceinline__ T ld(int y, int x) const { return Ld[y + (size_t)ny * x]; }
    __host__ __device__ __forceinline__ T ll(int y, int x) const { return Ll[y + (size_t)(ny - 1) * x]; }
    __host__ __device__ __forceinline__ T lu(int y, int x) const { return Lu[y + (size_t)(ny - 1) * x]; }
    __host__ __device__ __forceinline__ T ud(int y, int x) const { return Ud[y + (size_t)ny * x]; }
    __host__ __device__ __forceinline__ T ul(int y, int x) const { return Ul[y + (size_t)(ny - 1) * x]; }
    __host__ __device__ __forceinline__ T uu(int y, int x) const { return Uu[y + (size_t)(ny - 1) * x]; }
};

// Right-hand-side sources of a sweep.
enum SrcMode { SRC_NONE = 0, SRC_DENSE = 1, SRC_POINT = 2, SRC_SCATTER = 3 };

struct SrcView {
    int mode;
    const float2 *dense;     // SRC_DENSE: [ny, nx, S]
    const int32_t *lin;      // SRC_POINT: 0-based linear index per source (unit amplitude)
    const int32_t *at;       // SRC_SCATTER: [ny*nx] receiver slot or -1
    const float2 *vals;      // SRC_SCATTER: [n_slots, S]
    int n_slots;
    __device__ __forceinline__ float2 get(int y, int x, int s, int ny, int nx) const {
        size_t p = (size_t)y + (size_t)ny * x;
        if (mode == SRC_DENSE) return dense[p + (size_t)ny * nx * s];
        if (mode == SRC_POINT) return lin[s] == (int32_t)p ? make_float2(1.f, 0.f) : make_float2(0.f, 0.f);
        if (mode == SRC_SCATTER) {
            int k = at[p];
            return k >= 0 ? vals[k + (size_t)n_slots * s] : make_float2(0.f, 0.f);
        }
        return make_float2(0.f, 0.f);
    }
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Launch counter shared by the host drivers (reported through wust_solver_stats).
extern thread_local long long g_kernel_launches;

}  // namespace wust
