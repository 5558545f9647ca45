// The NCG update of wust_reconstruct (Runtime/matlab/wust_reconstruct.m:24-57)
// on the device, FP64: ROI restriction and the ringing filter of the gradient
// (wust_roi_gradient.m:1-10, ringingRemovalFilt.m:1-45; the FFTs through
// cuFFT), the PR/FR direction (wust_ncg_direction.m:1-17), dot products and
// the slowness projection (wust_project_slowness_update.m:1-10).  Fields are
// ny x nx column-major doubles, masks bytes (0/1).
//
// Reductions are deterministic: every block writes one partial and the host
// sums the partials in block order.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int kNcgThreads = 256;

int ncg_blocks(size_t n) { return (int)std::min<size_t>((n + kNcgThreads - 1) / kNcgThreads, kNcgMaxBlocks); }

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kNcgThreads / 32; ++k) t += sh[k];
    return t;
}

// roi = mask ? g : 0
__global__ void roi_kernel(const double *g, const uint8_t *mask, double *roi, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        roi[i] = mask[i] ? g[i] : 0.0;
}

// z = mask ? z * scale : 0
__global__ void mask_scale_kernel(double *z, const uint8_t *mask, double scale, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        z[i] = mask[i] ? z[i] * scale : 0.0;
}

// Radial Butterworth low-pass on the half spectrum of the real 2-D transform
// of a column-major ny x nx field (cuFFT dims (nx, ny): index (ix, iy), iy in
// [0, ny/2]).  The reference builds the filter on the fftshift-ed grid with
// k >= 1/(2 d) wrapped to k - 1/d and applies it to the shifted spectrum;
// unshifted, that is the standard FFT frequency of each index.
__global__ void butterworth_kernel(double2 *spec, int nx, int ny, double dx, double dy, double kc2, double order) {
    const int nyh = ny / 2 + 1;
    const size_t total = (size_t)nx * nyh;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i / nyh), iy = (int)(i % nyh);
        double kx = ((double)ix / nx) / dx, ky = ((double)iy / ny) / dy;
        if (kx >= 1.0 / (2.0 * dx)) kx -= 1.0 / dx;
        if (ky >= 1.0 / (2.0 * dy)) ky -= 1.0 / dy;
        const double f = 1.0 / (1.0 + pow((kx * kx + ky * ky) / kc2, order));
        spec[i].x *= f;
        spec[i].y *= f;
    }
}

// partials of sum a b and sum a (b - c)
__global__ void dot2_kernel(const double *a, const double *b, const double *c, size_t n, double *part) {
    __shared__ double sh[kNcgThreads / 32];
    double s0 = 0.0, s1 = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        s0 += a[i] * b[i];
        s1 += a[i] * (b[i] - c[i]);
    }
    const double t0 = block_sum(s0, sh);
    const double t1 = block_sum(s1, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = t0;
        part[2 * blockIdx.x + 1] = t1;
    }
}

__global__ void dot_kernel(const double *a, const double *b, size_t n, double *part) {
    __shared__ double sh[kNcgThreads / 32];
    double s = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    const double t = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// d = -z + beta d (beta = 0: d = -z); partials of sum g d and of the count of
// nonfinite entries of d
__global__ void direction_kernel(const double *z, const double *g, double beta, double *d, size_t n, double *part) {
    __shared__ double sh[kNcgThreads / 32];
    double s = 0.0, bad = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = beta == 0.0 ? -z[i] : -z[i] + beta * d[i];
        d[i] = v;
        s += g[i] * v;
        if (!isfinite(v)) bad += 1.0;
    }
    const double t0 = block_sum(s, sh);
    const double t1 = block_sum(bad, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = t0;
        part[2 * blockIdx.x + 1] = t1;
    }
}

// Clip in slowness, then invert; outside the mask c is unchanged.  Partials:
// nonfinite trials, sum over the mask of (1/c_new - 1/c_old)^2 and (1/c_old)^2.
__global__ void project_kernel(double *c, const double *d, double step, double max_update, double c_min, double c_max,
                               const uint8_t *mask, size_t n, double *part) {
    __shared__ double sh[kNcgThreads / 32];
    double bad = 0.0, du = 0.0, so = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double ci = c[i];
        const double c_lo = fmax(ci - max_update, c_min);
        const double c_hi = fmin(ci + max_update, c_max);
        const double s_old = 1.0 / ci;
        const double trial = s_old + step * d[i];
        if (!isfinite(trial)) bad += 1.0;
        if (mask[i]) {
            const double s_new = fmax(1.0 / c_hi, fmin(1.0 / c_lo, trial));
            const double cn = 1.0 / s_new;
            c[i] = cn;
            const double e = 1.0 / cn - s_old;
            du += e * e;
            so += s_old * s_old;
        }
    }
    const double t0 = block_sum(bad, sh);
    const double t1 = block_sum(du, sh);
    const double t2 = block_sum(so, sh);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = t0;
        part[3 * blockIdx.x + 1] = t1;
        part[3 * blockIdx.x + 2] = t2;
    }
}

void ncg_roi_launch(const double *g, const uint8_t *mask, double *roi, size_t n, cudaStream_t st) {
    roi_kernel<<<ncg_blocks(n), kNcgThreads, 0, st>>>(g, mask, roi, n);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}
void ncg_mask_scale_launch(double *z, const uint8_t *mask, double scale, size_t n, cudaStream_t st) {
    mask_scale_kernel<<<ncg_blocks(n), kNcgThreads, 0, st>>>(z, mask, scale, n);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}
void ncg_butterworth_launch(double2 *spec, int nx, int ny, double dx, double dy, double kc2, double order,
                            cudaStream_t st) {
    butterworth_kernel<<<ncg_blocks((size_t)nx * (ny / 2 + 1)), kNcgThreads, 0, st>>>(spec, nx, ny, dx, dy, kc2, order);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}
int ncg_dot2_launch(const double *a, const double *b, const double *c, size_t n, double *part, cudaStream_t st) {
    const int nb = ncg_blocks(n);
    dot2_kernel<<<nb, kNcgThreads, 0, st>>>(a, b, c, n, part);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
    return nb;
}
int ncg_dot_launch(const double *a, const double *b, size_t n, double *part, cudaStream_t st) {
    const int nb = ncg_blocks(n);
    dot_kernel<<<nb, kNcgThreads, 0, st>>>(a, b, n, part);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
    return nb;
}
int ncg_direction_launch(const double *z, const double *g, double beta, double *d, size_t n, double *part,
                         cudaStream_t st) {
    const int nb = ncg_blocks(n);
    direction_kernel<<<nb, kNcgThreads, 0, st>>>(z, g, beta, d, n, part);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
    return nb;
}
int ncg_project_launch(double *c, const double *d, double step, double max_update, double c_min, double c_max,
                       const uint8_t *mask, size_t n, double *part, cudaStream_t st) {
    const int nb = ncg_blocks(n);
    project_kernel<<<nb, kNcgThreads, 0, st>>>(c, d, step, max_update, c_min, c_max, mask, n, part);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
    return nb;
}

}  // namespace wust
