// FP64 residuals for iterative refinement of the block-LU solves.
//
// r = b - H x (or b - H^H x) with the complex128 coefficients, evaluated
// with the nine-point formula of the sparse assembly
// (HelmholtzSolver.m:118-135) and its conjugate transpose.  Rows on the top
// and bottom Dirichlet border (y = 0, Ny-1) are excluded: the block solver
// keeps them at zero (applyBlockLU.cu:10), so they never enter the other
// equations and cannot be corrected.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

__device__ __forceinline__ double2 zfma_c(double2 acc, double2 a, double2 b, bool conj_a) {
    if (conj_a) a.y = -a.y;
    acc.x += a.x * b.x - a.y * b.y;
    acc.y += a.x * b.y + a.y * b.x;
    return acc;
}

template <bool ADJ>
__global__ void residual_kernel(Coefs<double2> co, SrcView b, const double2 *x, int S, float2 *r32, double *rnorm2,
                                double *bnorm2) {
    const int ny = co.ny, nx = co.nx;
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    const int xi = blockIdx.y;
    const int s = blockIdx.z;
    double rr = 0, bb = 0;
    if (y < ny && xi < nx) {
        const size_t fs = (size_t)ny * nx * s;
        const double2 *xs = x + fs;
        auto X = [&](int yy, int xx) { return xs[(size_t)yy + (size_t)ny * xx]; };
        double2 r = make_double2(0.0, 0.0);
        if (y >= 1 && y <= ny - 2) {
            double2 h = make_double2(0.0, 0.0);
            if (!ADJ) {
                h = zfma_c(h, co.dd(y, xi), X(y, xi), false);
                h = zfma_c(h, co.dl(y - 1, xi), X(y - 1, xi), false);
                h = zfma_c(h, co.du(y, xi), X(y + 1, xi), false);
                if (xi >= 1) {
                    h = zfma_c(h, co.ld(y, xi - 1), X(y, xi - 1), false);
                    h = zfma_c(h, co.ll(y - 1, xi - 1), X(y - 1, xi - 1), false);
                    h = zfma_c(h, co.lu(y, xi - 1), X(y + 1, xi - 1), false);
                }
                if (xi <= nx - 2) {
                    h = zfma_c(h, co.ud(y, xi), X(y, xi + 1), false);
                    h = zfma_c(h, co.ul(y - 1, xi), X(y - 1, xi + 1), false);
                    h = zfma_c(h, co.uu(y, xi), X(y + 1, xi + 1), false);
                }
            } else {
                h = zfma_c(h, co.dd(y, xi), X(y, xi), true);
                h = zfma_c(h, co.dl(y, xi), X(y + 1, xi), true);
                h = zfma_c(h, co.du(y - 1, xi), X(y - 1, xi), true);
                if (xi <= nx - 2) {
                    h = zfma_c(h, co.ld(y, xi), X(y, xi + 1), true);
                    h = zfma_c(h, co.ll(y, xi), X(y + 1, xi + 1), true);
                    h = zfma_c(h, co.lu(y - 1, xi), X(y - 1, xi + 1), true);
                }
                if (xi >= 1) {
                    h = zfma_c(h, co.ud(y, xi - 1), X(y, xi - 1), true);
                    h = zfma_c(h, co.ul(y, xi - 1), X(y + 1, xi - 1), true);
                    h = zfma_c(h, co.uu(y - 1, xi - 1), X(y - 1, xi - 1), true);
                }
            }
            const double2 bv = z_from(b.get(y, xi, s, ny, nx));
            r = zsub(bv, h);
            rr = zabs2(r);
            bb = zabs2(bv);
        }
        r32[fs + (size_t)y + (size_t)ny * xi] = c_from(r);
    }
    // warp-level partial sums, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        bb += __shfl_xor_sync(0xffffffffu, bb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (rr != 0) atomicAdd(&rnorm2[s], rr);
        if (bnorm2 && bb != 0) atomicAdd(&bnorm2[s], bb);
    }
}

void residual_launch(const Coefs<double2> &co, const SrcView &b, const double2 *x, int S, bool adjoint, float2 *r32,
                     double *rnorm2, double *bnorm2, cudaStream_t st) {
    WUST_CUDA(cudaMemsetAsync(rnorm2, 0, sizeof(double) * S, st));
    if (bnorm2) WUST_CUDA(cudaMemsetAsync(bnorm2, 0, sizeof(double) * S, st));
    dim3 grid(ceil_div(co.ny, 128), co.nx, S);
    if (adjoint) residual_kernel<true><<<grid, 128, 0, st>>>(co, b, x, S, r32, rnorm2, bnorm2);
    else residual_kernel<false><<<grid, 128, 0, st>>>(co, b, x, S, r32, rnorm2, bnorm2);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

__global__ void promote_kernel(const float2 *u, double2 *x, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = z_from(u[i]);
}
// x += d over one source plane per blockIdx.y; per-source ||d||^2 and ||x||^2.
__global__ void accumulate_kernel(const float2 *d, double2 *x, size_t plane, double *dnorm2, double *xnorm2) {
    const int s = blockIdx.y;
    const float2 *ds = d + plane * s;
    double2 *xs = x + plane * s;
    double dd = 0, xx = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
        const double2 a = xs[i];
        const float2 b = ds[i];
        const double2 v = make_double2(a.x + (double)b.x, a.y + (double)b.y);
        xs[i] = v;
        dd += (double)b.x * b.x + (double)b.y * b.y;
        xx += v.x * v.x + v.y * v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dd += __shfl_xor_sync(0xffffffffu, dd, o);
        xx += __shfl_xor_sync(0xffffffffu, xx, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&dnorm2[s], dd);
        atomicAdd(&xnorm2[s], xx);
    }
}
__global__ void demote_kernel(const double2 *x, float2 *u, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        u[i] = c_from(x[i]);
}

static int elementwise_grid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 32); }

void promote_launch(const float2 *u, double2 *x, size_t n, cudaStream_t st) {
    promote_kernel<<<elementwise_grid(n), 256, 0, st>>>(u, x, n);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}
void accumulate_launch(const float2 *d, double2 *x, size_t plane, int S, double *dnorm2, double *xnorm2,
                       cudaStream_t st) {
    WUST_CUDA(cudaMemsetAsync(dnorm2, 0, sizeof(double) * S, st));
    WUST_CUDA(cudaMemsetAsync(xnorm2, 0, sizeof(double) * S, st));
    dim3 grid((unsigned)std::min<size_t>((plane + 255) / 256, 64), S);
    accumulate_kernel<<<grid, 256, 0, st>>>(d, x, plane, dnorm2, xnorm2);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}
void demote_launch(const double2 *x, float2 *u, size_t n, cudaStream_t st) {
    demote_kernel<<<elementwise_grid(n), 256, 0, st>>>(x, u, n);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
