// FP64 residuals for iterative refinement of the block-LU solves.
//
// r = b - H x (or b - H^H x) with the complex128 coefficients, evaluated
// with the nine-point formula of the sparse assembly
// (HelmholtzSolver.m:118-135) and its conjugate transpose.  Rows on the top
// and bottom Dirichlet border (y = 0, Ny-1) are excluded: the block solver
// keeps them at zero (applyBlockLU.cu:10), so they never enter the other
// equations and cannot be corrected.  The norms that steer the refinement
// (residual, correction, solution) are taken over the interior grid only:
// the whole Dirichlet ring is zero in forward fields and is zeroed by M^T
// before an adjoint field is used, while the block adjoint leaves its own
// values there that a correction cannot settle.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int kResRows = 128;          // grid rows per block (one per thread)
constexpr int kResSrc = 8;             // sources per thread
constexpr int kResCols = 16;           // columns per block

// One thread per grid row y of a block's 16 columns and 8 sources: the nine
// coefficients (or their conjugates for H^H) of a point are loaded once and
// reused for the 8 sources; walking the columns keeps the neighbour columns'
// lines in L1; the per-source norms accumulate in registers and are reduced
// once per warp at the end.
template <bool ADJ>
__global__ void __launch_bounds__(kResRows) residual_kernel(Coefs<double2> co, SrcView b, const double2 *__restrict__ x,
                                                            int S, float2 *r32, double *rnorm2, double *bnorm2) {
    const int ny = co.ny, nx = co.nx;
    const int y = blockIdx.x * kResRows + threadIdx.x;
    const int s0 = blockIdx.y * kResSrc;
    const int x0 = blockIdx.z * kResCols, x1 = min(nx, x0 + kResCols);
    const bool active = (y >= 1 && y <= ny - 2);
    const size_t plane = (size_t)ny * nx;
    const double2 z = make_double2(0.0, 0.0);
    double rr[kResSrc], bb[kResSrc];
#pragma unroll
    for (int q = 0; q < kResSrc; ++q) { rr[q] = 0.0; bb[q] = 0.0; }
    for (int xi = x0; xi < x1; ++xi) {
        // stencil taps: neighbour offsets (dy, dx) and coefficients
        double2 w[9];
        int dyv[9], dxv[9];
        if (active) {
            const bool xl = xi >= 1, xr = xi <= nx - 2;
            if (!ADJ) {
                w[0] = co.dd(y, xi);               dyv[0] = 0;  dxv[0] = 0;
                w[1] = co.dl(y - 1, xi);           dyv[1] = -1; dxv[1] = 0;
                w[2] = co.du(y, xi);               dyv[2] = 1;  dxv[2] = 0;
                w[3] = xl ? co.ld(y, xi - 1) : z;      dyv[3] = 0;  dxv[3] = -1;
                w[4] = xl ? co.ll(y - 1, xi - 1) : z;  dyv[4] = -1; dxv[4] = -1;
                w[5] = xl ? co.lu(y, xi - 1) : z;      dyv[5] = 1;  dxv[5] = -1;
                w[6] = xr ? co.ud(y, xi) : z;          dyv[6] = 0;  dxv[6] = 1;
                w[7] = xr ? co.ul(y - 1, xi) : z;      dyv[7] = -1; dxv[7] = 1;
                w[8] = xr ? co.uu(y, xi) : z;          dyv[8] = 1;  dxv[8] = 1;
            } else {
                w[0] = zconj(co.dd(y, xi));            dyv[0] = 0;  dxv[0] = 0;
                w[1] = zconj(co.dl(y, xi));            dyv[1] = 1;  dxv[1] = 0;
                w[2] = zconj(co.du(y - 1, xi));        dyv[2] = -1; dxv[2] = 0;
                w[3] = xr ? zconj(co.ld(y, xi)) : z;          dyv[3] = 0;  dxv[3] = 1;
                w[4] = xr ? zconj(co.ll(y, xi)) : z;          dyv[4] = 1;  dxv[4] = 1;
                w[5] = xr ? zconj(co.lu(y - 1, xi)) : z;      dyv[5] = -1; dxv[5] = 1;
                w[6] = xl ? zconj(co.ud(y, xi - 1)) : z;      dyv[6] = 0;  dxv[6] = -1;
                w[7] = xl ? zconj(co.ul(y, xi - 1)) : z;      dyv[7] = 1;  dxv[7] = -1;
                w[8] = xl ? zconj(co.uu(y - 1, xi - 1)) : z;  dyv[8] = -1; dxv[8] = -1;
            }
            // taps that leave the grid have zero weight; clamp their index
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int xx = xi + dxv[t];
                if (xx < 0 || xx >= nx) { dxv[t] = 0; w[t] = z; }
            }
        }
        const size_t me = (size_t)y + (size_t)ny * xi;
        const bool interior = xi > 0 && xi < nx - 1;    // norms over the interior grid (see accumulate_kernel)
#pragma unroll
        for (int q = 0; q < kResSrc; ++q) {
            const int s = s0 + q;
            if (s >= S || y >= ny) continue;
            double2 r = z;
            if (active) {
                const double2 *xs = x + plane * s;
                double2 h = z;
#pragma unroll
                for (int t = 0; t < 9; ++t) {
                    const double2 v = __ldg(xs + (size_t)(y + dyv[t]) + (size_t)ny * (xi + dxv[t]));
                    h.x += w[t].x * v.x - w[t].y * v.y;
                    h.y += w[t].x * v.y + w[t].y * v.x;
                }
                const double2 bv = z_from(b.get(y, xi, s, ny, nx));
                r = zsub(bv, h);
                if (interior) {
                    rr[q] += zabs2(r);
                    bb[q] += zabs2(bv);
                }
            }
            r32[plane * s + me] = c_from(r);
        }
    }
#pragma unroll
    for (int q = 0; q < kResSrc; ++q) {
        double a = rr[q], c = bb[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if ((threadIdx.x & 31) == 0 && s0 + q < S) {
            if (a != 0) atomicAdd(&rnorm2[s0 + q], a);
            if (bnorm2 && c != 0) atomicAdd(&bnorm2[s0 + q], c);
        }
    }
}

void residual_launch(const Coefs<double2> &co, const SrcView &b, const double2 *x, int S, bool adjoint, float2 *r32,
                     double *rnorm2, double *bnorm2, cudaStream_t st) {
    WUST_CUDA(cudaMemsetAsync(rnorm2, 0, sizeof(double) * S, st));
    if (bnorm2) WUST_CUDA(cudaMemsetAsync(bnorm2, 0, sizeof(double) * S, st));
    dim3 grid(ceil_div(co.ny, kResRows), ceil_div(S, kResSrc), ceil_div(co.nx, kResCols));
    if (adjoint) residual_kernel<true><<<grid, kResRows, 0, st>>>(co, b, x, S, r32, rnorm2, bnorm2);
    else residual_kernel<false><<<grid, kResRows, 0, st>>>(co, b, x, S, r32, rnorm2, bnorm2);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

__global__ void promote_kernel(const float2 *u, double2 *x, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = z_from(u[i]);
}
// x += d over one source plane per blockIdx.y; per-source ||d||^2 and ||x||^2.
// Norms over the interior grid: the Dirichlet ring (rows 0, ny-1, columns 0,
// nx-1) is zero in forward fields and is zeroed by M^T before an adjoint
// field is used (HelmholtzSolver.m:211-219), so its values do not enter any
// result and do not decide when a refinement has converged.
__global__ void accumulate_kernel(const float2 *d, double2 *x, int ny, int nx, double *dnorm2, double *xnorm2) {
    const int s = blockIdx.y;
    const size_t plane = (size_t)ny * nx;
    const float2 *ds = d + plane * s;
    double2 *xs = x + plane * s;
    double dd = 0, xx = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
        const double2 a = xs[i];
        const float2 b = ds[i];
        const double2 v = make_double2(a.x + (double)b.x, a.y + (double)b.y);
        xs[i] = v;
        const int y = (int)(i % ny), xc = (int)(i / ny);
        if (y > 0 && y < ny - 1 && xc > 0 && xc < nx - 1) {
            dd += (double)b.x * b.x + (double)b.y * b.y;
            xx += v.x * v.x + v.y * v.y;
        }
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
void accumulate_launch(const float2 *d, double2 *x, int ny, int nx, int S, double *dnorm2, double *xnorm2,
                       cudaStream_t st) {
    const size_t plane = (size_t)ny * nx;
    WUST_CUDA(cudaMemsetAsync(dnorm2, 0, sizeof(double) * S, st));
    WUST_CUDA(cudaMemsetAsync(xnorm2, 0, sizeof(double) * S, st));
    dim3 grid((unsigned)std::min<size_t>((plane + 255) / 256, 64), S);
    accumulate_kernel<<<grid, 256, 0, st>>>(d, x, ny, nx, dnorm2, xnorm2);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}
void demote_launch(const double2 *x, float2 *u, size_t n, cudaStream_t st) {
    demote_kernel<<<elementwise_grid(n), 256, 0, st>>>(x, u, n);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
