// Per-frequency objective pieces on the GPU (Runtime/matlab/wust_oracle.m,
// Runtime/matlab/directional_curvature.m, HelmholtzSolver.massApply):
//   fit_kernel          receiver gather, masked source fit a = p^H d / p^H p,
//                       residual, 0.5 |r|^2 (wust_oracle.m:43-61), FP64 sums
//   gradient_kernel     g += sum_s -Re(conj(a_s v_s) .* M^T lam_s), with the
//                       mass stencil's border zeroed first (wust_oracle.m:66-68,
//                       HelmholtzSolver.m:211-215); FP64 accumulation over s
//   mass_apply_kernel   massApply forward/adjoint (HelmholtzSolver.m:205-220)
//   curvature kernels   massApply(v .* direction) and sum |a u(rx) mask|^2
//                       (directional_curvature.m:12-20)
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

// ---------------------------------------------------------------------------
// block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int NT>
__device__ double block_sum(double v, double *sh) {
    v = warp_sum(v);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
    if (w == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

constexpr int FIT_THREADS = 256;

__global__ void __launch_bounds__(FIT_THREADS) fit_kernel(FitParams p) {
    __shared__ double sh[FIT_THREADS / 32];
    const int s = blockIdx.x;
    const int t = p.first_tx + s;
    const size_t off = (size_t)p.ny * p.nx * s;
    // The misfit residual is a small difference of the field at the receivers,
    // so refined solves are gathered from their FP64 accumulator.
    auto field = [&](int r) -> double2 {
        const int32_t q = p.rx_lin[r];
        return p.u64 ? p.u64[off + q] : z_from(p.u[off + q]);
    };
    double den = 0, nre = 0, nim = 0;
    for (int r = threadIdx.x; r < p.n_rx; r += FIT_THREADS) {
        const double m = p.mask[t + (size_t)p.n_tx * r] ? 1.0 : 0.0;
        const double2 pm = zscale(m, field(r));
        const double2 dm = zscale(m, z_from(p.Y[t + (size_t)p.n_tx * r]));
        den += zabs2(pm);
        nre += pm.x * dm.x + pm.y * dm.y;    // conj(pm) * dm
        nim += pm.x * dm.y - pm.y * dm.x;
    }
    den = block_sum<FIT_THREADS>(den, sh);
    nre = block_sum<FIT_THREADS>(nre, sh);
    nim = block_sum<FIT_THREADS>(nim, sh);
    const bool ok = isfinite(den) && den > 2.2250738585072014e-308 && isfinite(nre) && isfinite(nim);
    const double2 a = ok ? make_double2(nre / den, nim / den) : make_double2(0.0, 0.0);
    if (!ok || !isfinite(a.x) || !isfinite(a.y)) {
        if (threadIdx.x == 0) atomicCAS(p.status, 0, t + 1);
    }
    double loss = 0;
    for (int r = threadIdx.x; r < p.n_rx; r += FIT_THREADS) {
        const double m = p.mask[t + (size_t)p.n_tx * r] ? 1.0 : 0.0;
        const double2 pm = zscale(m, field(r));
        const double2 dm = zscale(m, z_from(p.Y[t + (size_t)p.n_tx * r]));
        const double2 res = zscale(m, zsub(zmul(pm, a), dm));
        loss += zabs2(res);
        p.residual[r + (size_t)p.n_rx * s] = c_from(res);
    }
    loss = block_sum<FIT_THREADS>(loss, sh);
    if (threadIdx.x == 0) {
        p.scale[s] = a;
        p.loss_per_src[s] = 0.5 * loss;
    }
}

void fit_launch(const FitParams &p, cudaStream_t st) {
    fit_kernel<<<p.nb, FIT_THREADS, 0, st>>>(p);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// 3x3 mass stencil tiles.  The kernel is symmetric, so convn and correlation
// coincide: w = [e/4 d/4 e/4; d/4 1-d-e d/4; e/4 d/4 e/4].
// ---------------------------------------------------------------------------
constexpr int TY = 32, TX = 8;

__device__ __forceinline__ double mass_w(int dy, int dx, double d, double e) {
    const int a = (dy != 0) + (dx != 0);
    return a == 0 ? 1.0 - d - e : (a == 1 ? d / 4 : e / 4);
}

__device__ __forceinline__ bool on_ring(int y, int x, int ny, int nx) {
    return y == 0 || x == 0 || y == ny - 1 || x == nx - 1;
}

// One thread per grid point of a 32 x 8 tile, all sources in order (the sum
// over s is the same at every point on every run).  The lambda tile with its
// one-point halo is double-buffered in shared memory; the halo values and
// field value of the source two ahead are loaded into registers while the
// current source is computed, so each source costs one barrier and its loads
// have two sources' time to land.
__global__ void __launch_bounds__(TY * TX) gradient_kernel(const float2 *u, const float2 *lam, const double2 *mult,
                                                           const double2 *scale, int ny, int nx, int nb, double d,
                                                           double e, double *grad) {
    constexpr int kHalo = (TY + 2) * (TX + 2);
    constexpr int kPer = (kHalo + TY * TX - 1) / (TY * TX);    // halo entries per thread
    __shared__ float2 L[2][TX + 2][TY + 2];
    const int ty = threadIdx.x % TY, tx = threadIdx.x / TY;
    const int y0 = blockIdx.x * TY, x0 = blockIdx.y * TX;
    const int y = y0 + ty, x = x0 + tx;
    const bool inside = (y < ny && x < nx);
    const size_t idx = (size_t)y + (size_t)ny * x;
    const double2 m = inside ? mult[idx] : make_double2(0.0, 0.0);
    double w[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) w[a][b] = mass_w(a - 1, b - 1, d, e);
    // this thread's halo entries: offset in a source plane, or -1 (outside the
    // tile's halo, or on the Dirichlet ring, which the adjoint massApply zeroes
    // before the convolution)
    long long hoff[kPer];
    int hl[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int q = threadIdx.x + TY * TX * k;
        const int ly = q % (TY + 2), lx = q / (TY + 2);
        const int gy = y0 + ly - 1, gx = x0 + lx - 1;
        hl[k] = q < kHalo ? lx * (TY + 2) + ly : -1;
        hoff[k] = (q < kHalo && gy > 0 && gx > 0 && gy < ny - 1 && gx < nx - 1) ? (long long)gy + (long long)ny * gx
                                                                                 : -1;
    }
    const size_t fs = (size_t)ny * nx;
    // two register sets: the next source (stashed after this one's
    // arithmetic) and the one after it (loading meanwhile)
    float2 hA[kPer], hB[kPer], uA = make_float2(0.f, 0.f), uB = make_float2(0.f, 0.f);
    auto fetch = [&](int s, float2 (&hv)[kPer], float2 &uv) {
#pragma unroll
        for (int k = 0; k < kPer; ++k)
            hv[k] = hoff[k] >= 0 ? lam[fs * s + (size_t)hoff[k]] : make_float2(0.f, 0.f);
        uv = inside ? u[fs * s + idx] : make_float2(0.f, 0.f);
    };
    auto stash = [&](int buf, const float2 (&hv)[kPer]) {
        float2 *Lb = &L[buf][0][0];
#pragma unroll
        for (int k = 0; k < kPer; ++k)
            if (hl[k] >= 0) Lb[hl[k]] = hv[k];
    };
    double acc = 0;
    float2 ucur = make_float2(0.f, 0.f);
    if (nb > 0) {
        fetch(0, hA, uA);
        stash(0, hA);
        ucur = uA;
    }
    if (nb > 1) fetch(1, hB, uB);
    __syncthreads();
    // source s from L[s & 1]; hn/un hold source s+1, hf/uf take source s+2
    auto body = [&](int s, const float2 (&hn)[kPer], const float2 &un, float2 (&hf)[kPer], float2 &uf) {
        const int cur = s & 1;
        if (s + 2 < nb) fetch(s + 2, hf, uf);       // in flight during two sources' arithmetic
        if (inside) {
            double2 ml = make_double2(0.0, 0.0);
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const float2 v = L[cur][tx + b][ty + a];
                    ml.x += w[a][b] * (double)v.x;
                    ml.y += w[a][b] * (double)v.y;
                }
            const double2 av = zmul(scale[s], zmul(m, z_from(ucur)));
            acc -= av.x * ml.x + av.y * ml.y;    // -Re(conj(av) * ml)
        }
        if (s + 1 < nb) {
            stash(cur ^ 1, hn);                     // last read in the previous source, before its barrier
            ucur = un;
        }
        __syncthreads();
    };
    for (int s = 0; s < nb; s += 2) {
        body(s, hB, uB, hA, uA);
        if (s + 1 < nb) body(s + 1, hA, uA, hB, uB);
    }
    if (inside) grad[idx] += acc;
}

void gradient_launch(const float2 *u, const float2 *lam, const double2 *mult, const double2 *scale, int ny, int nx,
                     int nb, double d, double e, double *grad, cudaStream_t st) {
    dim3 grid(ceil_div(ny, TY), ceil_div(nx, TX));
    gradient_kernel<<<grid, TY * TX, 0, st>>>(u, lam, mult, scale, ny, nx, nb, d, e, grad);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

// out(:,:,s) = massApply(v(:,:,s) [.* mult .* dir], adjoint)
template <bool CURV>
__global__ void __launch_bounds__(TY * TX) mass_kernel(const float2 *v, const double2 *mult, const double *dir,
                                                       float2 *out, int ny, int nx, int n, double d, double e,
                                                       bool adjoint) {
    __shared__ float2 V[TX + 2][TY + 2];
    const int ty = threadIdx.x % TY, tx = threadIdx.x / TY;
    const int y0 = blockIdx.x * TY, x0 = blockIdx.y * TX;
    const int y = y0 + ty, x = x0 + tx;
    const int s = blockIdx.z;
    const size_t fs = (size_t)ny * nx * s;
    for (int q = threadIdx.x; q < (TY + 2) * (TX + 2); q += TY * TX) {
        const int ly = q % (TY + 2), lx = q / (TY + 2);
        const int gy = y0 + ly - 1, gx = x0 + lx - 1;
        float2 val = make_float2(0.f, 0.f);
        if (gy >= 0 && gx >= 0 && gy < ny && gx < nx && !(adjoint && on_ring(gy, gx, ny, nx))) {
            const size_t gi = (size_t)gy + (size_t)ny * gx;
            if (CURV) {
                const double2 w = zscale(dir[gi], zmul(mult[gi], z_from(v[fs + gi])));
                val = c_from(w);
            } else {
                val = v[fs + gi];
            }
        }
        V[lx][ly] = val;
    }
    __syncthreads();
    if (y >= ny || x >= nx) return;
    float2 acc = make_float2(0.f, 0.f);
    if (adjoint || !on_ring(y, x, ny, nx)) {
        const float c0 = (float)(1.0 - d - e), c1 = (float)(d / 4), c2 = (float)(e / 4);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int k = (a != 1) + (b != 1);
                const float wgt = k == 0 ? c0 : (k == 1 ? c1 : c2);
                const float2 t = V[tx + b][ty + a];
                acc.x = fmaf(wgt, t.x, acc.x);
                acc.y = fmaf(wgt, t.y, acc.y);
            }
    }
    out[fs + (size_t)y + (size_t)ny * x] = acc;
}

void mass_apply_launch(const float2 *v, float2 *out, int ny, int nx, int n, double d, double e, bool adjoint,
                       cudaStream_t st) {
    dim3 grid(ceil_div(ny, TY), ceil_div(nx, TX), n);
    mass_kernel<false><<<grid, TY * TX, 0, st>>>(v, nullptr, nullptr, out, ny, nx, n, d, e, adjoint);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

void curvature_source_launch(const float2 *u, const double2 *mult, const double *direction, float2 *out, int ny,
                             int nx, int nb, double d, double e, cudaStream_t st) {
    dim3 grid(ceil_div(ny, TY), ceil_div(nx, TX), nb);
    mass_kernel<true><<<grid, TY * TX, 0, st>>>(u, mult, direction, out, ny, nx, nb, d, e, false);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

__global__ void __launch_bounds__(FIT_THREADS) curvature_reduce_kernel(const float2 *u, const int32_t *rx_lin,
                                                                       const uint8_t *mask, const double2 *scale,
                                                                       int n_tx, int n_rx, int first_tx, int ny,
                                                                       int nx, double *out) {
    __shared__ double sh[FIT_THREADS / 32];
    const int s = blockIdx.x, t = first_tx + s;
    const float2 *us = u + (size_t)ny * nx * s;
    double acc = 0;
    for (int r = threadIdx.x; r < n_rx; r += FIT_THREADS) {
        if (!mask[t + (size_t)n_tx * r]) continue;
        const double2 v = zmul(z_from(us[rx_lin[r]]), scale[s]);
        acc += zabs2(v);
    }
    acc = block_sum<FIT_THREADS>(acc, sh);
    if (threadIdx.x == 0) out[s] = acc;
}

void curvature_reduce_launch(const float2 *u, const int32_t *rx_lin, const uint8_t *mask, const double2 *scale,
                             int n_tx, int n_rx, int first_tx, int nb, int ny, int nx, double *out, cudaStream_t st) {
    curvature_reduce_kernel<<<nb, FIT_THREADS, 0, st>>>(u, rx_lin, mask, scale, n_tx, n_rx, first_tx, ny, nx, out);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

// The linearized residual of the Gauss-Newton product (source scales frozen,
// directional_curvature.m:12-20): q = J d = -a (H^{-1} M (v .* d))(rx) .* mask,
// written as the adjoint right-hand side of J^H q, with ||q||^2 per source.
__global__ void __launch_bounds__(FIT_THREADS) linearized_residual_kernel(const float2 *u, const int32_t *rx_lin,
                                                                          const uint8_t *mask, const double2 *scale,
                                                                          int n_tx, int n_rx, int first_tx, int ny,
                                                                          int nx, float2 *resid, double *out) {
    __shared__ double sh[FIT_THREADS / 32];
    const int s = blockIdx.x, t = first_tx + s;
    const float2 *us = u + (size_t)ny * nx * s;
    double acc = 0;
    for (int r = threadIdx.x; r < n_rx; r += FIT_THREADS) {
        double2 q = make_double2(0.0, 0.0);
        if (mask[t + (size_t)n_tx * r]) {
            const double2 v = zmul(z_from(us[rx_lin[r]]), scale[s]);
            q = make_double2(-v.x, -v.y);
            acc += zabs2(q);
        }
        resid[r + (size_t)n_rx * s] = c_from(q);
    }
    acc = block_sum<FIT_THREADS>(acc, sh);
    if (threadIdx.x == 0) out[s] = acc;
}

void linearized_residual_launch(const float2 *u, const int32_t *rx_lin, const uint8_t *mask, const double2 *scale,
                                int n_tx, int n_rx, int first_tx, int nb, int ny, int nx, float2 *resid, double *out,
                                cudaStream_t st) {
    linearized_residual_kernel<<<nb, FIT_THREADS, 0, st>>>(u, rx_lin, mask, scale, n_tx, n_rx, first_tx, ny, nx,
                                                           resid, out);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

__global__ void virtual_source_kernel(const float2 *u, const double2 *mult, float2 *virt, size_t plane, size_t total) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        virt[i] = c_from(zmul(mult[i % plane], z_from(u[i])));
}

void virtual_source_launch(const float2 *u, const double2 *mult, float2 *virt, int ny, int nx, int n, cudaStream_t st) {
    const size_t plane = (size_t)ny * nx, total = plane * n;
    const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    virtual_source_kernel<<<grid, 256, 0, st>>>(u, mult, virt, plane, total);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
