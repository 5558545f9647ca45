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
//
// One kernel does each refinement step's elementwise work in one pass over
// the fields:
//   RF_FIRST     r_0 = b - H u, with x_0 = u the solve's c64 field
//   RF_STEP_C64  x_1 = u + d in FP64, r_1 = b - H x_1 (u read from the
//                solve's output, which this step leaves alone)
//   RF_STEP      x_{k+1} = x_k + d (into the other FP64 buffer), the c64
//                copy of x_{k+1} into the solve's output, r = b - H x_{k+1}
// with the per-source squared norms of r, b (first step) and d, x (later
// steps).  A block owns a tile of up to 94 grid rows, 8 sources and a strip
// of about 48 columns; two threads per row take 4 sources each.  It walks
// the strip with cp.async: a ring of four field columns (three, with the
// rows above and below the tile, feed the nine taps while the fourth
// loads) and a ring of two columns of per-row data (the nine weights, and
// the dense sources or receiver slots), so no load is waited for in the
// column it is used.  Every field value is read from HBM once per block
// plus its halo; the weights of a column are read once per block for its 8
// sources, as one contiguous run of the interleaved weight array that
// refine_weights_kernel builds after each assembly ([x][y][9] complex128,
// for H and, conjugated, for H^H; zero for taps that leave the grid).
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

namespace {

constexpr int kRfRowThreads = 96;                  // threads per source half: one per grid row of the tile
constexpr int kRfThreads = 2 * kRfRowThreads;
constexpr int kRfRows = 94;                        // rows per tile at most: shared memory of two blocks per SM
constexpr int kRfSrc = 8;                          // sources per block
constexpr int kRfHalf = kRfSrc / 2;                // sources per thread
constexpr int kRfSlots = 4;                        // field ring
constexpr int kRfCols = 48;                        // target strip width
constexpr int kFieldIter = (kRfSrc * (kRfRows + 2) + kRfThreads - 1) / kRfThreads;   // field entries per thread
constexpr int kWeightIter = (9 * kRfRows + kRfThreads - 1) / kRfThreads;             // weight entries per thread

enum RefineMode { RF_FIRST = 0, RF_STEP_C64 = 1, RF_STEP = 2 };

struct RefineParams {
    int ny, nx;
    const double2 *w9;      // interleaved weights [x][y][9] of H or H^H
    SrcView b;
    const float2 *u;        // first step: the solve's field; later steps: the correction d
    const float2 *x_old32;  // RF_STEP_C64: x_0, c64
    const double2 *x_old;   // RF_STEP: x_k
    double2 *x_new;         // steps: x_{k+1}, every grid point
    float2 *out;            // RF_STEP: c64 copy of x_{k+1}, every grid point
    float2 *r32;            // residual, c64, every grid point (zero on rows 0 and ny-1)
    double *rnorm2, *bnorm2, *dnorm2, *xnorm2;
    int S, R, TX;
};

size_t refine_smem_bytes(int R) {
    const size_t RS = (size_t)R + 2;
    return (size_t)kRfSlots * kRfSrc * RS * (sizeof(double2) + sizeof(float2)) +
           2 * ((size_t)9 * R * sizeof(double2) + (size_t)kRfSrc * R * sizeof(float2) + (size_t)R * sizeof(int));
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Tap t of row y couples to grid point (y + tap_dy(t), xi + tap_dx(t)).
template <bool ADJ>
__host__ __device__ constexpr int tap_dy(int t) {
    return ADJ ? (t == 1 || t == 4 || t == 7 ? 1 : t == 2 || t == 5 || t == 8 ? -1 : 0)
               : (t == 1 || t == 4 || t == 7 ? -1 : t == 2 || t == 5 || t == 8 ? 1 : 0);
}
template <bool ADJ>
__host__ __device__ constexpr int tap_dx(int t) {
    return ADJ ? (t >= 3 && t <= 5 ? 1 : t >= 6 ? -1 : 0) : (t >= 3 && t <= 5 ? -1 : t >= 6 ? 1 : 0);
}

// Where weight t of row y (1 <= y <= ny-2) at column xi lives: H's row, or
// for H^H (conjugated on use) H's column; null for taps that leave the grid.
template <bool ADJ>
__device__ __forceinline__ const double2 *weight_ptr(const Coefs<double2> &co, int t, int y, int xi) {
    const size_t ny = co.ny, n1 = co.ny - 1;
    const bool xl = xi >= 1, xr = xi <= co.nx - 2;
    if (!ADJ) {
        switch (t) {
            case 0: return co.Dd + y + ny * xi;
            case 1: return co.Dl + (y - 1) + n1 * xi;
            case 2: return co.Du + y + n1 * xi;
            case 3: return xl ? co.Ld + y + ny * (xi - 1) : nullptr;
            case 4: return xl ? co.Ll + (y - 1) + n1 * (xi - 1) : nullptr;
            case 5: return xl ? co.Lu + y + n1 * (xi - 1) : nullptr;
            case 6: return xr ? co.Ud + y + ny * xi : nullptr;
            case 7: return xr ? co.Ul + (y - 1) + n1 * xi : nullptr;
            default: return xr ? co.Uu + y + n1 * xi : nullptr;
        }
    }
    switch (t) {
        case 0: return co.Dd + y + ny * xi;
        case 1: return co.Dl + y + n1 * xi;
        case 2: return co.Du + (y - 1) + n1 * xi;
        case 3: return xr ? co.Ld + y + ny * xi : nullptr;
        case 4: return xr ? co.Ll + y + n1 * xi : nullptr;
        case 5: return xr ? co.Lu + (y - 1) + n1 * xi : nullptr;
        case 6: return xl ? co.Ud + y + ny * (xi - 1) : nullptr;
        case 7: return xl ? co.Ul + y + n1 * (xi - 1) : nullptr;
        default: return xl ? co.Uu + (y - 1) + n1 * (xi - 1) : nullptr;
    }
}

// The nine weights of every grid point, interleaved: w9f for H's rows, w9a
// for H^H's rows (conjugates of H's columns); zero on rows 0 and ny-1.
__global__ void refine_weights_kernel(Coefs<double2> co, double2 *w9f, double2 *w9a) {
    const int ny = co.ny;
    const size_t n = (size_t)ny * co.nx;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(idx % ny), c = (int)(idx / ny);
        double2 *f = w9f + 9 * idx, *a = w9a + 9 * idx;
        const bool row_ok = y >= 1 && y <= ny - 2;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const double2 *pf = row_ok ? weight_ptr<false>(co, t, y, c) : nullptr;
            const double2 *pa = row_ok ? weight_ptr<true>(co, t, y, c) : nullptr;
            f[t] = pf ? *pf : make_double2(0.0, 0.0);
            a[t] = pa ? zconj(*pa) : make_double2(0.0, 0.0);
        }
    }
}

template <bool ADJ, int MODE>
__global__ void __launch_bounds__(kRfThreads, 2) refine_kernel(const RefineParams p) {
    constexpr bool STEP = MODE != RF_FIRST;
    extern __shared__ __align__(16) uint8_t rf_smem[];
    const int ny = p.ny, nx = p.nx, S = p.S, R = p.R;
    const int RS = R + 2;                                      // slot rows: the tile and one row above and below
    double2 *X = reinterpret_cast<double2 *>(rf_smem);         // [4][source][RS] FP64 x
    float2 *D = reinterpret_cast<float2 *>(X + (size_t)kRfSlots * kRfSrc * RS);   // [4][source][RS] u or d
    double2 *Wt = reinterpret_cast<double2 *>(D + (size_t)kRfSlots * kRfSrc * RS); // [2][R][9] weights
    float2 *Bd = reinterpret_cast<float2 *>(Wt + (size_t)2 * 9 * R);              // [2][source][R] dense b
    int *At = reinterpret_cast<int *>(Bd + (size_t)2 * kRfSrc * R);                // [2][R] receiver slot
    const int tid = threadIdx.x;
    const int row = tid % kRfRowThreads, half = tid / kRfRowThreads;
    const int y0 = 1 + blockIdx.x * R;                         // first row of the tile
    const int s0 = blockIdx.y * kRfSrc;
    const int x0 = blockIdx.z * p.TX, x1 = min(nx, x0 + p.TX);
    const int W = x1 - x0;                                     // columns computed; x0-1 .. x1 are loaded
    const size_t plane = (size_t)ny * nx;
    const int y = y0 + row;
    const bool row_ok = row < R && y <= ny - 2;
    const int mode = p.b.mode;

    // this thread's field entries e = tid + kRfThreads m of a ring column:
    // source q and slot row i packed as q * 256 + i, or -1
    int fqi[kFieldIter];
#pragma unroll
    for (int m = 0; m < kFieldIter; ++m) {
        const int e = tid + kRfThreads * m;
        fqi[m] = e < kRfSrc * RS ? (e / RS) * 256 + e % RS : -1;
    }
    // field column k of the ring is grid column x0 - 1 + k
    auto issue_field = [&](int k) {
        const int c = x0 - 1 + k;
        const int sl = k % kRfSlots;
        const bool col_ok = c >= 0 && c < nx;
#pragma unroll
        for (int m = 0; m < kFieldIter; ++m) {
            if (fqi[m] < 0) continue;
            const int q = fqi[m] >> 8, i = fqi[m] & 255;
            const int yy = y0 - 1 + i, s = s0 + q;
            const int o = (sl * kRfSrc + q) * RS + i;
            if (col_ok && yy < ny && s < S) {
                const size_t g = (size_t)yy + (size_t)ny * c + plane * s;
                cp_async8(D + o, p.u + g);
                if (MODE == RF_STEP) cp_async16(X + o, p.x_old + g);
                if (MODE == RF_STEP_C64) cp_async8(X + o, p.x_old32 + g);   // first half of the slot
            } else {
                D[o] = make_float2(0.f, 0.f);
                if (STEP) X[o] = make_double2(0.0, 0.0);
            }
        }
    };
    // the entries this thread loaded: x = x_old + d, or x = u (FP64 sums)
    auto convert = [&](int k) {
        const int sl = k % kRfSlots;
#pragma unroll
        for (int m = 0; m < kFieldIter; ++m) {
            if (fqi[m] < 0) continue;
            const int o = (sl * kRfSrc + (fqi[m] >> 8)) * RS + (fqi[m] & 255);
            const float2 dv = D[o];
            if (MODE == RF_STEP) {
                const double2 xv = X[o];
                X[o] = make_double2(xv.x + (double)dv.x, xv.y + (double)dv.y);
            } else if (MODE == RF_STEP_C64) {
                const float2 xv = *reinterpret_cast<const float2 *>(X + o);
                X[o] = make_double2((double)xv.x + (double)dv.x, (double)xv.y + (double)dv.y);
            } else {
                X[o] = z_from(dv);
            }
        }
    };
    // per-row data of computed column k: weights, dense sources, receiver slots
    auto issue_rows = [&](int k) {
        const int c = x0 - 1 + k;
        const int sl = k & 1;
        const double2 *wsrc = p.w9 + ((size_t)ny * c + y0) * 9;      // rows y0 .. of column c, contiguous
        double2 *wdst = Wt + sl * 9 * R;
#pragma unroll
        for (int m = 0; m < kWeightIter; ++m) {
            const int e = tid + kRfThreads * m;
            if (e >= 9 * R) break;
            if (y0 + e / 9 <= ny - 2) cp_async16(wdst + e, wsrc + e);
            else wdst[e] = make_double2(0.0, 0.0);
        }
        if (mode == SRC_DENSE) {
            for (int e = tid; e < kRfSrc * R; e += kRfThreads) {
                const int q = e / R, i = e - q * R;
                const int yy = y0 + i, s = s0 + q;
                float2 *dst = Bd + sl * kRfSrc * R + e;
                if (yy <= ny - 2 && s < S) cp_async8(dst, p.b.dense + (size_t)yy + (size_t)ny * c + plane * s);
                else *dst = make_float2(0.f, 0.f);
            }
        } else if (mode == SRC_SCATTER) {
            for (int i = tid; i < R; i += kRfThreads) {
                const int yy = y0 + i;
                if (yy <= ny - 2) cp_async4(At + sl * R + i, p.b.at + (size_t)yy + (size_t)ny * c);
                else At[sl * R + i] = -1;
            }
        }
    };

    int lin[kRfHalf];                                          // point sources: linear index per source
#pragma unroll
    for (int j = 0; j < kRfHalf; ++j) {
        const int s = s0 + half * kRfHalf + j;
        lin[j] = (mode == SRC_POINT && s < S) ? p.b.lin[s] : -1;
    }
    double rn[kRfHalf], an[kRfHalf], xn[kRfHalf];   // |r|^2; |b|^2 (first) or |d|^2 (later); |x|^2 (later)
#pragma unroll
    for (int j = 0; j < kRfHalf; ++j) rn[j] = an[j] = xn[j] = 0.0;

    issue_field(0);
    cp_async_commit();
    issue_field(1);
    cp_async_commit();
    issue_field(2);
    issue_rows(1);
    cp_async_commit();
    cp_async_wait<1>();
    convert(0);
    convert(1);
    for (int k = 1; k <= W; ++k) {
        const int c = x0 - 1 + k;
        cp_async_wait<0>();
        convert(k + 1);
        __syncthreads();          // field columns k-1 .. k+1 and row data k ready; older slots free
        if (k + 2 <= W + 1) issue_field(k + 2);
        if (k + 1 <= W) issue_rows(k + 1);
        cp_async_commit();
        if (row_ok) {
            const int slm = (k - 1) % kRfSlots, sl0 = k % kRfSlots, slp = (k + 1) % kRfSlots, slr = k & 1;
            double2 w[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) w[t] = Wt[slr * 9 * R + row * 9 + t];
            const int at = mode == SRC_SCATTER ? At[slr * R + row] : -1;
            const int pt = y + ny * c;
            const bool interior = c >= 1 && c <= nx - 2;
            // element (y, c) of this thread's first source, then one plane per source
            const size_t oc = (size_t)y + (size_t)ny * c + plane * (size_t)(s0 + half * kRfHalf);
#pragma unroll
            for (int j = 0; j < kRfHalf; ++j) {
                const int q = half * kRfHalf + j, s = s0 + q;
                if (s >= S) break;
                const double2 *cm = X + (slm * kRfSrc + q) * RS + row + 1;   // row y of column c-1
                const double2 *c0 = X + (sl0 * kRfSrc + q) * RS + row + 1;
                const double2 *cp = X + (slp * kRfSrc + q) * RS + row + 1;
                // h = sum_t w_t v_t as four independent real sums
                double hrr = 0.0, hii = 0.0, hri = 0.0, hir = 0.0;
#pragma unroll
                for (int t = 0; t < 9; ++t) {
                    const int dx = tap_dx<ADJ>(t), dy = tap_dy<ADJ>(t);
                    const double2 v = (dx < 0 ? cm : dx > 0 ? cp : c0)[dy];
                    hrr = fma(w[t].x, v.x, hrr);
                    hii = fma(w[t].y, v.y, hii);
                    hri = fma(w[t].x, v.y, hri);
                    hir = fma(w[t].y, v.x, hir);
                }
                const double2 h = make_double2(hrr - hii, hri + hir);
                float2 bf = make_float2(0.f, 0.f);
                if (mode == SRC_POINT) {
                    if (lin[j] == pt) bf.x = 1.f;
                } else if (mode == SRC_DENSE) {
                    bf = Bd[(slr * kRfSrc + q) * R + row];
                } else if (mode == SRC_SCATTER) {
                    if (at >= 0) bf = p.b.vals[at + (size_t)p.b.n_slots * s];
                }
                const double2 bv = z_from(bf);
                const double2 rv = zsub(bv, h);
                const size_t o = oc + plane * j;
                p.r32[o] = c_from(rv);
                const double2 xv = c0[0];
                if (STEP) p.x_new[o] = xv;
                if (MODE == RF_STEP) p.out[o] = c_from(xv);
                if (interior) {
                    rn[j] += zabs2(rv);
                    if (STEP) {
                        const float2 dv = D[(sl0 * kRfSrc + q) * RS + row + 1];
                        an[j] += (double)dv.x * dv.x + (double)dv.y * dv.y;
                        xn[j] += zabs2(xv);
                    } else {
                        an[j] += zabs2(bv);
                    }
                }
                // the Dirichlet rows above and below carry x through, residual zero
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    if (y != (side == 0 ? 1 : ny - 2)) continue;
                    const int dyb = side == 0 ? -1 : 1;          // row 0 or ny-1
                    const double2 xb = c0[dyb];
                    p.r32[o + dyb] = make_float2(0.f, 0.f);
                    if (STEP) p.x_new[o + dyb] = xb;
                    if (MODE == RF_STEP) p.out[o + dyb] = c_from(xb);
                }
            }
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int j = 0; j < kRfHalf; ++j) {
        const int s = s0 + half * kRfHalf + j;
        double a = rn[j], bq = an[j], cq = xn[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            bq += __shfl_xor_sync(0xffffffffu, bq, o);
            cq += __shfl_xor_sync(0xffffffffu, cq, o);
        }
        if ((tid & 31) == 0 && s < S) {
            if (a != 0) atomicAdd(&p.rnorm2[s], a);
            if (STEP) {
                if (bq != 0) atomicAdd(&p.dnorm2[s], bq);
                if (cq != 0) atomicAdd(&p.xnorm2[s], cq);
            } else if (p.bnorm2 && bq != 0) {
                atomicAdd(&p.bnorm2[s], bq);
            }
        }
    }
}

template <bool ADJ, int MODE>
void refine_launch_one(const RefineParams &p, dim3 grid, size_t smem, cudaStream_t st) {
    // per launch: the attribute lives in the current device's context
    WUST_CUDA(cudaFuncSetAttribute(refine_kernel<ADJ, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)refine_smem_bytes(kRfRows)));
    refine_kernel<ADJ, MODE><<<grid, kRfThreads, smem, st>>>(p);
}

template <bool ADJ>
void refine_launch_mode(const RefineParams &p, int mode, dim3 grid, size_t smem, cudaStream_t st) {
    if (mode == RF_FIRST) refine_launch_one<ADJ, RF_FIRST>(p, grid, smem, st);
    else if (mode == RF_STEP_C64) refine_launch_one<ADJ, RF_STEP_C64>(p, grid, smem, st);
    else refine_launch_one<ADJ, RF_STEP>(p, grid, smem, st);
}

void refine_launch(RefineParams &p, bool adjoint, int mode, cudaStream_t st) {
    const bool step = mode != RF_FIRST;
    const int ny = p.ny, nx = p.nx;
    const int rows = ny - 2;
    const int row_tiles = ceil_div(rows, kRfRows);
    p.R = ceil_div(rows, row_tiles);
    const int strips = ceil_div(nx, kRfCols);
    p.TX = ceil_div(nx, strips);
    const dim3 grid(ceil_div(rows, p.R), ceil_div(p.S, kRfSrc), ceil_div(nx, p.TX));
    const size_t smem = refine_smem_bytes(p.R);
    WUST_CUDA(cudaMemsetAsync(p.rnorm2, 0, sizeof(double) * p.S, st));
    if (step) {
        WUST_CUDA(cudaMemsetAsync(p.dnorm2, 0, sizeof(double) * p.S, st));
        WUST_CUDA(cudaMemsetAsync(p.xnorm2, 0, sizeof(double) * p.S, st));
    } else if (p.bnorm2) {
        WUST_CUDA(cudaMemsetAsync(p.bnorm2, 0, sizeof(double) * p.S, st));
    }
    if (adjoint) refine_launch_mode<true>(p, mode, grid, smem, st);
    else refine_launch_mode<false>(p, mode, grid, smem, st);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

}  // namespace

void refine_weights_launch(const Coefs<double2> &co, double2 *w9f, double2 *w9a, cudaStream_t st) {
    const size_t n = (size_t)co.ny * co.nx;
    refine_weights_kernel<<<(int)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(co, w9f, w9a);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

__global__ void demote_kernel(const double2 *x, float2 *u, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        u[i] = c_from(x[i]);
}

void refine_demote_launch(const double2 *x, float2 *u, size_t n, cudaStream_t st) {
    demote_kernel<<<(int)std::min<size_t>((n + 255) / 256, 148 * 32), 256, 0, st>>>(x, u, n);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

void refine_first_launch(const RefineWeights &w, const SrcView &b, const float2 *u, int S, bool adjoint,
                         float2 *r32, double *rnorm2, double *bnorm2, cudaStream_t st) {
    RefineParams p{};
    p.ny = w.ny;
    p.nx = w.nx;
    p.w9 = adjoint ? w.w9a : w.w9f;
    p.b = b;
    p.u = u;
    p.r32 = r32;
    p.rnorm2 = rnorm2;
    p.bnorm2 = bnorm2;
    p.S = S;
    refine_launch(p, adjoint, RF_FIRST, st);
}

void refine_step_launch(const RefineWeights &w, const SrcView &b, const float2 *d, const float2 *x_old32,
                        const double2 *x_old, int S, bool adjoint, double2 *x_new, float2 *out, float2 *r32,
                        double *rnorm2, double *dnorm2, double *xnorm2, cudaStream_t st) {
    if ((x_old32 == nullptr) == (x_old == nullptr) || (x_old32 && out) || (x_old && !out))
        fail(WUST_ERR_RUNTIME, "refinement step: one previous iterate (c64 without output, FP64 with output)");
    RefineParams p{};
    p.x_old32 = x_old32;
    p.ny = w.ny;
    p.nx = w.nx;
    p.w9 = adjoint ? w.w9a : w.w9f;
    p.b = b;
    p.u = d;
    p.x_old = x_old;
    p.x_new = x_new;
    p.out = out;
    p.r32 = r32;
    p.rnorm2 = rnorm2;
    p.dnorm2 = dnorm2;
    p.xnorm2 = xnorm2;
    p.S = S;
    refine_launch(p, adjoint, x_old32 ? RF_STEP_C64 : RF_STEP, st);
}

}  // namespace wust
