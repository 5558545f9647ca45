// Batched forward and adjoint block-tridiagonal sweeps of applyBlockLU
// (Runtime/solver/applyBlockLU.cu:433-467), complex single on CUDA cores.
//
// Forward (H u = src):
//   j = 1..Nx-1 :  tmp = SRC_j - L_{j-1} u_{j-1};   u_j  = invT_j tmp       [stencil, GEMM]
//   j = Nx-2..0 :  tmp = U_j u_{j+1};               u_j -= invT_j tmp       [stencil, GEMM]
// Adjoint (H^H u = src):
//   j = 1..Nx-1 :  tmp = invT_{j-1}^H u_{j-1};      u_j  = SRC_j - U_{j-1}^H tmp   [GEMM, stencil]
//   j = Nx-2..0 :  tmp = u_j - L_j^H u_{j+1};       u_j  = invT_j^H tmp     [stencil, GEMM]
//
// Each column step is two launches: a tridiagonal stencil over (y, source)
// that writes the dense operand tmp, and a 32 x 32-tile complex GEMM over the
// interior rows (invT pages have zero borders) whose K loop prefetches the
// next A and B slabs into registers while the current slab is multiplied from
// double-buffered shared memory.  Threads run along y, so every field access
// is a contiguous, coalesced column segment.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int SBM = 32, SBN = 32, SBK = 32, STHREADS = 256;

struct SweepParams {
    Coefs<float2> co;
    const float2 *invT;
    float2 *u;          // [ny, nx, S]
    float2 *tmp;        // [ny, S]
    SrcView src;
    int ny, nx, S, j;
};

// ---------------------------------------------------------------------------
// Tridiagonal stencils (rows 1..ny-2 unless stated), one thread per (y, s).
// ---------------------------------------------------------------------------
enum StencilMode { ST_L = 0, ST_U = 1, ST_LH = 2, ST_UH = 3 };

template <int MODE>
__global__ void stencil_kernel(SweepParams p) {
    const int ny = p.ny, j = p.j;
    const int s = blockIdx.y;
    const size_t fs = (size_t)ny * p.nx * s;
    if (MODE == ST_UH) {
        // u(:, j, s) = SRC(:, j, s) - U_{j-1}^H tmp(:, s) on every row, border
        // included (applyBlockLU.cu:159-202)
        const int y = blockIdx.x * blockDim.x + threadIdx.x;
        if (y >= ny || s >= p.S) return;
        const float2 *t = p.tmp + (size_t)ny * s;
        float2 acc = make_float2(0.f, 0.f);
        cfma_conj(acc, p.co.ud(y, j - 1), t[y]);
        if (y > 0) cfma_conj(acc, p.co.uu(y - 1, j - 1), t[y - 1]);
        if (y < ny - 1) cfma_conj(acc, p.co.ul(y, j - 1), t[y + 1]);
        p.u[fs + (size_t)ny * j + y] = csub(p.src.get(y, j, s, ny, p.nx), acc);
        return;
    }
    const int y = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (y >= ny - 1 || s >= p.S) return;
    float2 out;
    if (MODE == ST_L) {          // SRC_j - L_{j-1} u_{j-1}   (applyBlockLU.cu:29-73)
        const float2 *uc = p.u + fs + (size_t)ny * (j - 1);
        float2 acc = cmul(p.co.ld(y, j - 1), uc[y]);
        cfma(acc, p.co.ll(y - 1, j - 1), uc[y - 1]);
        cfma(acc, p.co.lu(y, j - 1), uc[y + 1]);
        out = csub(p.src.get(y, j, s, ny, p.nx), acc);
    } else if (MODE == ST_U) {   // U_j u_{j+1}   (applyBlockLU.cu:95-137)
        const float2 *uc = p.u + fs + (size_t)ny * (j + 1);
        out = cmul(p.co.ud(y, j), uc[y]);
        cfma(out, p.co.ul(y - 1, j), uc[y - 1]);
        cfma(out, p.co.uu(y, j), uc[y + 1]);
    } else {                     // u_j - L_j^H u_{j+1}   (applyBlockLU.cu:224-267)
        const float2 *un = p.u + fs + (size_t)ny * (j + 1);
        float2 acc = make_float2(0.f, 0.f);
        cfma_conj(acc, p.co.ld(y, j), un[y]);
        cfma_conj(acc, p.co.lu(y - 1, j), un[y - 1]);
        cfma_conj(acc, p.co.ll(y, j), un[y + 1]);
        out = csub(p.u[fs + (size_t)ny * j + y], acc);
    }
    p.tmp[y + (size_t)ny * s] = out;
}

// ---------------------------------------------------------------------------
// C(r, s) (op)= op(A)(r, k) B(k, s) over interior r, k in [1, ny-1).
// A: one invT page, column-major ld ny; op = identity or conjugate transpose.
// B(k, s) = Bp[k + ldb * s]; C(r, s) = Cp[r + ldc * s].
// EPI: 0 store, 1 subtract; RING: also zero C rows 0 and ny-1.
// ---------------------------------------------------------------------------
template <bool CONJT, int EPI, bool RING>
__global__ void __launch_bounds__(STHREADS) cgemm_step_kernel(const float2 *__restrict__ A, const float2 *Bp,
                                                              size_t ldb, float2 *Cp, size_t ldc, int ny, int S) {
    __shared__ float2 As[2][SBK][SBM + 1];   // As[buf][k][r] = op(A)(r, k)
    __shared__ float2 Bs[2][SBK][SBN + 1];   // Bs[buf][k][s]
    const int tid = threadIdx.x, tr = tid % 16, tc = tid / 16;
    const int r0 = 1 + blockIdx.x * SBM;
    const int s0 = blockIdx.y * SBN;
    const int nslab = (ny - 2 + SBK - 1) / SBK;
    constexpr int PER = SBM * SBK / STHREADS;   // 4

    float2 ra[PER], rb[PER];
    auto fetch = [&](int slab) {
        const int k0 = 1 + slab * SBK;
#pragma unroll
        for (int m = 0; m < PER; ++m) {
            const int e = tid + m * STHREADS;
            int rr, kk;
            if (CONJT) { kk = e % SBK; rr = e / SBK; }
            else { rr = e % SBM; kk = e / SBM; }
            const int r = r0 + rr, k = k0 + kk;
            float2 v = make_float2(0.f, 0.f);
            if (r < ny - 1 && k < ny - 1) v = CONJT ? cconj(A[k + (size_t)ny * r]) : A[r + (size_t)ny * k];
            ra[m] = v;
            const int kb = e % SBK, sb = e / SBK;
            const int kg = k0 + kb, sg = s0 + sb;
            rb[m] = (kg < ny - 1 && sg < S) ? Bp[kg + ldb * sg] : make_float2(0.f, 0.f);
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int m = 0; m < PER; ++m) {
            const int e = tid + m * STHREADS;
            if (CONJT) As[buf][e % SBK][e / SBK] = ra[m];
            else As[buf][e / SBM][e % SBM] = ra[m];
            Bs[buf][e % SBK][e / SBK] = rb[m];
        }
    };

    float2 acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) acc[i][jj] = make_float2(0.f, 0.f);

    fetch(0);
    for (int slab = 0; slab < nslab; ++slab) {
        const int buf = slab & 1;
        stash(buf);
        __syncthreads();
        if (slab + 1 < nslab) fetch(slab + 1);
#pragma unroll 8
        for (int kk = 0; kk < SBK; ++kk) {
            const float2 a0 = As[buf][kk][tr], a1 = As[buf][kk][tr + 16];
            const float2 b0 = Bs[buf][kk][tc], b1 = Bs[buf][kk][tc + 16];
            cfma(acc[0][0], a0, b0);
            cfma(acc[0][1], a0, b1);
            cfma(acc[1][0], a1, b0);
            cfma(acc[1][1], a1, b1);
        }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const int r = r0 + tr + 16 * i, s = s0 + tc + 16 * jj;
            if (r >= ny - 1 || s >= S) continue;
            float2 *dst = Cp + r + ldc * s;
            *dst = (EPI == 1) ? csub(*dst, acc[i][jj]) : acc[i][jj];
        }
    }
    if (RING && blockIdx.x == 0 && tid < 2 * SBN) {
        const int s = s0 + tid / 2;
        if (s < S) Cp[((tid % 2) ? ny - 1 : 0) + ldc * s] = make_float2(0.f, 0.f);
    }
}

template <int MODE>
static void launch_stencil(const SweepParams &p, cudaStream_t st) {
    const int rows = (MODE == ST_UH) ? p.ny : p.ny - 2;
    dim3 grid(ceil_div(rows, 128), p.S);
    stencil_kernel<MODE><<<grid, 128, 0, st>>>(p);
    ++g_kernel_launches;
}

template <bool CONJT, int EPI, bool RING>
static void launch_gemm(const float2 *A, const float2 *B, size_t ldb, float2 *C, size_t ldc, int ny, int S,
                        cudaStream_t st) {
    if (ny <= 2) return;
    dim3 grid(ceil_div(ny - 2, SBM), ceil_div(S, SBN));
    cgemm_step_kernel<CONJT, EPI, RING><<<grid, STHREADS, 0, st>>>(A, B, ldb, C, ldc, ny, S);
    ++g_kernel_launches;
}

void sweep_solve(const Coefs<float2> &co, const float2 *invT, const SrcView &src, int S, bool adjoint,
                 float2 *u, float2 *tmp, cudaStream_t st) {
    SweepParams p;
    p.co = co;
    p.invT = invT;
    p.u = u;
    p.tmp = tmp;
    p.src = src;
    p.ny = co.ny;
    p.nx = co.nx;
    p.S = S;
    const int ny = co.ny, nx = co.nx;
    const size_t page = (size_t)ny * ny, fld = (size_t)ny * nx;
    WUST_CUDA(cudaMemsetAsync(u, 0, sizeof(float2) * fld * S, st));
    WUST_CUDA(cudaMemsetAsync(tmp, 0, sizeof(float2) * (size_t)ny * S, st));   // border rows of tmp stay zero
    if (!adjoint) {
        for (int j = 1; j < nx; ++j) {
            p.j = j;
            launch_stencil<ST_L>(p, st);
            launch_gemm<false, 0, true>(invT + page * j, tmp, ny, u + (size_t)ny * j, fld, ny, S, st);
        }
        for (int j = nx - 2; j >= 0; --j) {
            p.j = j;
            launch_stencil<ST_U>(p, st);
            launch_gemm<false, 1, false>(invT + page * j, tmp, ny, u + (size_t)ny * j, fld, ny, S, st);
        }
    } else {
        for (int j = 1; j < nx; ++j) {
            p.j = j;
            launch_gemm<true, 0, false>(invT + page * (j - 1), u + (size_t)ny * (j - 1), fld, tmp, ny, ny, S, st);
            launch_stencil<ST_UH>(p, st);
        }
        for (int j = nx - 2; j >= 0; --j) {
            p.j = j;
            launch_stencil<ST_LH>(p, st);
            launch_gemm<true, 0, true>(invT + page * j, tmp, ny, u + (size_t)ny * j, fld, ny, S, st);
        }
    }
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
