// Batched forward and adjoint block-tridiagonal sweeps of applyBlockLU
// (Runtime/solver/applyBlockLU.cu:433-467), complex single on CUDA cores.
//
// Forward (H u = src):
//   j = 1..Nx-1 :  u_j  = invT_j (SRC_j - L_{j-1} u_{j-1})            [F1]
//   j = Nx-2..0 :  u_j -= invT_j (U_j u_{j+1})                        [F2]
// Adjoint (H^H u = src):
//   j = 1..Nx-1 :  u_j  = SRC_j - U_{j-1}^H (invT_{j-1}^H u_{j-1})    [A1 + stencil]
//   j = Nx-2..0 :  u_j  = invT_j^H (u_j - L_j^H u_{j+1})              [stencil + A2]
//
// One launch per column step: a 32x32-tile complex GEMM whose B operand is
// produced on the fly from the tridiagonal stencil (the reference runs a
// separate stencil kernel and cublasCgemm3m per step).  Threads run along y,
// so every field access is a contiguous, coalesced column segment.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int SBM = 32, SBN = 32, SBK = 32, STHREADS = 256;

struct SweepParams {
    Coefs<float2> co;
    const float2 *invT;
    float2 *u;          // [ny, nx, S]
    float2 *tmp;        // [ny, S] (adjoint first sweep)
    SrcView src;
    int ny, nx, S, j;
};

template <int MODE>
__device__ __forceinline__ float2 produce_b(const SweepParams &p, int k, int s) {
    const int ny = p.ny, j = p.j;
    const size_t fs = (size_t)ny * p.nx * s;
    if (MODE == SWEEP_F1) {
        const float2 *uc = p.u + fs + (size_t)ny * (j - 1);
        float2 acc = cmul(p.co.ld(k, j - 1), uc[k]);
        cfma(acc, p.co.ll(k - 1, j - 1), uc[k - 1]);
        cfma(acc, p.co.lu(k, j - 1), uc[k + 1]);
        return csub(p.src.get(k, j, s, ny, p.nx), acc);
    } else if (MODE == SWEEP_F2) {
        const float2 *uc = p.u + fs + (size_t)ny * (j + 1);
        float2 acc = cmul(p.co.ud(k, j), uc[k]);
        cfma(acc, p.co.ul(k - 1, j), uc[k - 1]);
        cfma(acc, p.co.uu(k, j), uc[k + 1]);
        return acc;
    } else if (MODE == SWEEP_A1) {
        return p.u[fs + (size_t)ny * (j - 1) + k];
    } else {  // SWEEP_A2: B = tmp = u_j - L_j^H u_{j+1} (adjoint_pre_kernel)
        return p.tmp[k + (size_t)ny * s];
    }
}

template <int MODE>
__global__ void __launch_bounds__(STHREADS) sweep_gemm_kernel(SweepParams p) {
    __shared__ float2 As[SBK][SBM + 1];   // As[k][r] = op(A)(r, k)
    __shared__ float2 Bs[SBK][SBN + 1];   // Bs[k][s]
    const int ny = p.ny, j = p.j;
    const int tid = threadIdx.x, tr = tid % 16, tc = tid / 16;
    const int r0 = 1 + blockIdx.x * SBM;
    const int s0 = blockIdx.y * SBN;
    const int page = (MODE == SWEEP_A1) ? j - 1 : j;
    const float2 *A = p.invT + (size_t)page * ny * ny;
    constexpr bool CONJT = (MODE == SWEEP_A1 || MODE == SWEEP_A2);

    float2 acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) acc[i][jj] = make_float2(0.f, 0.f);

    for (int k0 = 1; k0 < ny - 1; k0 += SBK) {
        for (int e = tid; e < SBM * SBK; e += STHREADS) {
            int rr, kk;
            if (CONJT) { kk = e % SBK; rr = e / SBK; }
            else { rr = e % SBM; kk = e / SBM; }
            const int r = r0 + rr, k = k0 + kk;
            float2 v = make_float2(0.f, 0.f);
            if (r < ny - 1 && k < ny - 1)
                v = CONJT ? cconj(A[k + (size_t)ny * r]) : A[r + (size_t)ny * k];
            As[kk][rr] = v;
        }
        for (int e = tid; e < SBK * SBN; e += STHREADS) {
            const int kk = e % SBK, ss = e / SBK;
            const int k = k0 + kk, s = s0 + ss;
            Bs[kk][ss] = (k < ny - 1 && s < p.S) ? produce_b<MODE>(p, k, s) : make_float2(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < SBK; ++kk) {
            const float2 a0 = As[kk][tr], a1 = As[kk][tr + 16];
            const float2 b0 = Bs[kk][tc], b1 = Bs[kk][tc + 16];
            cfma(acc[0][0], a0, b0);
            cfma(acc[0][1], a0, b1);
            cfma(acc[1][0], a1, b0);
            cfma(acc[1][1], a1, b1);
        }
        __syncthreads();
    }

    const size_t fstride = (size_t)ny * p.nx;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int jj = 0; jj < 2; ++jj) {
            const int r = r0 + tr + 16 * i, s = s0 + tc + 16 * jj;
            if (r >= ny - 1 || s >= p.S) continue;
            if (MODE == SWEEP_A1) {
                p.tmp[r + (size_t)ny * s] = acc[i][jj];
            } else {
                float2 *dst = p.u + fstride * s + (size_t)ny * j + r;
                if (MODE == SWEEP_F2) *dst = csub(*dst, acc[i][jj]);
                else *dst = acc[i][jj];
            }
        }
    }
    // Border rows of the written column: invT has zero border rows.
    if ((MODE == SWEEP_F1 || MODE == SWEEP_A2) && blockIdx.x == 0 && tid < 2 * SBN) {
        const int s = s0 + tid / 2;
        if (s < p.S) {
            const int r = (tid % 2) ? ny - 1 : 0;
            p.u[fstride * s + (size_t)ny * j + r] = make_float2(0.f, 0.f);
        }
    }
}

// tmp(:, s) = u(:, j, s) - L_j^H u(:, j+1, s) on interior rows
// (applyBlockLU.cu:224-267); the GEMM that follows ignores border rows.
__global__ void adjoint_pre_kernel(SweepParams p) {
    const int ny = p.ny, j = p.j;
    const int y = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int s = blockIdx.y;
    if (y >= ny - 1 || s >= p.S) return;
    const float2 *un = p.u + (size_t)ny * p.nx * s + (size_t)ny * (j + 1);
    float2 acc = make_float2(0.f, 0.f);
    cfma_conj(acc, p.co.ld(y, j), un[y]);
    cfma_conj(acc, p.co.lu(y - 1, j), un[y - 1]);
    cfma_conj(acc, p.co.ll(y, j), un[y + 1]);
    p.tmp[y + (size_t)ny * s] = csub(p.u[(size_t)ny * p.nx * s + (size_t)ny * j + y], acc);
}

// u(:, j, s) = SRC(:, j, s) - U_{j-1}^H tmp(:, s), every row including the
// border (applyBlockLU.cu:159-202).
__global__ void adjoint_stencil_kernel(SweepParams p) {
    const int ny = p.ny, j = p.j;
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (y >= ny || s >= p.S) return;
    const float2 *t = p.tmp + (size_t)ny * s;
    float2 acc = make_float2(0.f, 0.f);
    cfma_conj(acc, p.co.ud(y, j - 1), t[y]);
    if (y > 0) cfma_conj(acc, p.co.uu(y - 1, j - 1), t[y - 1]);
    if (y < ny - 1) cfma_conj(acc, p.co.ul(y, j - 1), t[y + 1]);
    p.u[(size_t)ny * p.nx * s + (size_t)ny * j + y] = csub(p.src.get(y, j, s, ny, p.nx), acc);
}

template <int MODE>
static void launch_step(const SweepParams &p, cudaStream_t st) {
    dim3 grid(ceil_div(p.ny - 2, SBM), ceil_div(p.S, SBN));
    sweep_gemm_kernel<MODE><<<grid, STHREADS, 0, st>>>(p);
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
    WUST_CUDA(cudaMemsetAsync(u, 0, sizeof(float2) * (size_t)ny * nx * S, st));
    if (!adjoint) {
        for (int j = 1; j < nx; ++j) { p.j = j; launch_step<SWEEP_F1>(p, st); }
        for (int j = nx - 2; j >= 0; --j) { p.j = j; launch_step<SWEEP_F2>(p, st); }
    } else {
        WUST_CUDA(cudaMemsetAsync(tmp, 0, sizeof(float2) * (size_t)ny * S, st));
        dim3 sgrid(ceil_div(ny, 128), S);
        for (int j = 1; j < nx; ++j) {
            p.j = j;
            launch_step<SWEEP_A1>(p, st);
            adjoint_stencil_kernel<<<sgrid, 128, 0, st>>>(p);
            ++g_kernel_launches;
        }
        dim3 pgrid(ceil_div(ny - 2, 128), S);
        for (int j = nx - 2; j >= 0; --j) {
            p.j = j;
            adjoint_pre_kernel<<<pgrid, 128, 0, st>>>(p);
            ++g_kernel_launches;
            launch_step<SWEEP_A2>(p, st);
        }
    }
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
