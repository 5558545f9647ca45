// Block-LU factorization of the nine-point Helmholtz operator: the Schur
// recursion of decompBlockLU (Runtime/solver/decompBlockLU.cu:337-368)
//
//     T_0 = D_0,  invT_j = inv(T_j[1:Ny-1, 1:Ny-1]),
//     T_{j+1} = D_{j+1} - L_j invT_j U_j,
//
// as ONE persistent cooperative kernel.  Each page is inverted in place by an
// unpivoted blocked Gauss-Jordan sweep (block = FT):
//
//     P = inv(A_KK);  A_KJ <- P A_KJ;  A_IJ <- A_IJ - A_IK (P A_KJ);
//     A_IK <- -A_IK P;  A_KK <- P.
//
// The reference pivots (cusolverDnCgetrf); the Schur blocks of this operator
// have their diagonal entry as the row maximum and condition numbers of
// 10..700 at 4+ points per wavelength, so partial pivoting selects the
// diagonal and the unpivoted sweep computes the same inverse.  A zero or
// non-finite pivot is reported as WUST_ERR_SINGULAR_SCHUR_BLOCK.
//
// The tridiagonal Schur product L_j invT_j U_j needs only the 3x3
// neighbourhood of each invT_j entry (decompBlockLU.cu:65-152); it is fused
// into the page prologue through a shared-memory halo tile.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int FT = 32;         // Gauss-Jordan block and output tile edge
constexpr int FTHREADS = 256;

struct FactorParams {
    Coefs<float2> co;
    float2 *invT;          // [ny, ny, nx] column-major pages
    float2 *ws;            // n_pad x n_pad working page (column-major)
    float2 *rbuf;          // FT x n_pad row panel P A_K.
    float2 *cbuf;          // n_pad x FT old column panel A_.K (rows of K zeroed)
    GridBarrier *bar;
    int *status;           // [0]: 1 + first page with a bad pivot; [1]: pivot index
    int n, n_pad;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ float2 crecip(float2 z) {
    float s = fmaxf(fabsf(z.x), fabsf(z.y));
    float a = z.x / s, b = z.y / s;
    float d = a * a + b * b;
    float inv = 1.f / (s * d);
    return make_float2(a * inv, -b * inv);
}

// In-place unpivoted Gauss-Jordan inverse of the FT x FT block Ps[c][r].
__device__ void gj_invert_block(float2 (*Ps)[FT + 1], int *status, int page, bool report) {
    const int tid = threadIdx.x;
    const int r = tid % FT;
    const int cb = tid / FT;                 // columns cb, cb+8, cb+16, cb+24
    constexpr int PER = FT * FT / FTHREADS;  // 4
    for (int q = 0; q < FT; ++q) {
        float2 piv = Ps[q][q];
        float mag = fabsf(piv.x) + fabsf(piv.y);
        if (report && tid == 0 && !(mag > 0.f && isfinite(mag))) {
            if (atomicCAS(&status[0], 0, page + 1) == 0) status[1] = q;
        }
        float2 ip = crecip(piv);
        float2 arq = Ps[q][r];               // A[r, q]
        float2 vals[PER];
#pragma unroll
        for (int e = 0; e < PER; ++e) {
            int c = cb + e * (FTHREADS / FT);
            float2 a = Ps[c][r];
            float2 aqc = Ps[c][q];           // A[q, c]
            float2 v;
            if (r == q && c == q) v = ip;
            else if (r == q) v = cmul(a, ip);
            else if (c == q) v = cmul(make_float2(-arq.x, -arq.y), ip);
            else v = csub(a, cmul(cmul(arq, aqc), ip));
            vals[e] = v;
        }
        __syncthreads();
#pragma unroll
        for (int e = 0; e < PER; ++e) Ps[cb + e * (FTHREADS / FT)][r] = vals[e];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(FTHREADS) factor_kernel(FactorParams p) {
    __shared__ float2 Ps[FT][FT + 1];
    __shared__ float2 Cs[FT][FT + 1];
    __shared__ float2 Rs[FT][FT + 1];
    __shared__ float2 Xs[FT + 2][FT + 3];   // invT_{j-1} halo tile, Xs[c][r]

    const int ny = p.co.ny, nx = p.co.nx, n = p.n, np_ = p.n_pad;
    const int nt = np_ / FT;                 // tiles per dimension
    const unsigned nblocks = gridDim.x;
    const int tid = threadIdx.x;
    const size_t gstride = (size_t)gridDim.x * blockDim.x;
    const size_t page_sz = (size_t)ny * ny;
    int site = 0;

    // Border rows/columns of every page are zero (decompBlockLU.cu:284-288).
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + tid; idx < (size_t)nx * 4 * ny; idx += gstride) {
        size_t page = idx / (4 * (size_t)ny);
        int rem = (int)(idx % (4 * (size_t)ny));
        int which = rem / ny, k = rem % ny;
        size_t off = which == 0 ? (size_t)ny * k
                   : which == 1 ? (size_t)(ny - 1) + (size_t)ny * k
                   : which == 2 ? (size_t)k
                                : (size_t)k + (size_t)ny * (ny - 1);
        p.invT[page * page_sz + off] = make_float2(0.f, 0.f);
    }

    const int tr = tid % 16, tc = tid / 16;
    for (int j = 0; j < nx; ++j) {
        // ---- prologue: ws = T_j interior (identity padding) -----------------
        const float2 *X = p.invT + (size_t)(j > 0 ? j - 1 : 0) * page_sz;
        for (int t = blockIdx.x; t < nt * nt; t += gridDim.x) {
            const int r0 = (t % nt) * FT, c0 = (t / nt) * FT;     // ws coordinates
            if (j > 0) {
                // halo tile of invT_{j-1} around grid rows r0+1.., cols c0+1..
                for (int e = tid; e < (FT + 2) * (FT + 2); e += FTHREADS) {
                    int rr = e % (FT + 2), cc = e / (FT + 2);
                    int R = r0 + rr, C = c0 + cc;                     // grid index (= ws index + 1) - 1
                    Xs[cc][rr] = (R < ny && C < ny) ? X[R + (size_t)ny * C] : make_float2(0.f, 0.f);
                }
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const int rl = tr + 16 * i, cl = tc + 16 * jj;
                    const int r = r0 + rl, c = c0 + cl;           // ws index
                    float2 v;
                    if (r >= n || c >= n) {
                        v = make_float2(r == c ? 1.f : 0.f, 0.f);
                    } else {
                        const int R = r + 1, C = c + 1;           // grid row/col, in [1, ny-2]
                        v = make_float2(0.f, 0.f);
                        if (R == C) v = p.co.dd(R, j);
                        else if (R == C + 1) v = p.co.dl(C, j);
                        else if (R + 1 == C) v = p.co.du(R, j);
                        if (j > 0) {
                            const int jm = j - 1;
                            const float2 udc = p.co.ud(C, jm), uuc = p.co.uu(C - 1, jm), ulc = p.co.ul(C, jm);
                            float2 right[3];
#pragma unroll
                            for (int d = 0; d < 3; ++d) {            // rows R-1, R, R+1
                                const int xr = rl + d;               // Xs row of grid row R-1+d
                                float2 acc = cmul(Xs[cl + 1][xr], udc);
                                cfma(acc, Xs[cl][xr], uuc);
                                cfma(acc, Xs[cl + 2][xr], ulc);
                                right[d] = acc;
                            }
                            float2 lr = cmul(p.co.ld(R, jm), right[1]);
                            cfma(lr, p.co.ll(R - 1, jm), right[0]);
                            cfma(lr, p.co.lu(R, jm), right[2]);
                            v = csub(v, lr);
                        }
                    }
                    p.ws[r + (size_t)np_ * c] = v;
                }
            }
            __syncthreads();
        }
        if (!grid_sync(p.bar, nblocks, p.timeout_ns, ++site)) return;

        // ---- blocked Gauss-Jordan inverse of ws --------------------------
        for (int kb = 0; kb < nt; ++kb) {
            const int k0 = kb * FT;
            // Phase A: P (every CTA), row panel R = P A_K. and column panel copy.
            for (int e = tid; e < FT * FT; e += FTHREADS) {
                int rr = e % FT, cc = e / FT;
                Ps[cc][rr] = p.ws[(k0 + rr) + (size_t)np_ * (k0 + cc)];
            }
            __syncthreads();
            gj_invert_block(Ps, p.status, j, blockIdx.x == 0);
            {
                // 8 columns per pass: thread (t = tid%32, cc = tid/32)
                const int t = tid % FT, cc = tid / FT;
                for (int cbase = blockIdx.x * 8; cbase < np_; cbase += gridDim.x * 8) {
                    const int c = cbase + cc;
                    // stage A[K, c] in Cs[cc][*] (Cs reused as scratch)
                    Cs[cc][t] = (c < np_) ? p.ws[(k0 + t) + (size_t)np_ * c] : make_float2(0.f, 0.f);
                    __syncthreads();
                    if (c < np_) {
                        float2 acc;
                        if (c >= k0 && c < k0 + FT) {
                            acc = Ps[c - k0][t];
                        } else {
                            acc = make_float2(0.f, 0.f);
#pragma unroll 8
                            for (int u = 0; u < FT; ++u) cfma(acc, Ps[u][t], Cs[cc][u]);
                        }
                        p.rbuf[t + (size_t)FT * c] = acc;
                    }
                    __syncthreads();
                }
                for (size_t e = (size_t)blockIdx.x * blockDim.x + tid; e < (size_t)np_ * FT; e += gstride) {
                    int r = (int)(e % np_), tt = (int)(e / np_);
                    p.cbuf[e] = (r >= k0 && r < k0 + FT) ? make_float2(0.f, 0.f)
                                                         : p.ws[r + (size_t)np_ * (k0 + tt)];
                }
            }
            if (!grid_sync(p.bar, nblocks, p.timeout_ns, ++site)) return;

            // Phase B: tile update.
            const bool last = (kb == nt - 1);
            for (int t = blockIdx.x; t < nt * nt; t += gridDim.x) {
                const int I = t % nt, J = t / nt;
                const int r0 = I * FT, c0 = J * FT;
                for (int e = tid; e < FT * FT; e += FTHREADS) {
                    int a = e % FT, b = e / FT;
                    Cs[b][a] = p.cbuf[(r0 + a) + (size_t)np_ * b];   // Cs[t][r]
                    Rs[b][a] = p.rbuf[a + (size_t)FT * (c0 + b)];   // Rs[c][t]
                }
                __syncthreads();
#pragma unroll
                for (int i = 0; i < 2; ++i) {
#pragma unroll
                    for (int jj = 0; jj < 2; ++jj) {
                        const int rl = tr + 16 * i, cl = tc + 16 * jj;
                        const int r = r0 + rl, c = c0 + cl;
                        float2 v;
                        if (I == kb) {
                            v = Rs[cl][rl];
                        } else {
                            float2 acc = (J == kb) ? make_float2(0.f, 0.f) : p.ws[r + (size_t)np_ * c];
                            float2 dot = make_float2(0.f, 0.f);
#pragma unroll 8
                            for (int u = 0; u < FT; ++u) cfma(dot, Cs[u][rl], Rs[cl][u]);
                            v = csub(acc, dot);
                        }
                        p.ws[r + (size_t)np_ * c] = v;
                        if (last && r < n && c < n)
                            p.invT[(size_t)j * page_sz + (size_t)(r + 1) + (size_t)ny * (c + 1)] = v;
                    }
                }
                __syncthreads();
            }
            if (!grid_sync(p.bar, nblocks, p.timeout_ns, ++site)) return;
        }
    }
}

// Scratch layout for one factorization.
size_t factor_scratch_bytes(int ny) {
    const int n = ny - 2;
    const int np_ = ceil_div(n, FT) * FT;
    return sizeof(float2) * ((size_t)np_ * np_ + 2 * (size_t)np_ * FT) + sizeof(GridBarrier) + 4 * sizeof(int) + 256;
}

void factor_launch(const Coefs<float2> &co, float2 *invT, void *scratch, size_t scratch_bytes,
                   cudaStream_t stream, double timeout_s, int *host_status) {
    const int ny = co.ny;
    const int n = ny - 2;
    const int np_ = ceil_div(n, FT) * FT;
    if (scratch_bytes < factor_scratch_bytes(ny)) fail(WUST_ERR_RUNTIME, "factor scratch too small");
    char *base = (char *)scratch;
    FactorParams p;
    p.co = co;
    p.invT = invT;
    p.ws = (float2 *)base;
    p.rbuf = p.ws + (size_t)np_ * np_;
    p.cbuf = p.rbuf + (size_t)np_ * FT;
    char *tail = (char *)(p.cbuf + (size_t)np_ * FT);
    p.bar = (GridBarrier *)tail;
    p.status = (int *)(tail + sizeof(GridBarrier));
    p.n = n;
    p.n_pad = np_;
    p.timeout_ns = (unsigned long long)(timeout_s * 1e9);
    WUST_CUDA(cudaMemsetAsync(tail, 0, sizeof(GridBarrier) + 4 * sizeof(int), stream));

    int dev = 0, sms = 0, per_sm = 0;
    WUST_CUDA(cudaGetDevice(&dev));
    WUST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WUST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, factor_kernel, FTHREADS, 0));
    if (per_sm < 1) fail(WUST_ERR_CUDA, "factor kernel cannot be resident");
    const int nt = np_ / FT;
    int grid = sms;                          // one CTA per SM
    if (grid > nt * nt) grid = nt * nt;
    void *args[] = {&p};
    WUST_CUDA(cudaLaunchCooperativeKernel((void *)factor_kernel, dim3(grid), dim3(FTHREADS), args, 0, stream));
    WUST_LAUNCH_CHECK();
    ++g_kernel_launches;
    if (host_status) {
        int st[4];
        GridBarrier gb;
        WUST_CUDA(cudaMemcpyAsync(&gb, p.bar, sizeof(gb), cudaMemcpyDeviceToHost, stream));
        WUST_CUDA(cudaMemcpyAsync(st, p.status, sizeof(st), cudaMemcpyDeviceToHost, stream));
        WUST_CUDA(cudaStreamSynchronize(stream));
        host_status[0] = st[0];
        host_status[1] = st[1];
        host_status[2] = gb.error;
    }
}

// Self-test of the bounded barrier: one CTA waits for an arrival that never
// comes (nblocks = grid + 1) and must give up after timeout_ns.
__global__ void barrier_timeout_probe(GridBarrier *bar, unsigned long long timeout_ns, int *passed) {
    bool ok = grid_sync(bar, gridDim.x + 1, timeout_ns, 77);
    if (threadIdx.x == 0) passed[blockIdx.x] = ok ? 1 : 0;
}

int barrier_selftest(double timeout_s, int *site_out) {
    GridBarrier *bar = nullptr;
    int *passed = nullptr;
    WUST_CUDA(cudaMalloc(&bar, sizeof(GridBarrier) + sizeof(int)));
    passed = (int *)((char *)bar + sizeof(GridBarrier));
    WUST_CUDA(cudaMemset(bar, 0, sizeof(GridBarrier) + sizeof(int)));
    barrier_timeout_probe<<<1, 32>>>(bar, (unsigned long long)(timeout_s * 1e9), passed);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    GridBarrier gb{};
    int ok = -1;
    if (e == cudaSuccess) {
        cudaMemcpy(&gb, bar, sizeof(gb), cudaMemcpyDeviceToHost);
        cudaMemcpy(&ok, passed, sizeof(int), cudaMemcpyDeviceToHost);
    }
    cudaFree(bar);
    if (e != cudaSuccess) fail(WUST_ERR_CUDA, "barrier self-test: %s", cudaGetErrorString(e));
    *site_out = gb.error;
    return ok;
}

}  // namespace wust
