// Block-LU factorization of the nine-point Helmholtz operator: the Schur
// recursion of decompBlockLU (Runtime/solver/decompBlockLU.cu:337-368)
//
//     T_0 = D_0,  invT_j = inv(T_j[1:Ny-1, 1:Ny-1]),
//     T_{j+1} = D_{j+1} - L_j invT_j U_j,
//
// as ONE persistent cooperative kernel (one CTA per SM, bounded grid barrier
// between phases).  Each page is inverted by an unpivoted blocked
// Gauss-Jordan sweep over NB-wide blocks K:
//
//     P = inv(A_KK);  R_K. = P A_K.  (R_KK = P);  C_.K = A_.K (rows of K zeroed)
//     A'_rc = (r in K) ? R_rc : ((c in K) ? 0 : A_rc) - sum_u C_ru R_uc
//
// The reference pivots (cusolverDnCgetrf); the Schur blocks of this operator
// keep their largest entry of each row on the diagonal and have condition
// numbers of 10..700 at 4+ points per wavelength, so partial pivoting selects
// the diagonal and the unpivoted sweep computes the same inverse.  A zero or
// non-finite pivot is reported as WUST_ERR_SINGULAR_SCHUR_BLOCK.
//
// Work split: every CTA owns G x G output tiles of the padded page.  The
// working page is double-buffered in global memory (L2-resident, 2 x 2.6 MB
// at 552^2), so a Gauss-Jordan step reads panels of step k from one buffer
// and writes step k+1 into the other: one grid barrier per step.  Each CTA
// inverts the small NB x NB pivot block itself (no extra barrier) and forms
// the row-panel slice its tile needs.  The tridiagonal Schur product
// L_j invT_j U_j needs only the 3x3 neighbourhood of each invT_j entry
// (decompBlockLU.cu:65-152) and is fused into the page prologue through a
// shared-memory halo tile.
#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int G = kFactorTile;   // output tile edge
constexpr int NB = 24;           // Gauss-Jordan block (divides G)
constexpr int GT = 256;          // threads: (tr, tc) in 16 x 16, rows tr + 16 i, cols tc + 16 j, i, j < 3
static_assert(G % NB == 0 && G == 48, "tile mapping assumes G = 48");

struct FactorParams {
    Coefs<float2> co;
    float2 *invT;          // [ny, ny, nx] column-major pages
    float2 *ws0, *ws1;     // n_pad x n_pad working pages (column-major), ping-pong
    unsigned *counter;     // monotonic barrier counter
    int *err;              // barrier timeout site
    int *status;           // [0]: 1 + first page with a bad pivot; [1]: pivot index
    int n, n_pad;
    int j0, j1;            // pages [j0, j1); page j0 - 1 (if any) is already in invT
    unsigned long long timeout_ns;
#ifdef WUST_FACTOR_PROFILE
    unsigned long long *prof;   // [0] prologue, [1] pivot block, [2] tile work, [3] barriers (block 0, ns)
#endif
};

#ifdef WUST_FACTOR_PROFILE
#define PROF_MARK(slot)                                                     \
    do {                                                                    \
        if (blockIdx.x == 0 && threadIdx.x == 0) {                          \
            const unsigned long long now_ = global_timer_ns();              \
            p.prof[slot] += now_ - prof_t;                                  \
            prof_t = now_;                                                  \
        }                                                                   \
    } while (0)
#else
#define PROF_MARK(slot) do { } while (0)
#endif

// Grid barrier on a monotonic counter: arrive with a release reduction, wait
// with acquire loads until the counter reaches epoch * nblocks.  The wait is
// bounded by timeout_ns (%globaltimer); on expiry the site is recorded in
// *err and every CTA leaves.
__device__ __forceinline__ bool grid_barrier(unsigned *counter, int *err, unsigned nblocks, unsigned &epoch,
                                             unsigned long long timeout_ns, int site) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ++epoch;
        const unsigned target = epoch * nblocks;
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(counter), "r"(1u) : "memory");
        int ok = 1;
        const unsigned long long t0 = global_timer_ns();
        for (unsigned spin = 0;; ++spin) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(counter) : "memory");
            if ((int)(v - target) >= 0) break;
            if (*(volatile int *)err) { ok = 0; break; }
            if ((spin & 31u) == 31u && global_timer_ns() - t0 > timeout_ns) {
                atomicCAS(err, 0, site);
                ok = 0;
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Shared-memory carve-up: the NB x (NB+1) pivot inverse, the double-buffered
// pivot column (in a second NB x (NB+1) slot), then three NB x (G+1) panels;
// the prologue's (G+2) x (G+3) halo tile aliases the panels.
constexpr int kPivElems = NB * (NB + 1);
constexpr int kPanelElems = NB * (G + 1);
constexpr int kHaloElems = (G + 2) * (G + 3);
constexpr int kFactorSmemElems = 2 * kPivElems + (3 * kPanelElems > kHaloElems ? 3 * kPanelElems : kHaloElems);
constexpr size_t kFactorSmemBytes = sizeof(float2) * kFactorSmemElems;

// Own G x G tile entries (rows tr + 16 i, cols tc + 16 j) into registers.
__device__ __forceinline__ void load_tile(const float2 *cur, int np_, int r0, int c0, int tr, int tc, float2 (&a)[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) a[i][jj] = cur[(r0 + tr + 16 * i) + (size_t)np_ * (c0 + tc + 16 * jj)];
}

// Panels of one tile: Kr[u][cl] = A[k0+u, c0+cl]; Cc[u][rl] = A[r0+rl, k0+u]
// (zero on the rows of K).  All loads of a thread are issued before its
// shared-memory stores.
template <int NTH>
__device__ __forceinline__ void stage_panels(const float2 *cur, int np_, int k0, int r0, int c0, float2 (*Kr)[G + 1],
                                             float2 (*Cc)[G + 1], int t0) {
    constexpr int PER = (NB * G + NTH - 1) / NTH;
    float2 kv[PER], cv[PER];
#pragma unroll
    for (int m = 0; m < PER; ++m) {
        const int e = t0 + m * NTH;
        if (e < NB * G) {
            const int u = e % NB, cl = e / NB;
            kv[m] = cur[(k0 + u) + (size_t)np_ * (c0 + cl)];
            const int rl = e % G, uu = e / G, r = r0 + rl;
            cv[m] = (r >= k0 && r < k0 + NB) ? make_float2(0.f, 0.f) : cur[r + (size_t)np_ * (k0 + uu)];
        }
    }
#pragma unroll
    for (int m = 0; m < PER; ++m) {
        const int e = t0 + m * NTH;
        if (e < NB * G) {
            Kr[e % NB][e / NB] = kv[m];
            Cc[e / G][e % G] = cv[m];
        }
    }
}

// 1/z as conj(z) / |z|^2 with the correctly rounded reciprocal intrinsic
// (pivot magnitudes of this operator are O(1/h^2), far from FP32 overflow).
__device__ __forceinline__ float2 crecip_fast(float2 z) {
    const float inv = __frcp_rn(fmaf(z.x, z.x, z.y * z.y));
    return make_float2(z.x * inv, -z.y * inv);
}

// Unpivoted Gauss-Jordan inverse of the NB x NB pivot block on warps 0-3:
// lane r holds row r, warp w holds columns [6w, 6w + 6).  Per pivot q the
// owner warp publishes column q through shared memory (one 128-thread named
// barrier per pivot, double-buffered), the pivot row travels by warp
// shuffles.  Result -> Pa[row][col].
__device__ __forceinline__ void invert_pivot_block(const float2 *cur, int np_, int k0, float2 (*Pa)[NB + 1],
                                                   float2 (*fcol)[NB], int *status, int page, bool report) {
    static_assert(NB == 24, "4 warps x 6 columns");
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = 6 * w;
    float2 a[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
        a[c] = (lane < NB) ? cur[(k0 + lane) + (size_t)np_ * (k0 + col0 + c)] : make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        float2 *fc = fcol[q & 1];
        if (w == q / 6 && lane < NB) fc[lane] = a[q % 6];
        asm volatile("bar.sync 1, 128;" ::: "memory");
        const float2 piv = fc[q];
        if (report && threadIdx.x == 0) {
            const float mag = fabsf(piv.x) + fabsf(piv.y);
            if (!(mag > 0.f && isfinite(mag)) && atomicCAS(&status[0], 0, page + 1) == 0) status[1] = k0 + q;
        }
        const float2 ip = crecip_fast(piv);
        const float2 f = (lane < NB) ? fc[lane] : make_float2(0.f, 0.f);
        const float2 mf = make_float2(-f.x, -f.y);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            float2 pr;
            pr.x = __shfl_sync(0xffffffffu, a[c].x, q);
            pr.y = __shfl_sync(0xffffffffu, a[c].y, q);
            pr = cmul(pr, ip);
            float2 nv;
            if (col0 + c == q) nv = (lane == q) ? ip : cmul(mf, ip);
            else if (lane == q) nv = pr;
            else {
                nv = a[c];
                cfma(nv, mf, pr);
            }
            a[c] = nv;
        }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c)
        if (lane < NB) Pa[lane][col0 + c] = a[c];
}

__global__ void __launch_bounds__(GT, 1) factor_kernel(FactorParams p) {
    extern __shared__ float2 smem[];
    float2(*Pa)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(smem);
    float2(*fcol)[NB] = reinterpret_cast<float2(*)[NB]>(smem + kPivElems);          // pivot column, double-buffered
    float2(*Kr)[G + 1] = reinterpret_cast<float2(*)[G + 1]>(smem + 2 * kPivElems);   // A[K, tile cols]
    float2(*Rr)[G + 1] = Kr + NB;                                                   // R[u][tile col]
    float2(*Cc)[G + 1] = Kr + 2 * NB;                                               // C[tile row][u], as Cc[u][row]
    float2(*Xs)[G + 3] = reinterpret_cast<float2(*)[G + 3]>(smem + 2 * kPivElems);   // prologue halo, Xs[col][row]

    const int ny = p.co.ny, n = p.n, np_ = p.n_pad;
    const int nt = np_ / G, nsteps = np_ / NB;
    const unsigned nblocks = gridDim.x;
    const int tid = threadIdx.x, tr = tid % 16, tc = tid / 16;
    const size_t page_sz = (size_t)ny * ny;
    unsigned epoch = 0;
    int site = 0;
#ifdef WUST_FACTOR_PROFILE
    unsigned long long prof_t = global_timer_ns();
#endif

    // Border rows/columns of every page are zero (decompBlockLU.cu:284-288).
    const size_t gstride = (size_t)gridDim.x * blockDim.x;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + tid; idx < (size_t)(p.j1 - p.j0) * 4 * ny; idx += gstride) {
        const size_t page = p.j0 + idx / (4 * (size_t)ny);
        const int rem = (int)(idx % (4 * (size_t)ny));
        const int which = rem / ny, k = rem % ny;
        const size_t off = which == 0 ? (size_t)ny * k
                         : which == 1 ? (size_t)(ny - 1) + (size_t)ny * k
                         : which == 2 ? (size_t)k
                                      : (size_t)k + (size_t)ny * (ny - 1);
        p.invT[page * page_sz + off] = make_float2(0.f, 0.f);
    }

    for (int j = p.j0; j < p.j1; ++j) {
        // ---- prologue: ws0 = T_j interior (identity padding) ----------------
        const float2 *X = p.invT + (size_t)(j > 0 ? j - 1 : 0) * page_sz;
        for (int t = blockIdx.x; t < nt * nt; t += gridDim.x) {
            const int r0 = (t % nt) * G, c0 = (t / nt) * G;     // ws coordinates
            if (j > 0) {
                for (int e = tid; e < (G + 2) * (G + 2); e += GT) {
                    const int rr = e % (G + 2), cc = e / (G + 2);
                    const int R = r0 + rr, C = c0 + cc;          // grid indices of invT_{j-1}
                    Xs[cc][rr] = (R < ny && C < ny) ? X[R + (size_t)ny * C] : make_float2(0.f, 0.f);
                }
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 3; ++i) {
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) {
                    const int rl = tr + 16 * i, cl = tc + 16 * jj;
                    const int r = r0 + rl, c = c0 + cl;
                    float2 v;
                    if (r >= n || c >= n) {
                        v = make_float2(r == c ? 1.f : 0.f, 0.f);
                    } else {
                        const int R = r + 1, C = c + 1;          // grid row/col in [1, ny-2]
                        v = make_float2(0.f, 0.f);
                        if (R == C) v = p.co.dd(R, j);
                        else if (R == C + 1) v = p.co.dl(C, j);
                        else if (R + 1 == C) v = p.co.du(R, j);
                        if (j > 0) {
                            const int jm = j - 1;
                            const float2 udc = p.co.ud(C, jm), uuc = p.co.uu(C - 1, jm), ulc = p.co.ul(C, jm);
                            float2 right[3];
#pragma unroll
                            for (int d = 0; d < 3; ++d) {            // grid rows R-1, R, R+1
                                float2 acc = cmul(Xs[cl + 1][rl + d], udc);
                                cfma(acc, Xs[cl][rl + d], uuc);
                                cfma(acc, Xs[cl + 2][rl + d], ulc);
                                right[d] = acc;
                            }
                            float2 lr = cmul(p.co.ld(R, jm), right[1]);
                            cfma(lr, p.co.ll(R - 1, jm), right[0]);
                            cfma(lr, p.co.lu(R, jm), right[2]);
                            v = csub(v, lr);
                        }
                    }
                    p.ws0[r + (size_t)np_ * c] = v;
                }
            }
            __syncthreads();
        }
        PROF_MARK(0);
        if (!grid_barrier(p.counter, p.err, nblocks, epoch, p.timeout_ns, ++site)) return;
        PROF_MARK(3);

        // ---- blocked Gauss-Jordan inverse -----------------------------------
        for (int kb = 0; kb < nsteps; ++kb) {
            const float2 *cur = (kb & 1) ? p.ws1 : p.ws0;
            float2 *nxt = (kb & 1) ? p.ws0 : p.ws1;
            const int k0 = kb * NB;
            const bool last = (kb == nsteps - 1);

            // Warps 0-3 invert the pivot block A_KK in registers while warps 4-7
            // stage this CTA's first tile panels; all threads prefetch their
            // own tile entries first so every load is in flight at once.
            const int warp = tid >> 5;
            int t = blockIdx.x;
            float2 a[3][3];
            if (t < nt * nt) load_tile(cur, np_, (t % nt) * G, (t / nt) * G, tr, tc, a);
            if (warp < 4) {
                invert_pivot_block(cur, np_, k0, Pa, fcol, p.status, j, blockIdx.x == 0);
            } else if (t < nt * nt) {
                stage_panels<GT - 128>(cur, np_, k0, (t % nt) * G, (t / nt) * G, Kr, Cc, tid - 128);
            }
            __syncthreads();
            PROF_MARK(1);
            while (t < nt * nt) {
                const int I = t % nt, J = t / nt;
                const int r0 = I * G, c0 = J * G;
                // row panel slice R[u][cl] = (P A[K, .])_{u, c0+cl}; R = P on the columns of K
                if (tid < 8 * NB) {
                    const int u = tid % NB, cb = tid / NB;
                    float2 acc[G / 8];
#pragma unroll
                    for (int m = 0; m < G / 8; ++m) acc[m] = make_float2(0.f, 0.f);
#pragma unroll 4
                    for (int v = 0; v < NB; ++v) {
                        const float2 pv = Pa[u][v];
#pragma unroll
                        for (int m = 0; m < G / 8; ++m) cfma(acc[m], pv, Kr[v][cb + 8 * m]);
                    }
#pragma unroll
                    for (int m = 0; m < G / 8; ++m) {
                        const int cl = cb + 8 * m, c = c0 + cl;
                        Rr[u][cl] = (c >= k0 && c < k0 + NB) ? Pa[u][c - k0] : acc[m];
                    }
                }
                __syncthreads();
#pragma unroll
                for (int i = 0; i < 3; ++i) {
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) {
                        const int rl = tr + 16 * i, cl = tc + 16 * jj;
                        const int r = r0 + rl, c = c0 + cl;
                        const bool rk = (r >= k0 && r < k0 + NB), ck = (c >= k0 && c < k0 + NB);
                        float2 v = rk ? Rr[r - k0][cl] : (ck ? make_float2(0.f, 0.f) : a[i][jj]);
                        float2 dot = make_float2(0.f, 0.f);
#pragma unroll 8
                        for (int u = 0; u < NB; ++u) cfma(dot, Cc[u][rl], Rr[u][cl]);
                        v = csub(v, dot);
                        nxt[r + (size_t)np_ * c] = v;
                        if (last && r < n && c < n)
                            p.invT[(size_t)j * page_sz + (size_t)(r + 1) + (size_t)ny * (c + 1)] = v;
                    }
                }
                __syncthreads();
                t += gridDim.x;
                if (t < nt * nt) {          // more tiles than CTAs: stage the next one with all threads
                    load_tile(cur, np_, (t % nt) * G, (t / nt) * G, tr, tc, a);
                    stage_panels<GT>(cur, np_, k0, (t % nt) * G, (t / nt) * G, Kr, Cc, tid);
                    __syncthreads();
                }
            }
            PROF_MARK(2);
            if (!grid_barrier(p.counter, p.err, nblocks, epoch, p.timeout_ns, ++site)) return;
            PROF_MARK(3);
        }
    }
}

size_t factor_scratch_bytes(int ny) { return factor_scratch_bytes_for(ny); }

void factor_launch(const Coefs<float2> &co, float2 *invT, void *scratch, size_t scratch_bytes,
                   cudaStream_t stream, double timeout_s, int *host_status, int j0, int j1, int max_ctas) {
    const int ny = co.ny;
    const int n = ny - 2;
    const int np_ = (int)factor_pad(ny);
    if (scratch_bytes < factor_scratch_bytes(ny)) fail(WUST_ERR_RUNTIME, "factor scratch too small");
    FactorParams p;
    p.co = co;
    p.invT = invT;
    p.ws0 = (float2 *)scratch;
    p.ws1 = p.ws0 + (size_t)np_ * np_;
    int *tail = (int *)(p.ws1 + (size_t)np_ * np_);
    p.counter = (unsigned *)tail;
    p.err = tail + 1;
    p.status = tail + 2;
    p.n = n;
    p.n_pad = np_;
    p.j0 = j0;
    p.j1 = j1 < 0 ? co.nx : j1;
    if (p.j0 < 0 || p.j0 >= p.j1 || p.j1 > co.nx) fail(WUST_ERR_RUNTIME, "factor page range [%d, %d) invalid", j0, j1);
    p.timeout_ns = (unsigned long long)(timeout_s * 1e9);
    WUST_CUDA(cudaMemsetAsync(tail, 0, 8 * sizeof(int), stream));

    // Set on every launch: the attribute belongs to the current device's
    // context, which a caller may switch or reset between calls.
    WUST_CUDA(cudaFuncSetAttribute(factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFactorSmemBytes));
    int dev = 0, sms = 0, per_sm = 0;
    WUST_CUDA(cudaGetDevice(&dev));
    WUST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WUST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, factor_kernel, GT, kFactorSmemBytes));
    if (per_sm < 1) fail(WUST_ERR_CUDA, "factor kernel cannot be resident");
    const int nt = np_ / G;
    int grid = sms;                          // one CTA per SM
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid > nt * nt) grid = nt * nt;
    void *args[] = {&p};
    WUST_CUDA(cudaLaunchCooperativeKernel((void *)factor_kernel, dim3(grid), dim3(GT), args, kFactorSmemBytes, stream));
    WUST_LAUNCH_CHECK();
    ++g_kernel_launches;
    if (host_status) {
        int st[8];
        WUST_CUDA(cudaMemcpyAsync(st, tail, sizeof(st), cudaMemcpyDeviceToHost, stream));
        WUST_CUDA(cudaStreamSynchronize(stream));
        host_status[0] = st[2];
        host_status[1] = st[3];
        host_status[2] = st[1];
    }
}

// Self-test of the bounded wait: one CTA waits at a barrier sized for
// gridDim.x + 1 CTAs, which can never fill, and must give up after timeout_ns.
__global__ void barrier_timeout_probe(unsigned *counter, int *err, unsigned long long timeout_ns, int *passed) {
    unsigned epoch = 0;
    const bool ok = grid_barrier(counter, err, gridDim.x + 1, epoch, timeout_ns, 77);
    if (threadIdx.x == 0) passed[blockIdx.x] = ok ? 1 : 0;
}

int barrier_selftest(double timeout_s, int *site_out) {
    int *buf = nullptr;
    WUST_CUDA(cudaMalloc(&buf, 4 * sizeof(int)));
    WUST_CUDA(cudaMemset(buf, 0, 4 * sizeof(int)));
    barrier_timeout_probe<<<1, 32>>>((unsigned *)buf, buf + 1, (unsigned long long)(timeout_s * 1e9), buf + 2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    int host[4] = {0, 0, -1, 0};
    if (e == cudaSuccess) cudaMemcpy(host, buf, sizeof(host), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) fail(WUST_ERR_CUDA, "barrier self-test: %s", cudaGetErrorString(e));
    *site_out = host[1];
    return host[2];
}

}  // namespace wust
