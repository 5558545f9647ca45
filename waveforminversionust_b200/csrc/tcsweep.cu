// Block-tridiagonal sweeps of applyBlockLU (Runtime/solver/applyBlockLU.cu:433-467)
// with the dense invT_j products on the tensor cores (tcgen05, TF32 inputs,
// FP32 accumulation in tensor memory).  Used by the refined TF32 profile:
// the FP64-residual refinement in api.cu restores full accuracy.
//
// Complex products are split into one real GEMM:
//     [Cr]   [Ar  -Ai] [Br]
//     [Ci] = [Ai   Ar] [Bi]
// A 128-row tile of the stacked operand holds 64 complex rows: rows 0-63
// are [Ar, -Ai], rows 64-127 are [Ai, Ar], so one 128 x TN accumulator tile
// yields Cr and Ci of 64 complex rows for TN sources.  The stacked invT_j
// (and, for adjoint sweeps, invT_j^H) are packed once per factorization into
// the chunked core-matrix layout of tc.cuh; the B operand (the stencil
// result, [Br; Bi]) is written in that layout by the stencil kernels.
#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace wust {

constexpr int TN = 64;          // sources per tile (MMA N)
constexpr int kElemPerChunk = tc::kChunkBytes / 4;   // fp32 elements per row per chunk (32)

TcSweepGeom tc_sweep_geom(int ny, int S) {
    TcSweepGeom g;
    g.n = ny - 2;
    g.mt = ceil_div(g.n, 64);
    g.nk = ceil_div(g.n, kElemPerChunk) * kElemPerChunk;
    g.kc = 2 * g.nk / kElemPerChunk;
    g.nt = ceil_div(S, TN);
    g.page_bytes = (size_t)g.mt * g.kc * tc::kAChunk;
    g.b_bytes = (size_t)g.nt * g.kc * (TN * tc::kChunkBytes);
    return g;
}

// Round to TF32 (10-bit mantissa, nearest, ties away).  The tensor core
// would otherwise drop the low mantissa bits of fp32 operands (truncation),
// a bias that accumulates over the column sweep.
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// byte offset of element (row, ke) inside one chunk of a 128-row (or TN-row) tile
__device__ __forceinline__ size_t chunk_off(int row, int ke) {
    return (size_t)(row >> 3) * tc::kRowGroupBytes + (size_t)(ke >> 2) * 128 + (size_t)(row & 7) * 16 + (ke & 3) * 4;
}

// ---------------------------------------------------------------------------
// Pack invT pages into stacked TF32 operands (forward and conjugate transpose).
// One thread per (row of the stacked tile, chunk, page, M-tile), 32 k values.
// ---------------------------------------------------------------------------
__global__ void pack_invT_kernel(const float2 *__restrict__ invT, int ny, int nx, TcSweepGeom g, uint8_t *afwd,
                                 uint8_t *aadj) {
    const int i_s = threadIdx.x;                    // stacked row 0..127
    const int c = blockIdx.x;                       // chunk
    const int mt = blockIdx.y;
    const int j = blockIdx.z;                       // page
    const int i = mt * 64 + (i_s & 63);             // complex interior row
    const bool imrow = i_s >= 64;
    const size_t tile = ((size_t)j * g.mt + mt) * g.kc + c;
    uint8_t *pf = afwd + tile * tc::kAChunk;
    uint8_t *pa = aadj + tile * tc::kAChunk;
    const float2 *page = invT + (size_t)j * ny * ny;
#pragma unroll 4
    for (int ke = 0; ke < kElemPerChunk; ++ke) {
        const int kp = c * kElemPerChunk + ke;      // stacked K index
        const bool imcol = kp >= g.nk;
        const int k = imcol ? kp - g.nk : kp;       // complex interior column
        float vf = 0.f, va = 0.f;
        if (i < g.n && k < g.n) {
            const float2 af = page[(size_t)(i + 1) + (size_t)ny * (k + 1)];           // invT(i, k)
            const float2 at = page[(size_t)(k + 1) + (size_t)ny * (i + 1)];           // invT(k, i)
            const float2 aa = make_float2(at.x, -at.y);                               // invT^H(i, k)
            // [Ar -Ai; Ai Ar]
            vf = imrow ? (imcol ? af.x : af.y) : (imcol ? -af.y : af.x);
            va = imrow ? (imcol ? aa.x : aa.y) : (imcol ? -aa.y : aa.x);
        }
        *reinterpret_cast<float *>(pf + chunk_off(i_s, ke)) = to_tf32(vf);
        *reinterpret_cast<float *>(pa + chunk_off(i_s, ke)) = to_tf32(va);
    }
}

void tc_pack_invT(const float2 *invT, int ny, int nx, const TcSweepGeom &g, uint8_t *afwd, uint8_t *aadj,
                  cudaStream_t st) {
    dim3 grid(g.kc, g.mt, nx);
    pack_invT_kernel<<<grid, 128, 0, st>>>(invT, ny, nx, g, afwd, aadj);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Stencils writing the B operand [Br; Bi] of source s at K rows (y-1, nk+y-1).
// ---------------------------------------------------------------------------
struct TcStencilParams {
    Coefs<float2> co;
    float2 *u;
    const float2 *tmp;     // c64 [ny, S] (ST_UH input)
    SrcView src;
    uint8_t *bt;
    TcSweepGeom g;
    int ny, nx, S, j;
};

__device__ __forceinline__ void put_b(const TcStencilParams &p, int y, int s, float2 v) {
    const int nt = s / TN, row = s % TN;
    const int kr = y - 1, ki = p.g.nk + y - 1;
    uint8_t *base = p.bt + (size_t)nt * p.g.kc * (TN * tc::kChunkBytes);
    *reinterpret_cast<float *>(base + (size_t)(kr / kElemPerChunk) * (TN * tc::kChunkBytes) +
                               chunk_off(row, kr % kElemPerChunk)) = to_tf32(v.x);
    *reinterpret_cast<float *>(base + (size_t)(ki / kElemPerChunk) * (TN * tc::kChunkBytes) +
                               chunk_off(row, ki % kElemPerChunk)) = to_tf32(v.y);
}

enum TcStencil { TS_L = 0, TS_U = 1, TS_LH = 2, TS_PACK = 3, TS_UH = 4 };

template <int MODE>
__global__ void tc_stencil_kernel(TcStencilParams p) {
    const int ny = p.ny, j = p.j;
    const int s = blockIdx.y;
    const size_t fs = (size_t)ny * p.nx * s;
    if (MODE == TS_UH) {   // u(:, j) = SRC_j - U_{j-1}^H tmp, every row (applyBlockLU.cu:159-202)
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
    if (MODE == TS_L) {
        const float2 *uc = p.u + fs + (size_t)ny * (j - 1);
        float2 acc = cmul(p.co.ld(y, j - 1), uc[y]);
        cfma(acc, p.co.ll(y - 1, j - 1), uc[y - 1]);
        cfma(acc, p.co.lu(y, j - 1), uc[y + 1]);
        out = csub(p.src.get(y, j, s, ny, p.nx), acc);
    } else if (MODE == TS_U) {
        const float2 *uc = p.u + fs + (size_t)ny * (j + 1);
        out = cmul(p.co.ud(y, j), uc[y]);
        cfma(out, p.co.ul(y - 1, j), uc[y - 1]);
        cfma(out, p.co.uu(y, j), uc[y + 1]);
    } else if (MODE == TS_LH) {
        const float2 *un = p.u + fs + (size_t)ny * (j + 1);
        float2 acc = make_float2(0.f, 0.f);
        cfma_conj(acc, p.co.ld(y, j), un[y]);
        cfma_conj(acc, p.co.lu(y - 1, j), un[y - 1]);
        cfma_conj(acc, p.co.ll(y, j), un[y + 1]);
        out = csub(p.u[fs + (size_t)ny * j + y], acc);
        // the GEMM that follows rewrites the interior of u(:, j); its border
        // rows are zero after the adjoint back-substitution (invT^H rows)
        if (y == 1) p.u[fs + (size_t)ny * j] = make_float2(0.f, 0.f);
        if (y == ny - 2) p.u[fs + (size_t)ny * j + ny - 1] = make_float2(0.f, 0.f);
    } else {               // TS_PACK: B = u(:, j-1)
        out = p.u[fs + (size_t)ny * (j - 1) + y];
    }
    put_b(p, y, s, out);
}

// ---------------------------------------------------------------------------
// C(i+1, s) (op)= sum_k A(i, k) B(k, s) on one 64-row x TN-source tile,
// split over K across a thread-block cluster of `ksplit` CTAs.  Each CTA
// issues the bulk copies of all its K chunks at once (up to
// kMaxChunksPerCta x 24 KB in flight per SM), accumulates its partial tile
// in TMEM, parks it in shared memory, and after a cluster barrier every CTA
// sums a slice of the columns over all partials through distributed shared
// memory in rank order (deterministic), then writes that slice.
// ---------------------------------------------------------------------------
constexpr int kMaxChunksPerCta = 9;
constexpr int kBChunk = TN * tc::kChunkBytes;             // 8 KB
constexpr int kStageBytes = tc::kAChunk + kBChunk;         // 24 KB
constexpr size_t kGemmSmem = (size_t)kMaxChunksPerCta * kStageBytes + (kMaxChunksPerCta + 2) * 8 + 16;
static_assert((size_t)128 * (TN + 4) * 4 <= (size_t)kMaxChunksPerCta * kStageBytes, "partial tile fits");

struct TcGemmParams {
    const uint8_t *a;        // packed operand of this page: [mt][kc] chunks
    const uint8_t *bt;       // packed B: [nt][kc] chunks
    float2 *c;               // output column: element (row r, source s) at c[r + ldc * s]
    size_t ldc;
    TcSweepGeom g;
    int S;
    int subtract;
    int ksplit, per;         // cluster size along K, chunks per CTA
    int *err;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// 4 consecutive floats of the same shared-memory offset in CTA `rank` of the
// cluster (16-byte aligned).  No memory clobber: the loads of one thread may
// be scheduled together; the cluster barrier before them orders the data.
__device__ __forceinline__ float4 ld_cluster_f32x4(const float *local, uint32_t rank) {
    uint32_t ra;
    asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(tc::smem_u32(local)), "r"(rank));
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(ra));
    return v;
}

template <int KSPLIT>
__global__ void __launch_bounds__(128, 1) tc_gemm_kernel(TcGemmParams p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)kMaxChunksPerCta * kStageBytes);
    uint64_t *done = full + kMaxChunksPerCta;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = blockIdx.x, nt = blockIdx.y, ks = blockIdx.z;   // ks == rank in the (1,1,ksplit) cluster
    const int c0 = ks * p.per;
    const int nch = max(0, min(p.g.kc, c0 + p.per) - c0);

    if (tid == 0) {
        for (int q = 0; q < kMaxChunksPerCta; ++q) tc::mbar_init(&full[q], 1);
        tc::mbar_init(done, 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, TN);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;

    if (tid == 0) {
        const uint8_t *abase = p.a + ((size_t)mt * p.g.kc + c0) * tc::kAChunk;
        const uint8_t *bbase = p.bt + ((size_t)nt * p.g.kc + c0) * kBChunk;
        for (int q = 0; q < nch; ++q) {
            uint8_t *st = smem + (size_t)q * kStageBytes;
            tc::mbar_expect_tx(&full[q], kStageBytes);
            tc::bulk_g2s(st, abase + (size_t)q * tc::kAChunk, tc::kAChunk, &full[q]);
            tc::bulk_g2s(st + tc::kAChunk, bbase + (size_t)q * kBChunk, kBChunk, &full[q]);
        }
        constexpr uint32_t kIdesc = tc::instr_desc<true>(tc::kTileRows, TN);
        bool ok = true;
        for (int q = 0; q < nch; ++q) {
            if (!tc::mbar_wait(&full[q], 0, p.timeout_ns)) {
                ok = false;
                break;
            }
            tc::fence_after();
            const uint8_t *st = smem + (size_t)q * kStageBytes;
#pragma unroll
            for (int k = 0; k < tc::kChunkBytes / 32; ++k)
                tc::mma<true>(tmem, tc::smem_desc(st + k * 256), tc::smem_desc(st + tc::kAChunk + k * 256), kIdesc,
                              (q > 0 || k > 0) ? 1u : 0u);
        }
        if (!ok) {
            atomicCAS(p.err, 0, 1);
            for (int q = 0; q < nch; ++q) tc::mbar_wait(&full[q], 0, p.timeout_ns);   // drain copies in flight
        }
        tc::commit(done);
    }
    __syncthreads();
    const bool ready = tc::mbar_wait(done, 0, p.timeout_ns);
    if (!ready && tid == 0) atomicCAS(p.err, 0, 2);
    tc::fence_after();

    // partial tile -> own shared memory (the operand stages are consumed);
    // rows padded to 68 floats keep float4 stores and loads aligned and
    // conflict-free
    constexpr int PP = TN + 4;
    float *part = reinterpret_cast<float *>(smem);            // [128][PP]
    const int row = 32 * warp + lane;
#pragma unroll
    for (int cb = 0; cb < TN; cb += 8) {
        float t[8];
        if (nch > 0) {
            tc::tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)cb, t);
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) t[q] = 0.f;
        }
        float4 *dst4 = reinterpret_cast<float4 *>(part + row * PP + cb);
        dst4[0] = make_float4(t[0], t[1], t[2], t[3]);
        dst4[1] = make_float4(t[4], t[5], t[6], t[7]);
    }
    tc::fence_before();
    cluster_sync_all();

    // this CTA finalizes columns [ks * CPR, (ks + 1) * CPR); thread -> (row i,
    // half of the slice); all remote loads of a thread are issued before the sums
    constexpr int CPR = TN / KSPLIT, NV = CPR / 8;               // float4 per row per rank
    const int i = tid & 63, half = tid >> 6;
    const int cbeg = ks * CPR + half * (CPR / 2);
    float4 re[KSPLIT][NV], im[KSPLIT][NV];
#pragma unroll
    for (int r = 0; r < KSPLIT; ++r)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            re[r][v] = ld_cluster_f32x4(part + i * PP + cbeg + 4 * v, r);
            im[r][v] = ld_cluster_f32x4(part + (i + 64) * PP + cbeg + 4 * v, r);
        }
    const int gi = mt * 64 + i;                                  // complex interior row
    if (ready && gi < p.g.n) {
        float2 *dst = p.c + (size_t)(gi + 1);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            float4 sr = re[0][v], si = im[0][v];
#pragma unroll
            for (int r = 1; r < KSPLIT; ++r) {
                sr.x += re[r][v].x; sr.y += re[r][v].y; sr.z += re[r][v].z; sr.w += re[r][v].w;
                si.x += im[r][v].x; si.y += im[r][v].y; si.z += im[r][v].z; si.w += im[r][v].w;
            }
            const float vr[4] = {sr.x, sr.y, sr.z, sr.w}, vi[4] = {si.x, si.y, si.z, si.w};
            float2 old[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int s = nt * TN + cbeg + 4 * v + q;
                old[q] = (p.subtract && s < p.S) ? dst[p.ldc * s] : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int s = nt * TN + cbeg + 4 * v + q;
                if (s < p.S)
                    dst[p.ldc * s] = p.subtract ? make_float2(old[q].x - vr[q], old[q].y - vi[q])
                                                : make_float2(vr[q], vi[q]);
            }
        }
    }
    cluster_sync_all();                                          // remote reads done before any CTA exits
    if (warp == 0) tc::tmem_dealloc(tmem, TN);
}

template <int MODE>
static void launch_tc_stencil(const TcStencilParams &p, cudaStream_t st) {
    const int rows = (MODE == TS_UH) ? p.ny : p.ny - 2;
    dim3 grid(ceil_div(rows, 128), p.S);
    tc_stencil_kernel<MODE><<<grid, 128, 0, st>>>(p);
    ++g_kernel_launches;
}

static void launch_tc_gemm(const TcGemmParams &p, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.g.mt, p.g.nt, p.ksplit);
    cfg.blockDim = dim3(128, 1, 1);
    cfg.dynamicSmemBytes = kGemmSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = p.ksplit;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    switch (p.ksplit) {
        case 1: WUST_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<1>, p)); break;
        case 2: WUST_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<2>, p)); break;
        case 4: WUST_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<4>, p)); break;
        default: WUST_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<8>, p)); break;
    }
    ++g_kernel_launches;
}

void tc_sweep_solve(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcSweepGeom &g,
                    const SrcView &src, int S, bool adjoint, float2 *u, float2 *tmp, uint8_t *bt, int *err,
                    cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        WUST_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
        WUST_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
        WUST_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
        WUST_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
        configured = true;
    }
    const int ny = co.ny, nx = co.nx;
    const size_t fld = (size_t)ny * nx;
    TcStencilParams sp;
    sp.co = co; sp.u = u; sp.tmp = tmp; sp.src = src; sp.bt = bt; sp.g = g; sp.ny = ny; sp.nx = nx; sp.S = S;
    TcGemmParams gp;
    gp.bt = bt; gp.g = g; gp.S = S; gp.err = err; gp.timeout_ns = 2000000000ull;
    // K split: smallest power of two that keeps every CTA's chunks in flight at once
    gp.ksplit = 1;
    while (gp.ksplit * kMaxChunksPerCta < g.kc) gp.ksplit *= 2;
    if (gp.ksplit > 8) fail(WUST_ERR_INVALID_INPUT, "grid too large for the tensor-core sweep (K split %d > 8)", gp.ksplit);
    gp.per = ceil_div(g.kc, gp.ksplit);
    WUST_CUDA(cudaMemsetAsync(u, 0, sizeof(float2) * fld * S, st));
    WUST_CUDA(cudaMemsetAsync(bt, 0, g.b_bytes, st));       // K and source padding stay zero
    if (!adjoint) {
        for (int j = 1; j < nx; ++j) {
            sp.j = j;
            launch_tc_stencil<TS_L>(sp, st);
            gp.a = afwd + (size_t)j * g.page_bytes; gp.c = u + (size_t)ny * j; gp.ldc = fld; gp.subtract = 0;
            launch_tc_gemm(gp, st);
        }
        for (int j = nx - 2; j >= 0; --j) {
            sp.j = j;
            launch_tc_stencil<TS_U>(sp, st);
            gp.a = afwd + (size_t)j * g.page_bytes; gp.c = u + (size_t)ny * j; gp.ldc = fld; gp.subtract = 1;
            launch_tc_gemm(gp, st);
        }
    } else {
        WUST_CUDA(cudaMemsetAsync(tmp, 0, sizeof(float2) * (size_t)ny * S, st));
        for (int j = 1; j < nx; ++j) {
            sp.j = j;
            launch_tc_stencil<TS_PACK>(sp, st);
            gp.a = aadj + (size_t)(j - 1) * g.page_bytes; gp.c = tmp; gp.ldc = ny; gp.subtract = 0;
            launch_tc_gemm(gp, st);
            launch_tc_stencil<TS_UH>(sp, st);
        }
        for (int j = nx - 2; j >= 0; --j) {
            sp.j = j;
            launch_tc_stencil<TS_LH>(sp, st);
            gp.a = aadj + (size_t)j * g.page_bytes; gp.c = u + (size_t)ny * j; gp.ldc = fld; gp.subtract = 0;
            launch_tc_gemm(gp, st);
        }
    }
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
