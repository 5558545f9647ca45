// Block-tridiagonal sweeps of applyBlockLU (Runtime/solver/applyBlockLU.cu:433-467)
// with the dense invT_j products on the tensor cores (tcgen05, TF32 inputs,
// FP32 accumulation in tensor memory).  Used by the refined TF32 profile:
// the FP64-residual refinement in api.cu restores full accuracy.
//
// One persistent cooperative kernel runs a whole solve (forward sweep, then
// backward sweep): every column step is one complex GEMM
//     C (n x S) = invT_j (n x n) * B (n x S),   B = base - stencil(previous column),
// followed by a barrier among the CTAs that share the step's sources.
//
// Complex products are one real GEMM with re/im interleaved along K:
//     row r of Cr:  sum_k  Ar(r,k) Br(k) - Ai(r,k) Bi(k)   -> A pair (Ar, -Ai)
//     row r of Ci:  sum_k  Ai(r,k) Br(k) + Ar(r,k) Bi(k)   -> A pair (Ai,  Ar)
// so B is the complex column itself (re, im, re, im, ...) and a 128-row A
// tile holds 64 complex rows (rows 0-63 give Cr, rows 64-127 give Ci).
//
// Work split: output tiles of 64 complex rows x 64 sources; the K range of a
// tile is split over `ks` <= 4 CTAs (at most 9 K chunks of 16 complex rows
// each, so every CTA keeps its whole A slice and B slice in shared memory).
// Grid = (M tiles, source tiles, ks), one CTA per SM, launched cooperatively;
// the CTAs of one source tile form a group that synchronises through one
// monotonic counter, and groups of different sources never wait on each other.
//
// Per step and CTA (8 warps):
//   bulk-copy this step's packed B chunks (produced once per chunk, below)
//     into shared memory; one thread issues the MMAs; the next step's A
//     chunks are copied (cp.async.bulk) as soon as they retire, so the HBM
//     stream of invT overlaps the epilogue and the barriers;
//   TMEM -> split-K partial tile in L2; prefetch the next step's static
//     inputs; group barrier;
//   each CTA owns whole K chunks (16 rows) of the next B: it sums the split-K
//     partials of those rows plus a 2-row halo (fixed rank order, so results
//     are deterministic), finishes column j of u for them, evaluates the
//     stencil of the next step and writes the packed chunk to L2; group
//     barrier.
// So every B value is computed once, and the only data exchanged per step
// is the partial tiles and the packed B chunks.  Every wait is bounded and
// reports its site through *err.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"
#include "tcstep.cuh"

namespace wust {

constexpr int TN = 64;                       // sources per tile (MMA N)
constexpr int kRowsPerChunk = 16;            // complex rows per K chunk (32 fp32 K values)
constexpr int kMaxPer = 9;                   // K chunks per CTA
constexpr int kMaxKSplit = 4;
constexpr int kSweepThreads = 256;
constexpr int kMaxOwned = 3;                        // B chunks produced per CTA and step
constexpr int kBChunk = TN * tc::kChunkBytes;       // 8 KB
constexpr size_t kSmemA = (size_t)kMaxPer * tc::kAChunk;
constexpr size_t kSmemB = (size_t)kMaxPer * kBChunk;
constexpr size_t kSmemBar = 256;
constexpr size_t kSweepSmem = kSmemA + kSmemB + kSmemBar;
static_assert(kSweepSmem <= 232448, "shared memory of one CTA");

using tc::chunk_off;
using tc::to_tf32;

TcSweepGeom tc_sweep_geom(int ny, int S, int max_ctas) {
    TcSweepGeom g{};
    g.n = ny - 2;
    g.mt = ceil_div(g.n, 64);
    g.kc = ceil_div(g.n, kRowsPerChunk);
    g.ks = 1;
    while (g.ks * kMaxPer < g.kc) g.ks *= 2;
    if (g.ks > kMaxKSplit)
        fail(WUST_ERR_INVALID_INPUT, "tensor-core sweep supports Ny <= %d (got %d)",
             kMaxKSplit * kMaxPer * kRowsPerChunk + 2, ny);
    // every CTA of a source tile produces at most kMaxOwned B chunks per step
    while (g.kc > kMaxOwned * g.mt * g.ks && g.ks < kMaxKSplit) g.ks *= 2;
    if (g.kc > kMaxOwned * g.mt * g.ks)
        fail(WUST_ERR_INVALID_INPUT, "tensor-core sweep: grid shape Ny = %d not supported", ny);
    g.per = ceil_div(g.kc, g.ks);
    const int per_tile = g.mt * g.ks;
    if (per_tile > max_ctas)
        fail(WUST_ERR_INVALID_INPUT, "tensor-core sweep needs %d co-resident CTAs per source tile (device holds %d)",
             per_tile, max_ctas);
    g.nt = std::max(1, std::min(ceil_div(std::max(S, 1), TN), max_ctas / per_tile));
    g.page_bytes = (size_t)g.mt * g.kc * tc::kAChunk;
    g.part_bytes = (size_t)g.mt * g.nt * g.ks * 128 * TN * sizeof(float);
    g.b_bytes = (size_t)g.nt * g.kc * kBChunk;
    g.sync_words = g.nt;
    return g;
}

// ---------------------------------------------------------------------------
// Pack invT pages into the interleaved real-split TF32 operands of invT_j and
// invT_j^H.  One thread per (row of the 128-row tile, chunk, M tile, page).
// ---------------------------------------------------------------------------
__global__ void pack_invT_kernel(const float2 *__restrict__ invT, int ny, TcSweepGeom g, uint8_t *afwd,
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
#pragma unroll 2
    for (int k4 = 0; k4 < 8; ++k4) {                // 4 K values = 2 complex columns
        float vf[4], va[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = c * kRowsPerChunk + 2 * k4 + h;   // complex interior column
            float2 af = make_float2(0.f, 0.f), aa = af;
            if (i < g.n && k < g.n) {
                af = page[(size_t)(i + 1) + (size_t)ny * (k + 1)];                  // invT(i, k)
                const float2 at = page[(size_t)(k + 1) + (size_t)ny * (i + 1)];     // invT(k, i)
                aa = make_float2(at.x, -at.y);                                      // invT^H(i, k)
            }
            vf[2 * h] = imrow ? af.y : af.x;
            vf[2 * h + 1] = imrow ? af.x : -af.y;
            va[2 * h] = imrow ? aa.y : aa.x;
            va[2 * h + 1] = imrow ? aa.x : -aa.y;
        }
        *reinterpret_cast<float4 *>(pf + chunk_off(i_s, 4 * k4)) =
            make_float4(to_tf32(vf[0]), to_tf32(vf[1]), to_tf32(vf[2]), to_tf32(vf[3]));
        *reinterpret_cast<float4 *>(pa + chunk_off(i_s, 4 * k4)) =
            make_float4(to_tf32(va[0]), to_tf32(va[1]), to_tf32(va[2]), to_tf32(va[3]));
    }
}

void tc_pack_invT(const float2 *invT, int ny, int nx, const TcSweepGeom &g, uint8_t *afwd, uint8_t *aadj,
                  cudaStream_t st) {
    dim3 grid(g.kc, g.mt, nx);
    pack_invT_kernel<<<grid, 128, 0, st>>>(invT, ny, g, afwd, aadj);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Persistent sweep kernel.
// ---------------------------------------------------------------------------
struct SweepParams {
    const uint8_t *apack;     // packed pages (invT or invT^H): [page][mt][kc] chunks
    size_t page_bytes;
    Coefs<float2> co;
    SrcView src;
    float2 *u;                // [ny, nx, S] (global source index)
    uint8_t *bglob;           // packed B chunks of the next step: [nt][kc] x kBChunk
    float *part;              // [tile][ks][128][TN]
    unsigned *group_ctr;      // [nt]
    int *err;
    int ny, nx, n, mt, kc, ks, per;
    int s0, s_end;            // global sources [s0, s_end) of this launch
    unsigned long long timeout_ns;
};


// Optional phase timer (SM cycles of CTA (0,0,0), summed over steps), built
// only into profiling builds of the library.
#ifdef WUST_SWEEP_PROFILE
__device__ unsigned long long g_sweep_prof[16];
#define SPROF(k)                                                                                   \
    do {                                                                                           \
        if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) {          \
            const long long t_ = clock64();                                                        \
            g_sweep_prof[k] += (unsigned long long)(t_ - prof_t);                                  \
            prof_t = t_;                                                                           \
        }                                                                                          \
    } while (0)
extern "C" int wust_sweep_profile_read(unsigned long long *out) {
    return (int)cudaMemcpyFromSymbol(out, g_sweep_prof, sizeof(g_sweep_prof));
}
extern "C" int wust_sweep_profile_reset() {
    unsigned long long z[16] = {};
    return (int)cudaMemcpyToSymbol(g_sweep_prof, z, sizeof(z));
}
#else
#define SPROF(k) ((void)0)
#endif

// Shared-memory scratch of the reduce/produce phase (inside the B stage area,
// which is free between the MMAs and the next step's B copy).
constexpr int kHalo = 2;
constexpr int kCRows = kRowsPerChunk + 2 * kHalo;          // 20
constexpr size_t kOffC = 0;                                 // c: [kCRows][TN] float2
constexpr size_t kOffC2 = kOffC + (size_t)kCRows * TN * 8;  // transformed c (ADJ fwd -> bwd turn)
constexpr size_t kOffStage = kOffC2 + (size_t)kCRows * TN * 8;
constexpr size_t kOffPre = kOffStage + kBChunk;             // prefetch: [kMaxOwned][kCRows][TN] float2
constexpr size_t kOffW = kOffPre + (size_t)kMaxOwned * kCRows * TN * 8;   // weights: [kMaxOwned][3][16] float2
static_assert(kOffW + (size_t)kMaxOwned * 3 * kRowsPerChunk * 8 <= kSmemB, "reduce scratch fits the B stage area");

template <bool ADJ, int KS>
__global__ void __launch_bounds__(kSweepThreads, 1) tc_sweep_kernel(SweepParams p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;
    uint8_t *sB = smem + kSmemA;
    uint64_t *full = reinterpret_cast<uint64_t *>(sB + kSmemB);
    uint64_t *done = full + kMaxPer;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *s_ok = reinterpret_cast<int *>(tmem_slot + 1);
    float2 *cbuf = reinterpret_cast<float2 *>(sB + kOffC);
    float2 *cbuf2 = reinterpret_cast<float2 *>(sB + kOffC2);
    uint8_t *stage = sB + kOffStage;
    float2 *pre = reinterpret_cast<float2 *>(sB + kOffPre);
    float2 *wbuf = reinterpret_cast<float2 *>(sB + kOffW);

    const int tid = threadIdx.x, warp = tid >> 5;
    const int mt = blockIdx.x, nt = blockIdx.y, ks = blockIdx.z;
    const int ny = p.ny, nx = p.nx, n = p.n;
    const size_t plane = (size_t)ny * nx;
    const int c0 = ks * p.per;
    const int nch = max(0, min(p.kc, c0 + p.per) - c0);
    const int tile = mt + p.mt * nt;
    const int G = p.mt * KS;                       // CTAs of this source tile
    const int rank = mt + p.mt * ks;               // this CTA's rank among them
    const int nsteps = 2 * (nx - 1);
    uint8_t *bg = p.bglob + (size_t)nt * p.kc * kBChunk;
    const int sbase = p.s0 + nt * TN;              // global index of source 0 of this tile

    if (tid == 0) {
        for (int q = 0; q < kMaxPer; ++q) tc::mbar_init(&full[q], 2);   // A copy + B copy of chunk q
        tc::mbar_init(done, 1);
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, TN);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;

    // A chunks of step i: page j (forward sweep of H^H: page j-1)
    auto issue_a = [&](int i) {
        bool f;
        const int jj = step_col(i, nx, f);
        const int page = (ADJ && f) ? jj - 1 : jj;
        const uint8_t *abase = p.apack + (size_t)page * p.page_bytes + ((size_t)mt * p.kc + c0) * tc::kAChunk;
        for (int q = 0; q < nch; ++q) {
            tc::mbar_expect_tx(&full[q], tc::kAChunk);
            tc::bulk_g2s(sA + (size_t)q * tc::kAChunk, abase + (size_t)q * tc::kAChunk, tc::kAChunk, &full[q]);
        }
    };

    // Produce the packed B chunk Q of step (fwd1, j1) from c (rows 16Q-2 ..
    // 16Q+17 at cbuf rows 0..19) and the prefetched base (pre_k rows 0..15);
    // ADJ forward steps also write B into u(:, j1-1) (with its border rows).
    auto produce = [&](int Q, const float2 *c, const float2 *pre_k, const float2 *w_k, bool fwd1, int j1) {
        const int s_l = tid & (TN - 1);
        const int s = sbase + s_l;
        const bool sv = s < p.s_end;
        for (int yl = tid >> 6; yl < kRowsPerChunk; yl += kSweepThreads / TN) {
            const int yp = kRowsPerChunk * Q + yl, y = yp + 1;
            float2 b = f2(0.f, 0.f);
            if (sv && yp < n) {
                const int r = yl + kHalo;
                float2 acc = cmul(w_k[yl], c[r * TN + s_l]);
                cfma(acc, w_k[kRowsPerChunk + yl], c[(r - 1) * TN + s_l]);
                cfma(acc, w_k[2 * kRowsPerChunk + yl], c[(r + 1) * TN + s_l]);
                b = csub(pre_k[yl * TN + s_l], acc);
                if (ADJ && fwd1) p.u[plane * s + (size_t)ny * (j1 - 1) + y] = b;
            }
            *reinterpret_cast<float2 *>(stage + chunk_off(s_l, 2 * yl)) = f2(to_tf32(b.x), to_tf32(b.y));
        }
        if (ADJ && fwd1 && sv && tid < TN) {
            // border rows 0 and ny-1 of u(:, j1-1) (no B entry)
            for (int e = 0; e < 2; ++e) {
                const int yp = e == 0 ? -1 : n;
                const int r = yp - kRowsPerChunk * Q + kHalo;
                if (r < 1 || r > kCRows - 2) continue;
                const int y = yp + 1;
                float2 wc, wm, wp;
                step_weights<ADJ>(p.co, fwd1, j1, y, wc, wm, wp);
                float2 acc = cmul(wc, c[r * TN + s_l]);
                cfma(acc, wm, c[(r - 1) * TN + s_l]);
                cfma(acc, wp, c[(r + 1) * TN + s_l]);
                p.u[plane * s + (size_t)ny * (j1 - 1) + y] = csub(step_base<ADJ>(p.src, p.u, ny, nx, fwd1, j1, y, s), acc);
            }
        }
        __syncthreads();
        const float4 *src4 = reinterpret_cast<const float4 *>(stage);
        float4 *dst4 = reinterpret_cast<float4 *>(bg + (size_t)Q * kBChunk);
        for (int v = tid; v < kBChunk / 16; v += kSweepThreads) dst4[v] = src4[v];
        __syncthreads();
    };

    // Prefetch (static data of the next step, or the old column that a
    // subtracting step needs) for owned chunk Q into pre_k.
    auto prefetch = [&](int Q, float2 *pre_k, float2 *w_k, bool fwd1, int j1, bool old_of_j, int j) {
        constexpr int kItems = kCRows * TN / kSweepThreads;   // 5: all loads in flight before any store
        float2 v[kItems];
#pragma unroll
        for (int m = 0; m < kItems; ++m) {
            const int idx = tid + kSweepThreads * m;
            const int s_l = idx / kCRows, r = idx % kCRows;    // consecutive rows per source
            const int s = sbase + s_l;
            v[m] = f2(0.f, 0.f);
            if (s < p.s_end) {
                if (old_of_j) {
                    const int yp = kRowsPerChunk * Q - kHalo + r;
                    if (yp >= 0 && yp < n) v[m] = __ldcg(p.u + plane * s + (size_t)ny * j + yp + 1);
                } else if (r < kRowsPerChunk) {
                    const int yp = kRowsPerChunk * Q + r;
                    if (yp < n) v[m] = step_base<ADJ>(p.src, p.u, p.ny, p.nx, fwd1, j1, yp + 1, s);
                }
            }
        }
        if (tid < kRowsPerChunk) {
            const int yp = kRowsPerChunk * Q + tid;
            float2 wc = f2(0.f, 0.f), wm = wc, wp = wc;
            if (yp < n) step_weights<ADJ>(p.co, fwd1, j1, yp + 1, wc, wm, wp);
            w_k[tid] = wc;
            w_k[kRowsPerChunk + tid] = wm;
            w_k[2 * kRowsPerChunk + tid] = wp;
        }
#pragma unroll
        for (int m = 0; m < kItems; ++m) {
            const int idx = tid + kSweepThreads * m;
            pre_k[(idx % kCRows) * TN + idx / kCRows] = v[m];
        }
    };

    int a_step = -1;          // step whose A copies are in flight (thread 0)
    if (tid == 0 && nch > 0) {
        issue_a(0);
        a_step = 0;
    }
    unsigned group_epoch = 0;
    bool ok = true;
#ifdef WUST_SWEEP_PROFILE
    long long prof_t = clock64();
#endif

    // prologue: B of step 0 from c = 0
    {
        bool f0;
        const int j0 = step_col(0, nx, f0);
        for (int k = 0, Q = rank; Q < p.kc; ++k, Q += G) {
            for (int idx = tid; idx < kCRows * TN; idx += kSweepThreads) cbuf[idx] = f2(0.f, 0.f);
            prefetch(Q, pre, wbuf, f0, j0, false, 0);
            __syncthreads();
            produce(Q, cbuf, pre, wbuf, f0, j0);
        }
        group_epoch += (unsigned)G;
        ok = counter_sync(p.group_ctr + nt, group_epoch, p.err, s_ok, p.timeout_ns, SITE_B);
    }

    for (int i = 0; i < nsteps && ok; ++i) {
        bool fwd;
        const int j = step_col(i, nx, fwd);
        SPROF(0);

        // ---- B of this step -> shared memory; MMAs (one thread) -------------
        if (tid == 0) {
            for (int q = 0; q < nch; ++q) {
                tc::mbar_expect_tx(&full[q], kBChunk);
                tc::bulk_g2s(sB + (size_t)q * kBChunk, bg + (size_t)(c0 + q) * kBChunk, kBChunk, &full[q]);
            }
            constexpr uint32_t kIdesc = tc::instr_desc<true>(tc::kTileRows, TN);
            int got = 0;
            for (int q = 0; q < nch; ++q) {
                if (!tc::mbar_wait(&full[q], (uint32_t)(i & 1), p.timeout_ns)) break;
                ++got;
                tc::fence_after();
#pragma unroll
                for (int k = 0; k < tc::kChunkBytes / 32; ++k)
                    tc::mma<true>(tmem, tc::smem_desc(sA + (size_t)q * tc::kAChunk + k * 256),
                                  tc::smem_desc(sB + (size_t)q * kBChunk + k * 256), kIdesc,
                                  (q > 0 || k > 0) ? 1u : 0u);
            }
            if (got < nch) {
                atomicCAS(p.err, 0, SITE_COPY);
                for (int q = got; q < nch; ++q) tc::mbar_wait(&full[q], (uint32_t)(i & 1), p.timeout_ns);
            }
            a_step = -1;
            tc::commit(done);
        }
        SPROF(1);
        if (!tc::mbar_wait(done, (uint32_t)(i & 1), p.timeout_ns)) atomicCAS(p.err, 0, SITE_MMA);
        tc::fence_after();
        if (tid == 0) *s_ok = (*(volatile int *)p.err == 0);
        __syncthreads();
        if (!*s_ok) {
            ok = false;
            break;
        }
        if (tid == 0 && i + 1 < nsteps && nch > 0) {
            issue_a(i + 1);                  // stages are free: this step's MMAs retired
            a_step = i + 1;
        }
        SPROF(2);

        // ---- partial tile -> L2 (warp w: TMEM lanes 32(w%4).., 32 columns) -----
        {
            const int row = 32 * (warp & 3) + (tid & 31);
            const int cbase = 32 * (warp >> 2);
            float *mypart = p.part + ((size_t)(tile * KS + ks) * 128 + row) * TN + cbase;
#pragma unroll
            for (int cb = 0; cb < 32; cb += 8) {
                float t[8];
                if (nch > 0) {
                    tc::tmem_ld8(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(cbase + cb), t);
                } else {
#pragma unroll
                    for (int q = 0; q < 8; ++q) t[q] = 0.f;
                }
                __stcg(reinterpret_cast<float4 *>(mypart + cb), make_float4(t[0], t[1], t[2], t[3]));
                __stcg(reinterpret_cast<float4 *>(mypart + cb + 4), make_float4(t[4], t[5], t[6], t[7]));
            }
        }
        tc::fence_before();
        // static inputs of the next step (or the old column of a subtracting
        // step) for the owned chunks, read before anyone rewrites column j
        bool fwd1 = false;
        int j1 = 0;
        const bool has_next = i + 1 < nsteps;
        if (has_next) j1 = step_col(i + 1, nx, fwd1);
        const bool sub = !ADJ && !fwd;
        for (int k = 0, Q = rank; Q < p.kc; ++k, Q += G) {
            float2 *pre_k = pre + (size_t)k * kCRows * TN;
            float2 *w_k = wbuf + (size_t)k * 3 * kRowsPerChunk;
            if (sub) prefetch(Q, pre_k, w_k, fwd1, j1, true, j);
            else if (has_next) prefetch(Q, pre_k, w_k, fwd1, j1, false, j);
        }
        SPROF(3);
        group_epoch += (unsigned)G;
        if (!counter_sync(p.group_ctr + nt, group_epoch, p.err, s_ok, p.timeout_ns, SITE_GROUP)) {
            ok = false;
            break;
        }
        tc::fence_after();
        SPROF(4);

        // ---- owned chunks: reduce the K split, finish column j, produce B ------
        for (int k = 0, Q = rank; Q < p.kc; ++k, Q += G) {
            float2 *pre_k = pre + (size_t)k * kCRows * TN;
            {
                const int s_l = tid & (TN - 1);
#pragma unroll
                for (int rr = 0; rr < kCRows / 4; ++rr) {
                    const int r = (tid >> 6) + 4 * rr;
                    const int yp = kRowsPerChunk * Q - kHalo + r;
                    float2 v = f2(0.f, 0.f);
                    if (yp >= 0 && yp < n) {
                        const int t2 = yp / 64 + p.mt * nt, rw = yp % 64;
                        const float *pt = p.part + (size_t)t2 * KS * 128 * TN + (size_t)rw * TN + s_l;
                        float re[KS], im[KS];
#pragma unroll
                        for (int q = 0; q < KS; ++q) {
                            re[q] = __ldcg(pt + (size_t)q * 128 * TN);
                            im[q] = __ldcg(pt + (size_t)q * 128 * TN + 64 * TN);
                        }
#pragma unroll
                        for (int q = 0; q < KS; ++q) { v.x += re[q]; v.y += im[q]; }
                        if (sub) {
                            const float2 o = pre_k[r * TN + s_l];
                            v = f2(o.x - v.x, o.y - v.y);
                        }
                    }
                    cbuf[r * TN + s_l] = v;
                }
            }
            __syncthreads();
            const float2 *c = cbuf;
            if (ADJ && fwd && j == nx - 1) {
                // turn of the H^H solve: w = u(:, nx-1) = SRC_{nx-1} - U_{nx-2}^H t, every row
                for (int idx = tid; idx < kCRows * TN; idx += kSweepThreads) {
                    const int r = idx / TN, s_l = idx % TN;
                    const int yp = kRowsPerChunk * Q - kHalo + r, y = yp + 1;
                    const int s = sbase + s_l;
                    float2 w = f2(0.f, 0.f);
                    if (r >= 1 && r <= kCRows - 2 && y >= 0 && y <= ny - 1 && s < p.s_end) {
                        float2 acc = f2(0.f, 0.f);
                        cfma_conj(acc, p.co.ud(y, nx - 2), cbuf[r * TN + s_l]);
                        if (y > 0) cfma_conj(acc, p.co.uu(y - 1, nx - 2), cbuf[(r - 1) * TN + s_l]);
                        if (y < ny - 1) cfma_conj(acc, p.co.ul(y, nx - 2), cbuf[(r + 1) * TN + s_l]);
                        w = csub(p.src.get(y, nx - 1, s, ny, nx), acc);
                        const bool own = (yp >= kRowsPerChunk * Q && yp < kRowsPerChunk * (Q + 1) && yp < n) ||
                                         (yp == -1) || (yp == n);
                        if (own) p.u[plane * s + (size_t)ny * (nx - 1) + y] = w;
                    }
                    cbuf2[idx] = w;
                }
                __syncthreads();
                c = cbuf2;
            }
            // finished column j of u (own rows; ADJ backward: zero border rows)
            if (!ADJ || !fwd) {
                for (int idx = tid; idx < kRowsPerChunk * TN; idx += kSweepThreads) {
                    const int s_l = idx / kRowsPerChunk, yl = idx % kRowsPerChunk;
                    const int yp = kRowsPerChunk * Q + yl;
                    const int s = sbase + s_l;
                    if (yp < n && s < p.s_end) p.u[plane * s + (size_t)ny * j + yp + 1] = c[(yl + kHalo) * TN + s_l];
                }
                if (ADJ && tid < TN && sbase + tid < p.s_end) {
                    const int s = sbase + tid;
                    if (Q == 0) p.u[plane * s + (size_t)ny * j] = f2(0.f, 0.f);
                    if (Q == p.kc - 1) p.u[plane * s + (size_t)ny * j + ny - 1] = f2(0.f, 0.f);
                }
            }
            if (has_next) {
                if (sub) {
                    // the subtracting step's prefetch held the old column; the
                    // next step (also backward) has base 0
                    for (int idx = tid; idx < kCRows * TN; idx += kSweepThreads) pre_k[idx] = f2(0.f, 0.f);
                    __syncthreads();
                }
                produce(Q, c, pre_k, wbuf + (size_t)k * 3 * kRowsPerChunk, fwd1, j1);
            } else {
                __syncthreads();
            }
        }
        SPROF(5);
        if (has_next) {
            group_epoch += (unsigned)G;
            if (!counter_sync(p.group_ctr + nt, group_epoch, p.err, s_ok, p.timeout_ns, SITE_B)) {
                ok = false;
                break;
            }
        }
        SPROF(6);
    }

    // A copies still in flight after a failure: stand in for the B arrival
    // that will not come, then let them land (bounded)
    if (tid == 0 && a_step >= 0)
        for (int q = 0; q < nch; ++q) {
            tc::mbar_arrive(&full[q]);
            tc::mbar_wait(&full[q], (uint32_t)(a_step & 1), p.timeout_ns);
        }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, TN);
}

template <bool ADJ, int KS>
static void configure_one() {
    WUST_CUDA(cudaFuncSetAttribute(tc_sweep_kernel<ADJ, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kSweepSmem));
}
static void configure_all() {
    // before every launch: the attribute lives in the current device's context
    configure_one<false, 1>(); configure_one<false, 2>(); configure_one<false, 4>();
    configure_one<true, 1>(); configure_one<true, 2>(); configure_one<true, 4>();
}

int tc_sweep_max_ctas() {
    configure_all();
    int dev = 0, sms = 0, per_sm = 0;
    WUST_CUDA(cudaGetDevice(&dev));
    WUST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WUST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc_sweep_kernel<false, 4>, kSweepThreads,
                                                            kSweepSmem));
    return sms * per_sm;
}

template <bool ADJ>
static void launch_sweep(const SweepParams &p, dim3 grid, cudaStream_t st) {
    void *args[] = {const_cast<SweepParams *>(&p)};
    const dim3 block(kSweepThreads);
    switch (p.ks) {
        case 1:
            WUST_CUDA(cudaLaunchCooperativeKernel((void *)tc_sweep_kernel<ADJ, 1>, grid, block, args, kSweepSmem, st));
            break;
        case 2:
            WUST_CUDA(cudaLaunchCooperativeKernel((void *)tc_sweep_kernel<ADJ, 2>, grid, block, args, kSweepSmem, st));
            break;
        default:
            WUST_CUDA(cudaLaunchCooperativeKernel((void *)tc_sweep_kernel<ADJ, 4>, grid, block, args, kSweepSmem, st));
            break;
    }
    ++g_kernel_launches;
}

void tc_sweep_solve(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcSweepGeom &g,
                    const SrcView &src, int S, bool adjoint, float2 *u, uint8_t *bglob, float *part, unsigned *sync,
                    int *err, cudaStream_t st) {
    configure_all();
    const int ny = co.ny, nx = co.nx;
    if (nx < 2) fail(WUST_ERR_INVALID_INPUT, "tensor-core sweep needs Nx >= 2");
    WUST_CUDA(cudaMemsetAsync(u, 0, sizeof(float2) * (size_t)ny * nx * S, st));
    SweepParams p;
    p.apack = adjoint ? aadj : afwd;
    p.page_bytes = g.page_bytes;
    p.co = co;
    p.src = src;
    p.u = u;
    p.bglob = bglob;
    p.part = part;
    p.err = err;
    p.ny = ny;
    p.nx = nx;
    p.n = g.n;
    p.mt = g.mt;
    p.kc = g.kc;
    p.ks = g.ks;
    p.per = g.per;
    p.timeout_ns = 1000000000ull;
    for (int s0 = 0; s0 < S; s0 += g.nt * TN) {
        const int s_end = std::min(S, s0 + g.nt * TN);
        const int nt = ceil_div(s_end - s0, TN);
        WUST_CUDA(cudaMemsetAsync(sync, 0, sizeof(unsigned) * g.sync_words, st));
        p.s0 = s0;
        p.s_end = s_end;
        p.group_ctr = sync;
        const dim3 grid(g.mt, nt, g.ks);
        if (adjoint) launch_sweep<true>(p, grid, st);
        else launch_sweep<false>(p, grid, st);
    }
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
