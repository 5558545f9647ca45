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
// The split-K partial tiles go through L2 and each CTA of the tile sums one
// column slice in rank order (deterministic).  Grid = (M tiles, source tiles,
// ks), one CTA per SM, launched cooperatively; tiles of different sources
// never wait on each other.
//
// Per step and CTA (8 warps):
//   stage B: every load the step depends on is issued at once (the previous
//     column, the base term, two edge rows), then the stencil is evaluated
//     with weights staged in shared memory and written straight into the MMA
//     operand layout;
//   one thread issues the MMAs; the next step's A chunks are copied
//     (cp.async.bulk) as soon as they retire, so the HBM stream of invT
//     overlaps the epilogue and the barriers;
//   partial tile -> L2, next step's weights -> shared memory, tile barrier,
//   reduce one column slice, write the column, group barrier.
// Every wait is bounded and reports its site through *err.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace wust {

constexpr int TN = 64;                       // sources per tile (MMA N)
constexpr int kRowsPerChunk = 16;            // complex rows per K chunk (32 fp32 K values)
constexpr int kMaxPer = 9;                   // K chunks per CTA
constexpr int kMaxKSplit = 4;
constexpr int kMaxRows = kMaxPer * kRowsPerChunk;   // 144 complex rows per CTA
constexpr int kQuads = kMaxRows / 4;                // 36 row quads
constexpr int kSweepThreads = 256;
constexpr int kBChunk = TN * tc::kChunkBytes;       // 8 KB
constexpr size_t kSmemA = (size_t)kMaxPer * tc::kAChunk;
constexpr size_t kSmemB = (size_t)kMaxPer * kBChunk;
constexpr size_t kSmemBar = 256;
constexpr size_t kSmemW = 3 * kMaxRows * sizeof(float2);
constexpr size_t kSweepSmem = kSmemA + kSmemB + kSmemBar + kSmemW;
static_assert(kSweepSmem <= 232448, "shared memory of one CTA");

// byte offset of element (row, ke) inside one chunk of a 128-row (or TN-row) tile
__host__ __device__ __forceinline__ size_t chunk_off(int row, int ke) {
    return (size_t)(row >> 3) * tc::kRowGroupBytes + (size_t)(ke >> 2) * 128 + (size_t)(row & 7) * 16 + (ke & 3) * 4;
}

// Round to TF32 (10-bit mantissa, nearest, ties away).  The tensor core
// would otherwise drop the low mantissa bits of fp32 operands (truncation),
// a bias that accumulates over the column sweep.  Integer form (two ALU
// ops): add half of the 13 dropped bits to the magnitude, clear them.  Inf
// and NaN pass unchanged.
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    return __uint_as_float(u);
}

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
    g.per = ceil_div(g.kc, g.ks);
    const int per_tile = g.mt * g.ks;
    if (per_tile > max_ctas)
        fail(WUST_ERR_INVALID_INPUT, "tensor-core sweep needs %d co-resident CTAs per source tile (device holds %d)",
             per_tile, max_ctas);
    g.nt = std::max(1, std::min(ceil_div(std::max(S, 1), TN), max_ctas / per_tile));
    g.page_bytes = (size_t)g.mt * g.kc * tc::kAChunk;
    g.part_bytes = (size_t)g.mt * g.nt * g.ks * 128 * TN * sizeof(float);
    g.tmp_elems = 2 * (size_t)ny * g.nt * TN;
    g.sync_words = g.nt + g.mt * g.nt;
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
    float2 *tmp;              // adjoint: two [ny, tb] buffers (launch-local source index)
    float *part;              // [tile][ks][128][TN]
    unsigned *group_ctr;      // [nt]
    unsigned *tile_ctr;       // [mt * nt]
    int *err;
    int ny, nx, n, mt, kc, ks, per;
    int s0, s_end, tb;        // global sources [s0, s_end) of this launch; tmp row pitch tb
    unsigned long long timeout_ns;
};

// Device-wait sites reported through *err.
enum { SITE_COPY = 1, SITE_MMA = 2, SITE_TILE = 3, SITE_GROUP = 4 };

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

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// Arrive on a monotonic counter and wait until it reaches target (bounded).
// __syncthreads on both sides; the result is uniform over the CTA and false
// when this or another CTA gave up.
__device__ __forceinline__ bool counter_sync(unsigned *ctr, unsigned target, int *err, int *s_ok,
                                             unsigned long long timeout_ns, int site) {
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(ctr), "r"(1u) : "memory");
        int ok = 1;
        const unsigned long long t0 = global_timer_ns();
        for (unsigned spin = 0;; ++spin) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
            if ((int)(v - target) >= 0) break;
            if ((spin & 15u) == 15u) {
                if (*(volatile int *)err) { ok = 0; break; }
                if (global_timer_ns() - t0 > timeout_ns) {
                    atomicCAS(err, 0, site);
                    ok = 0;
                    break;
                }
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Column index of step i and its direction.
__device__ __forceinline__ int step_col(int i, int nx, bool &fwd) {
    fwd = i < nx - 1;
    return fwd ? 1 + i : (nx - 2) - (i - (nx - 1));
}

// Stencil weights of step (fwd, j) for this CTA's rows, so that
//     B(y) = base(y) - (wc(y) c(y) + wm(y) c(y-1) + wp(y) c(y+1)),
// c = the column the step depends on:
//   !ADJ fwd: L_{j-1} of u(:, j-1)     base = SRC_j
//   !ADJ bwd: -U_j of u(:, j+1)         base = 0
//   ADJ fwd:  U_{j-2}^H of tmp          base = SRC_{j-1}   (j == 1: B = u(:, 0))
//   ADJ bwd:  L_j^H of u(:, j+1)        base = u(:, j)
template <bool ADJ>
__device__ __forceinline__ void stage_weights(const SweepParams &p, float2 *w, int y0, int rows, bool fwd, int j) {
    const Coefs<float2> &co = p.co;
    for (int r = threadIdx.x; r < rows; r += kSweepThreads) {
        const int yp = y0 + r, y = yp + 1;
        float2 wc = f2(0.f, 0.f), wm = wc, wp = wc;
        if (yp < p.n) {
            if (!ADJ && fwd) {
                wc = co.ld(y, j - 1); wm = co.ll(y - 1, j - 1); wp = co.lu(y, j - 1);
            } else if (!ADJ) {
                wc = co.ud(y, j); wm = co.ul(y - 1, j); wp = co.uu(y, j);
                wc = f2(-wc.x, -wc.y); wm = f2(-wm.x, -wm.y); wp = f2(-wp.x, -wp.y);
            } else if (fwd) {
                if (j >= 2) {
                    wc = cconj(co.ud(y, j - 2)); wm = cconj(co.uu(y - 1, j - 2)); wp = cconj(co.ul(y, j - 2));
                } else {
                    wc = f2(-1.f, 0.f);
                }
            } else {
                wc = cconj(co.ld(y, j)); wm = cconj(co.lu(y - 1, j)); wp = cconj(co.ll(y, j));
            }
        }
        w[r] = wc;
        w[kMaxRows + r] = wm;
        w[2 * kMaxRows + r] = wp;
    }
}

// Registers of one thread's share of a B slice: the column values c and the
// base term of its 36 items, and the two window-edge rows.
struct StageRegs {
    float2 c[kQuads], base[kQuads];
    float2 e_lo, e_hi;
};

// Issue every load of this CTA's B slice of step (fwd, j).  Warp w owns
// sources 8w..8w+7; lane = (source & 7, row & 3), item q = row quad, so each
// source reads 32 contiguous bytes of a column per item.
template <bool ADJ>
__device__ __forceinline__ void stage_b_load(const SweepParams &p, StageRegs &R, int nt, int c0, int nch, bool fwd,
                                             int j) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s8 = lane & 7, r4 = lane >> 3;
    const int ny = p.ny, nx = p.nx;
    const size_t plane = (size_t)ny * nx;
    const int y0 = kRowsPerChunk * c0;
    const int nq = 4 * nch;
    const int sl = 8 * warp + s8;                   // source within the tile
    const int sb = nt * TN + sl;                    // source within the launch
    const int s = p.s0 + sb;                        // global source
    const bool sv = s < p.s_end;
    const bool from_tmp = ADJ && (fwd ? j >= 2 : j <= nx - 3);
    const int fcol = fwd ? (ADJ ? 0 : j - 1) : (ADJ ? nx - 1 : j + 1);
    const float2 *tbuf = p.tmp + (size_t)ny * p.tb * (fwd ? ((j - 1) & 1) : ((j + 1) & 1));
    const float2 *col = from_tmp ? tbuf + (size_t)ny * sb : p.u + plane * s + (size_t)ny * fcol;
    // base term: SRC column bx, u(:, j) (ADJ bwd) or zero
    const int bx = (!ADJ && fwd) ? j : ((ADJ && fwd && j >= 2) ? j - 1 : -1);
    const float2 *ubase = (ADJ && !fwd) ? p.u + plane * s + (size_t)ny * j : nullptr;
    float2 *c = R.c, *base = R.base;
#pragma unroll
    for (int q = 0; q < kQuads; ++q) {
        c[q] = f2(0.f, 0.f);
        base[q] = f2(0.f, 0.f);
        if (q < nq && sv) {
            const int yp = y0 + 4 * q + r4, y = yp + 1;
            if (yp <= p.n) c[q] = __ldcg(col + y);
            if (yp < p.n) {
                if (ubase) {
                    base[q] = __ldcg(ubase + y);
                } else if (bx >= 0) {
                    if (p.src.mode == SRC_DENSE) {
                        base[q] = p.src.dense[(size_t)y + (size_t)ny * bx + plane * s];
                    } else if (p.src.mode == SRC_POINT) {
                        base[q] = (p.src.lin[s] == y + ny * bx) ? f2(1.f, 0.f) : f2(0.f, 0.f);
                    } else if (p.src.mode == SRC_SCATTER) {
                        const int k = p.src.at[(size_t)y + (size_t)ny * bx];
                        base[q] = k >= 0 ? p.src.vals[k + (size_t)p.src.n_slots * s] : f2(0.f, 0.f);
                    }
                }
            }
        }
    }
    R.e_lo = f2(0.f, 0.f);
    R.e_hi = f2(0.f, 0.f);
    if (sv && r4 == 0) R.e_lo = __ldcg(col + y0);                       // row before the window
    const int yhi = y0 + kRowsPerChunk * nch + 1;                      // row after the window
    if (sv && r4 == 3 && yhi <= ny - 1) R.e_hi = __ldcg(col + yhi);
}

// Evaluate the stencil and write the B slice into shared memory, in the
// operand layout: element (source sl, complex row yp) of chunk (yp - y0)/16
// at chunk_off(sl, 2 * ((yp - y0) % 16)); the 8-byte stores of a warp cover
// all 32 banks.  The stencil neighbours come from the lane 8 apart in the
// same quad or the lane 24 apart in the neighbouring quad (one shuffle
// each), the two window edges from R.  ADJ modes also write the finished
// column of the previous step into u (write_u: the CTAs of M tile 0 own that).
template <bool ADJ>
__device__ __forceinline__ void stage_b_compute(const SweepParams &p, const StageRegs &R, uint8_t *sB,
                                                const float2 *w, int nt, int c0, int nch, bool fwd, int j,
                                                bool write_u) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s8 = lane & 7, r4 = lane >> 3;
    const int ny = p.ny, nx = p.nx;
    const size_t plane = (size_t)ny * nx;
    const int y0 = kRowsPerChunk * c0;
    const int nq = 4 * nch;
    const int sl = 8 * warp + s8;
    const int sb = nt * TN + sl;
    const int s = p.s0 + sb;
    const bool sv = s < p.s_end;
    const float2 *tbuf = p.tmp + (size_t)ny * p.tb * (fwd ? ((j - 1) & 1) : ((j + 1) & 1));
    const float2 *c = R.c, *base = R.base;

    float2 *ucol = nullptr;   // column of u finished by the previous step (ADJ)
    if (ADJ && write_u && sv) {
        if (fwd && j >= 2) ucol = p.u + plane * s + (size_t)ny * (j - 1);
        if (!fwd && j <= nx - 3) ucol = p.u + plane * s + (size_t)ny * (j + 1);
    }
    const int lane_m = (r4 == 0) ? lane + 24 : lane - 8;
    const int lane_p = (r4 == 3) ? lane - 24 : lane + 8;
#pragma unroll
    for (int q = 0; q < kQuads; ++q) {
        if (q < nq) {
            const float2 sup_m = (r4 == 3 && q > 0) ? c[q > 0 ? q - 1 : 0] : c[q];
            const float2 sup_p = (r4 == 0 && q + 1 < kQuads) ? c[q + 1 < kQuads ? q + 1 : q] : c[q];
            float2 m, pn;
            m.x = __shfl_sync(0xffffffffu, sup_m.x, lane_m);
            m.y = __shfl_sync(0xffffffffu, sup_m.y, lane_m);
            pn.x = __shfl_sync(0xffffffffu, sup_p.x, lane_p);
            pn.y = __shfl_sync(0xffffffffu, sup_p.y, lane_p);
            if (q == 0 && r4 == 0) m = R.e_lo;
            if (q == nq - 1 && r4 == 3) pn = R.e_hi;
            const int r = 4 * q + r4;                 // row within the window
            const int yp = y0 + r;
            float2 b = f2(0.f, 0.f);
            if (sv && yp < p.n) {
                float2 acc = cmul(w[r], c[q]);
                cfma(acc, w[kMaxRows + r], m);
                cfma(acc, w[2 * kMaxRows + r], pn);
                b = csub(base[q], acc);
                if (ucol) ucol[yp + 1] = (fwd ? b : c[q]);
            }
            *reinterpret_cast<float2 *>(sB + (q >> 2) * kBChunk + chunk_off(sl, 2 * (4 * (q & 3) + r4))) =
                f2(to_tf32(b.x), to_tf32(b.y));
        }
    }
    // border rows of the finished column (ADJ): rows 0 / ny-1 computed in the
    // forward sweep, zero in the backward sweep
    if (ADJ && ucol && r4 == 0) {
        const Coefs<float2> &co = p.co;
        const bool first = (c0 == 0);
        const bool last = (y0 <= p.n - 1) && (y0 + kRowsPerChunk * nch >= p.n);
        if (fwd) {
            const float2 *t = tbuf + (size_t)ny * sb;
            if (first) {
                float2 acc = f2(0.f, 0.f);
                cfma_conj(acc, co.ud(0, j - 2), __ldcg(t));
                cfma_conj(acc, co.ul(0, j - 2), __ldcg(t + 1));
                ucol[0] = csub(p.src.get(0, j - 1, s, ny, nx), acc);
            }
            if (last) {
                float2 acc = f2(0.f, 0.f);
                cfma_conj(acc, co.ud(ny - 1, j - 2), __ldcg(t + ny - 1));
                cfma_conj(acc, co.uu(ny - 2, j - 2), __ldcg(t + ny - 2));
                ucol[ny - 1] = csub(p.src.get(ny - 1, j - 1, s, ny, nx), acc);
            }
        } else {
            if (first) ucol[0] = f2(0.f, 0.f);
            if (last) ucol[ny - 1] = f2(0.f, 0.f);
        }
    }
}

template <bool ADJ, int KS>
__global__ void __launch_bounds__(kSweepThreads, 1) tc_sweep_kernel(SweepParams p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;
    uint8_t *sB = smem + kSmemA;
    uint64_t *full = reinterpret_cast<uint64_t *>(sB + kSmemB);
    uint64_t *done = full + kMaxPer;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *s_ok = reinterpret_cast<int *>(tmem_slot + 1);
    float2 *sW = reinterpret_cast<float2 *>(smem + kSmemA + kSmemB + kSmemBar);

    const int tid = threadIdx.x, warp = tid >> 5;
    const int mt = blockIdx.x, nt = blockIdx.y, ks = blockIdx.z;
    const int ny = p.ny, nx = p.nx;
    const size_t plane = (size_t)ny * nx;
    const int c0 = ks * p.per;
    const int nch = max(0, min(p.kc, c0 + p.per) - c0);
    const int y0 = kRowsPerChunk * c0;
    const int tile = mt + p.mt * nt;
    const unsigned group_size = (unsigned)(p.mt * KS);
    const int rank_in_group = mt + p.mt * ks;
    const int nsteps = 2 * (nx - 1);

    if (tid == 0) {
        for (int q = 0; q < kMaxPer; ++q) tc::mbar_init(&full[q], 1);
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

    int a_step = -1;          // step whose A copies are in flight (thread 0)
    if (tid == 0 && nch > 0) {
        issue_a(0);
        a_step = 0;
    }
    {
        bool f0;
        const int j0 = step_col(0, nx, f0);
        stage_weights<ADJ>(p, sW, y0, kRowsPerChunk * nch, f0, j0);
    }
    unsigned group_epoch = 0;
    bool ok = true;
#ifdef WUST_SWEEP_PROFILE
    long long prof_t = clock64();
#endif

    for (int i = 0; i < nsteps; ++i) {
        bool fwd;
        const int j = step_col(i, nx, fwd);

        if (ADJ && i == nx - 1) {
            // u(:, nx-1) = SRC_{nx-1} - U_{nx-2}^H tmp  (every row)
            const float2 *t0 = p.tmp + (size_t)ny * p.tb * ((nx - 1) & 1);
            for (int idx = rank_in_group * kSweepThreads + tid; idx < ny * TN;
                 idx += (int)group_size * kSweepThreads) {
                const int y = idx % ny, sl = idx / ny;
                const int sb = nt * TN + sl, s = p.s0 + sb;
                if (s >= p.s_end) continue;
                const float2 *t = t0 + (size_t)ny * sb;
                float2 acc = f2(0.f, 0.f);
                cfma_conj(acc, p.co.ud(y, nx - 2), __ldcg(t + y));
                if (y > 0) cfma_conj(acc, p.co.uu(y - 1, nx - 2), __ldcg(t + y - 1));
                if (y < ny - 1) cfma_conj(acc, p.co.ul(y, nx - 2), __ldcg(t + y + 1));
                p.u[plane * s + (size_t)ny * (nx - 1) + y] = csub(p.src.get(y, nx - 1, s, ny, nx), acc);
            }
            group_epoch += group_size;
            if (!counter_sync(p.group_ctr + nt, group_epoch, p.err, s_ok, p.timeout_ns, SITE_GROUP)) {
                ok = false;
                break;
            }
        }

        // ---- B operand ------------------------------------------------------
        SPROF(0);
        {
            StageRegs R;
            stage_b_load<ADJ>(p, R, nt, c0, nch, fwd, j);
#ifdef WUST_SWEEP_PROFILE
            {   // wait for every load (profiling builds only)
                float d = R.e_lo.x + R.e_hi.x;
#pragma unroll
                for (int q = 0; q < kQuads; ++q) d += R.c[q].x + R.base[q].y;
                if (d == 1.2345e30f) sW[0] = f2(d, d);
                SPROF(9);
            }
#endif
            stage_b_compute<ADJ>(p, R, sB, sW, nt, c0, nch, fwd, j, mt == 0);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        SPROF(1);

        // ---- MMAs (one thread) -----------------------------------------------
        if (tid == 0) {
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
        SPROF(7);
        if (!tc::mbar_wait(done, (uint32_t)(i & 1), p.timeout_ns)) atomicCAS(p.err, 0, SITE_MMA);
        tc::fence_after();
        SPROF(8);
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
        // weights of the next step (the stencil of this step is done)
        if (i + 1 < nsteps) {
            bool f1;
            const int j1 = step_col(i + 1, nx, f1);
            stage_weights<ADJ>(p, sW, y0, kRowsPerChunk * nch, f1, j1);
        }
        SPROF(3);
        tc::fence_before();
        if (KS > 1) {
            if (!counter_sync(p.tile_ctr + tile, (unsigned)(KS * (i + 1)), p.err, s_ok, p.timeout_ns, SITE_TILE)) {
                ok = false;
                break;
            }
        } else {
            __syncthreads();
        }
        tc::fence_after();
        SPROF(4);

        // ---- reduce one column slice over the KS partials, write the column ---
        {
            constexpr int CPR = TN / KS, QTR = CPR / 4, NV = QTR / 4;   // columns per thread, float4 per rank
            const int ir = tid & 63, qt = tid >> 6;
            const int cb = ks * CPR + qt * QTR;
            const float *pt = p.part + (size_t)tile * KS * 128 * TN;
            float4 re[KS][NV], im[KS][NV];
#pragma unroll
            for (int r = 0; r < KS; ++r)
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    re[r][v] = __ldcg(reinterpret_cast<const float4 *>(pt + ((size_t)r * 128 + ir) * TN + cb + 4 * v));
                    im[r][v] =
                        __ldcg(reinterpret_cast<const float4 *>(pt + ((size_t)r * 128 + ir + 64) * TN + cb + 4 * v));
                }
            const int gi = mt * 64 + ir;
            if (gi < p.n) {
                float2 old[NV][4];
                if (!ADJ && !fwd) {
#pragma unroll
                    for (int v = 0; v < NV; ++v)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int s = p.s0 + nt * TN + cb + 4 * v + q;
                            old[v][q] =
                                s < p.s_end ? __ldcg(p.u + plane * s + (size_t)ny * j + gi + 1) : f2(0.f, 0.f);
                        }
                }
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    float4 sr = re[0][v], si = im[0][v];
#pragma unroll
                    for (int r = 1; r < KS; ++r) {
                        sr.x += re[r][v].x; sr.y += re[r][v].y; sr.z += re[r][v].z; sr.w += re[r][v].w;
                        si.x += im[r][v].x; si.y += im[r][v].y; si.z += im[r][v].z; si.w += im[r][v].w;
                    }
                    const float vr[4] = {sr.x, sr.y, sr.z, sr.w}, vi[4] = {si.x, si.y, si.z, si.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int sb = nt * TN + cb + 4 * v + q;
                        const int s = p.s0 + sb;
                        if (s >= p.s_end) continue;
                        if (ADJ) {
                            p.tmp[(size_t)ny * p.tb * (j & 1) + (size_t)ny * sb + gi + 1] = f2(vr[q], vi[q]);
                        } else {
                            float2 *dst = p.u + plane * s + (size_t)ny * j + gi + 1;
                            *dst = fwd ? f2(vr[q], vi[q]) : f2(old[v][q].x - vr[q], old[v][q].y - vi[q]);
                        }
                    }
                }
            }
        }
        SPROF(5);
        group_epoch += group_size;
        if (!counter_sync(p.group_ctr + nt, group_epoch, p.err, s_ok, p.timeout_ns, SITE_GROUP)) {
            ok = false;
            break;
        }
        SPROF(6);
    }

    if (ADJ && ok) {
        // u(:, 0) = [0; tmp; 0] from the last backward step (j = 0)
        const float2 *t0 = p.tmp;
        for (int idx = rank_in_group * kSweepThreads + tid; idx < ny * TN; idx += (int)group_size * kSweepThreads) {
            const int y = idx % ny, sl = idx / ny;
            const int sb = nt * TN + sl, s = p.s0 + sb;
            if (s >= p.s_end) continue;
            p.u[plane * s + y] = (y == 0 || y == ny - 1) ? f2(0.f, 0.f) : __ldcg(t0 + (size_t)ny * sb + y);
        }
    }
    // copies still in flight after a failure: let them land (bounded)
    if (tid == 0 && a_step >= 0)
        for (int q = 0; q < nch; ++q) tc::mbar_wait(&full[q], (uint32_t)(a_step & 1), p.timeout_ns);
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
    static thread_local int configured_device = -1;
    int dev = 0;
    WUST_CUDA(cudaGetDevice(&dev));
    if (configured_device == dev) return;
    configure_one<false, 1>(); configure_one<false, 2>(); configure_one<false, 4>();
    configure_one<true, 1>(); configure_one<true, 2>(); configure_one<true, 4>();
    configured_device = dev;
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
                    const SrcView &src, int S, bool adjoint, float2 *u, float2 *tmp, float *part, unsigned *sync,
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
    p.tmp = tmp;
    p.part = part;
    p.err = err;
    p.ny = ny;
    p.nx = nx;
    p.n = g.n;
    p.mt = g.mt;
    p.kc = g.kc;
    p.ks = g.ks;
    p.per = g.per;
    p.tb = g.nt * TN;
    p.timeout_ns = 1000000000ull;
    for (int s0 = 0; s0 < S; s0 += g.nt * TN) {
        const int s_end = std::min(S, s0 + g.nt * TN);
        const int nt = ceil_div(s_end - s0, TN);
        WUST_CUDA(cudaMemsetAsync(sync, 0, sizeof(unsigned) * g.sync_words, st));
        if (adjoint) WUST_CUDA(cudaMemsetAsync(tmp, 0, sizeof(float2) * g.tmp_elems, st));
        p.s0 = s0;
        p.s_end = s_end;
        p.group_ctr = sync;
        p.tile_ctr = sync + g.nt;
        const dim3 grid(g.mt, nt, g.ks);
        if (adjoint) launch_sweep<true>(p, grid, st);
        else launch_sweep<false>(p, grid, st);
    }
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
