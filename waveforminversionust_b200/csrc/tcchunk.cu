// Chunked tensor-core sweeps: the column recurrence of each substitution of
// applyBlockLU (Runtime/solver/applyBlockLU.cu:433-467) cut into C chunks of
// columns that run concurrently.
//
// Step by step, every substitution is an affine recurrence on one column
// state c (ny x S):  c_i = Lambda_i c_{i-1} + g_i,  Lambda_i = -+ invT_j W_i
// (W_i the tridiagonal coupling block of the step, g_i the source or the
// already-solved column).  Cutting the nx - 1 steps of a substitution into C
// chunks of consecutive steps:
//   pass 1    every chunk runs its steps from c = 0, chunk 0 from its true
//             incoming state (it also writes its columns of u): end states z_c;
//   boundary  s_0 = z_0,  s_c = z_c + Lambda_c s_{c-1}  for c = 1 .. C-2,
//             Lambda_c the chunk's composed propagator (formed once per
//             factorization by running the chunk on the identity);
//   pass 2    chunks 1 .. C-1 rerun from s_{c-1} and write their columns.
// The serial depth drops from nx - 1 steps to about 2 (nx - 1) / C + C.
//
// A group of mt CTAs (one per 64-row complex M tile, one CTA per SM) runs a
// chunk.  Each step is one full-K complex GEMM per CTA,
//     C (64 rows x N) = A (64 rows x n) B (n x N),  N <= 256 sources,
// real-split with re/im interleaved along K exactly as in tcsweep.cu; A (the
// packed invT page) and B (the packed right-hand side) stream through a
// 4-stage bulk-copy ring into kind::tf32 MMAs of N columns, the accumulator
// sits in tensor memory.  After the MMAs each CTA writes its rows of the new
// state (re and im planes, rows fastest) and of u, meets its group on a
// counter barrier, evaluates the next step's stencil for its rows (the
// neighbour rows come from L2) into the packed B chunks, and meets the group
// again.  The A chunks of the next step are copied while that happens.
// Groups never wait on each other.  Every device wait is bounded and reports
// its site through *err.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"
#include "tcstep.cuh"

namespace wust {

constexpr int kCkThreads = 512;
constexpr int kCkWarps = kCkThreads / 32;
constexpr int kCkStages = 4;
constexpr int kCopyTid = 96;                                     // the ring's copy thread (warp 3, lane 0)
constexpr int kCkMaxN = 256;                                     // sources per launch (MMA N)
constexpr int kCkRowsPerChunk = 16;                              // complex rows per K chunk (TF32)
constexpr int kCkRowsPerChunk16 = 32;                            // complex rows per K chunk (BF16)
constexpr int kCkMaxChunks = 148;
constexpr size_t kCkBSlot = (size_t)kCkMaxN * tc::kChunkBytes;   // 32 KB
constexpr size_t kCkSmemRing = (size_t)kCkStages * (tc::kAChunk + kCkBSlot);
constexpr size_t kCkSmemHalo = 2 * kCkMaxN * sizeof(float2);
constexpr size_t kCkSmemW = 3 * 64 * sizeof(float2);
constexpr size_t kCkSmem = kCkSmemRing + kCkSmemHalo + kCkSmemW + 256;
static_assert((size_t)kCkStages * kCkBSlot >= (size_t)kCkMaxN * 64 * sizeof(float2), "B stages hold the staged state");
static_assert(kCkSmem <= 232448, "shared memory of one CTA");

__host__ __device__ constexpr int ceil_div8(int x) { return (x + 7) / 8 * 8; }

using tc::chunk_off;
using tc::to_tf32;

// Launch kinds and the kind of work of one group.
enum CkPass { CK_FIRST = 0, CK_SECOND = 1, CK_PROP = 2, CK_BOUNDARY = 3 };
enum CkKind { K_EXACT = 0, K_LOCAL = 1, K_PROP = 2, K_BOUND = 3 };
// Where the incoming state of a chunk comes from.
enum CkIn { IN_ZERO = 0, IN_PLANES = 1, IN_UCOL = 2, IN_IDENT = 3 };
// What produce makes of the staged state.
enum CkProduce { P_STENCIL = 0, P_IDENT = 1, P_TURN = 2 };

size_t tc_chunk_state_floats(int ny) { return (size_t)2 * kCkMaxN * ny; }

TcChunkGeom tc_chunk_geom(int ny, int nx, int max_ctas, int chunks) {
    TcChunkGeom g{};
    g.n = ny - 2;
    g.mt = ceil_div(g.n, 64);
    g.kc = ceil_div(g.n, kCkRowsPerChunk);
    g.kc16 = ceil_div(g.n, kCkRowsPerChunk16);
    const int steps = nx - 1;
    if (steps < 1 || g.n < 1) fail(WUST_ERR_INVALID_INPUT, "chunked sweep needs Nx >= 2 and Ny >= 3");
    if (g.mt > max_ctas)
        fail(WUST_ERR_INVALID_INPUT, "chunked sweep needs %d co-resident CTAs (device holds %d)", g.mt, max_ctas);
    // about sqrt(2 steps) chunks balance the two passes against the boundary
    // chain; every chunk keeps at least 2 steps (the mirrored H^H backward
    // cuts then leave no chunk empty)
    int C = chunks > 0 ? chunks : (int)std::lround(std::sqrt(2.0 * steps));
    C = std::max(1, std::min({C, max_ctas / g.mt, steps / 2, kCkMaxChunks}));
    g.C = C;
    g.page_bytes = (size_t)g.mt * g.kc * tc::kAChunk;
    g.page_bytes16 = (size_t)g.mt * g.kc16 * tc::kAChunk;
    g.lpack_bytes = C >= 3 ? (size_t)4 * C * g.page_bytes : 0;
    g.lpack16_bytes = C >= 3 ? (size_t)4 * C * g.page_bytes16 : 0;
    g.b_bytes = (size_t)C * g.kc * kCkBSlot;
    g.state_bytes = (size_t)C * tc_chunk_state_floats(ny) * sizeof(float);
    g.edge_bytes = (size_t)C * g.mt * 2 * kCkMaxN * sizeof(float2);
    g.sync_words = C;
    return g;
}

// Optional phase timer (SM cycles of CTA 0, summed over steps, per launch
// kind), built only into profiling builds of the library.
#ifdef WUST_CHUNK_PROFILE
__device__ unsigned long long g_chunk_prof[4][8];
#define CPROF(k)                                                                                  \
    do {                                                                                          \
        if (blockIdx.x == 0 && threadIdx.x == 0) {                                                \
            const long long t_ = clock64();                                                       \
            g_chunk_prof[p.pass][k] += (unsigned long long)(t_ - prof_t);                         \
            prof_t = t_;                                                                          \
        }                                                                                         \
    } while (0)
extern "C" int wust_chunk_profile_read(unsigned long long *out) {
    return (int)cudaMemcpyFromSymbol(out, g_chunk_prof, sizeof(g_chunk_prof));
}
extern "C" int wust_chunk_profile_reset() {
    unsigned long long z[32] = {};
    return (int)cudaMemcpyToSymbol(g_chunk_prof, z, sizeof(z));
}
#else
#define CPROF(k) ((void)0)
#endif

struct ChunkParams {
    const uint8_t *apack;     // packed pages of the solve (invT or invT^H): [page][mt][kc] chunks
    const uint8_t *lpack;     // boundary launches: packed -Lambda_c pages, [chunk][mt][kc]
    size_t page_bytes;
    Coefs<float2> co;
    SrcView src;
    float2 *u;                // [ny, nx, S] (global source index)
    uint8_t *bglob;           // [group][kc] chunks of N x 128 bytes
    float *zst;               // [chunk] states: re plane [kCkMaxN][ny], im plane [kCkMaxN][ny]
    float *sb;                // [chunk] boundary states s_c (c >= 1), same layout
    float2 *edges;            // [group][mt][2][kCkMaxN]: first and last own row of each CTA's state
    unsigned *group_ctr;      // [group]
    int *err;
    int ny, nx, n, mt, kc, N;
    int s0, s_end;            // global sources [s0, s_end) of this launch
    int half;                 // 0: forward substitution (steps 0 .. nx-2), 1: backward
    int pass, C;
    int bounds[kCkMaxChunks + 1];   // first step (within the half) of each chunk
    unsigned long long timeout_ns;
};

// BF: BF16 operands (kind::f16 MMAs, 32 complex rows per K chunk) for the
// correction solves of the refinement; TF32 otherwise.
template <bool ADJ, bool BF>
__global__ void __launch_bounds__(kCkThreads, 1) tc_chunk_kernel(const __grid_constant__ ChunkParams p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;                                          // [stage] 16 KB
    uint8_t *sB = smem + (size_t)kCkStages * tc::kAChunk;        // [stage] 32 KB
    // Between a step's MMAs and the next step's B copies the B stages hold the
    // state of this CTA's 64 rows: cs[s * 64 + row] (complex).
    float2 *cs = reinterpret_cast<float2 *>(sB);
    float2 *halo = reinterpret_cast<float2 *>(smem + kCkSmemRing);  // [2][kCkMaxN]: rows 64t-1 and 64t+64
    float2 *wts = halo + 2 * kCkMaxN;                                // [3][64] stencil weights of own rows
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kCkSmemRing + kCkSmemHalo + kCkSmemW);
    uint64_t *empty = full + kCkStages;
    uint64_t *done = empty + kCkStages;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    int *s_ok = reinterpret_cast<int *>(tmem_slot + 1);
    uint32_t *s_ring = reinterpret_cast<uint32_t *>(s_ok + 1);   // [0] A, [1] B copies issued, [2] full waits done

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = blockIdx.x / p.mt, t = blockIdx.x % p.mt;
    const int ny = p.ny, nx = p.nx, n = p.n, kc = p.kc, N = p.N;
    const size_t plane = (size_t)ny * nx;
    const size_t sfl = (size_t)2 * kCkMaxN * ny;                 // floats per state
    const size_t bbytes = (size_t)N * tc::kChunkBytes;
    uint8_t *bg = p.bglob + (size_t)g * kc * bbytes;
    unsigned *ctr = p.group_ctr + g;
    const int row0 = 64 * t;                                     // first complex interior row of this CTA
    // the boundary chain splits the launch's sources over its groups: group g
    // takes sources [so, so + N) of the launch (every other pass: so = 0)
    const int so = p.pass == CK_BOUNDARY ? g * N : 0;

    // this group's chunk, kind and steps
    int chunk, kind, t0, nsteps;
    if (p.pass == CK_BOUNDARY) {
        chunk = 0; kind = K_BOUND; t0 = 1; nsteps = p.C - 2;
    } else {
        chunk = (p.pass == CK_FIRST ? 0 : 1) + g;
        kind = p.pass == CK_PROP ? K_PROP : (p.pass == CK_SECOND || chunk == 0) ? K_EXACT : K_LOCAL;
        t0 = p.bounds[chunk];
        nsteps = p.bounds[chunk + 1] - t0;
    }
    // state planes of the boundary sequence: s_0 = z_0 (the end state of
    // chunk 0), s_c in sb.  H^H solves carry B states between chunks (the
    // first B of the next chunk), kept in sb from the start.
    auto bstate = [&](int c) -> float * { return (c == 0 && !ADJ) ? p.zst : p.sb + (size_t)c * sfl; };

    auto col_of = [&](int k, bool &fwd) -> int {
        if (kind == K_BOUND) { fwd = false; return 0; }
        return step_col(p.half * (nx - 1) + t0 + k, nx, fwd);
    };
    auto apage = [&](int k) -> const uint8_t * {
        if (kind == K_BOUND) return p.lpack + (size_t)(t0 + k) * p.page_bytes;
        bool f;
        const int j = col_of(k, f);
        return p.apack + (size_t)((ADJ && f) ? j - 1 : j) * p.page_bytes;
    };
    // incoming state value at grid row y (0 .. ny-1; 0 outside), local source s
    // (0 for the padding sources beyond s_end: the caller's fields hold only
    // s_end sources)
    auto cval = [&](int in, const float *pl, int y, int s) -> float2 {
        if (y < 0 || y >= ny || p.s0 + so + s >= p.s_end) return f2(0.f, 0.f);
        if (in == IN_PLANES)
            return f2(__ldcg(pl + (size_t)(so + s) * ny + y), __ldcg(pl + (size_t)(kCkMaxN + so + s) * ny + y));
        if (in == IN_UCOL) return __ldcg(p.u + plane * (p.s0 + so + s) + (size_t)ny * (nx - 1) + y);
        if (in == IN_IDENT) return f2((y >= 1 && y <= n && y - 1 == p.s0 + so + s) ? 1.f : 0.f, 0.f);
        return f2(0.f, 0.f);
    };
    // staged state at complex interior row yp (row0 - 1 .. row0 + 64)
    auto cs_get = [&](int yp, int s) -> float2 {
        const int l = yp - row0;
        if (l >= 0 && l < 64) return cs[s * 64 + l];
        if (l == -1) return halo[s];
        if (l == 64) return halo[kCkMaxN + s];
        return f2(0.f, 0.f);
    };
    // own rows and halo rows of an incoming state -> shared memory
    auto stage_in = [&](int in, const float *pl) {
        __syncthreads();
        for (int it0 = tid; it0 < 64 * N; it0 += 4 * kCkThreads) {
            float2 v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int it = it0 + q * kCkThreads;
                v[q] = it < 64 * N ? cval(in, pl, row0 + (it & 63) + 1, it >> 6) : f2(0.f, 0.f);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int it = it0 + q * kCkThreads;
                if (it < 64 * N) cs[(it >> 6) * 64 + (it & 63)] = v[q];
            }
        }
        for (int it = tid; it < 2 * N; it += kCkThreads) {
            const int e = it / N, s = it % N;
            halo[e * kCkMaxN + s] = cval(in, pl, e == 0 ? row0 : row0 + 65, s);
        }
    };
    // halo rows: the last row of the CTA above and the first row of the CTA
    // below (zero at the grid's edges)
    float2 *my_edges = p.edges + ((size_t)g * p.mt + t) * 2 * kCkMaxN;
    auto stage_halo = [&]() {
        __syncthreads();
        for (int it = tid; it < 2 * N; it += kCkThreads) {
            const int e = it / N, s = it % N;
            float2 v = f2(0.f, 0.f);
            if (e == 0 && t > 0) v = __ldcg(my_edges - 2 * kCkMaxN + kCkMaxN + s);
            if (e == 1 && t < p.mt - 1) v = __ldcg(my_edges + 2 * kCkMaxN + s);
            halo[e * kCkMaxN + s] = v;
        }
    };

    // stencil weights of own row row0 + r for step (fwd1, j1) -> wts
    auto fill_weights = [&](int r, bool ident, bool fwd1, int j1) {
        const int yp = row0 + r, y = yp + 1;
        float2 wc = f2(0.f, 0.f), wm = wc, wp = wc;
        if (yp < n) {
            if (ident) wc = f2(-1.f, 0.f);
            else step_weights<ADJ>(p.co, fwd1, j1, y, wc, wm, wp);
        }
        wts[r] = wc;
        wts[64 + r] = wm;
        wts[128 + r] = wp;
    };

    // B of step k for this CTA's rows from the staged state:
    //   P_STENCIL  B = base - stencil(state), into the packed chunks, or as
    //              FP32 planes into `out` (a chunk's outgoing B state);
    //   P_IDENT    B = state (an incoming B state, or a boundary step);
    //   P_TURN     the turn of the H^H solve: u(:, nx-1) = SRC_{nx-1} -
    //              U_{nx-2}^H c on every row, no B.
    // Exact H^H forward steps also write B into u(:, j-1) (stencil mode:
    // with its border rows).  Warp w handles sources w, w+8, ...; lane r the
    // rows 2r, 2r+1 (neighbour rows by shuffles).
    auto produce = [&](int k, int mode, float *out, bool wts_ready) {
        bool fwd1 = true;
        int j1 = nx;
        if (mode != P_TURN) j1 = col_of(k, fwd1);
        const bool pack = mode != P_TURN && !out;
        const bool ident = mode == P_IDENT;
        const bool wu = kind == K_EXACT && ADJ && fwd1 && !out;
        const bool has_base = (kind == K_EXACT || kind == K_LOCAL) && !ident;
        __syncthreads();
        if (!wts_ready && tid < 64) fill_weights(tid, ident, fwd1, j1);
        __syncthreads();
        if (wu && !ident) {
            // border rows 0 and ny-1 of u(:, j1-1) (no B entry)
            for (int it = tid; it < 2 * N; it += kCkThreads) {
                const int e = it / N, s = it % N, gs = p.s0 + so + s;
                if ((e == 0 && t != 0) || (e == 1 && t != p.mt - 1) || gs >= p.s_end) continue;
                const int y = e == 0 ? 0 : ny - 1, yp = y - 1;
                float2 wc, wm, wp;
                step_weights<ADJ>(p.co, fwd1, j1, y, wc, wm, wp);
                float2 acc = cmul(wc, cs_get(yp, s));
                cfma(acc, wm, cs_get(yp - 1, s));
                cfma(acc, wp, cs_get(yp + 1, s));
                p.u[plane * gs + (size_t)ny * (j1 - 1) + y] =
                    csub(step_base<ADJ>(p.src, p.u, ny, nx, fwd1, j1, y, gs), acc);
            }
            __syncthreads();                               // the packing below overwrites the staged state
        }
        const int yp0 = row0 + 2 * lane, y0 = yp0 + 1;
        const bool v0 = yp0 < n, v1 = yp0 + 1 < n;
        const float2 wc0 = wts[2 * lane], wm0 = wts[64 + 2 * lane], wp0 = wts[128 + 2 * lane];
        const float2 wc1 = wts[2 * lane + 1], wm1 = wts[64 + 2 * lane + 1], wp1 = wts[128 + 2 * lane + 1];
        const int q_own = min(4, kc - row0 / kCkRowsPerChunk);    // packed chunks of this CTA's rows
        // Warp: groups of 8 consecutive sources.  The packed chunks take the
        // 8 sources of one row pair as one 128-byte row, so the warp writes
        // its results over its own (already consumed) 4 KB of staged state in
        // that order (XOR-swizzled against bank conflicts) and copies them out
        // as contiguous 512-byte stores.
        for (int grp = warp; grp < N / 8; grp += kCkWarps) {
            float4 bq[8];
#pragma unroll
            for (int h4 = 0; h4 < 2; ++h4) {
                float2 base[4][2];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int gs = p.s0 + so + 8 * grp + 4 * h4 + q;
                    base[q][0] = base[q][1] = f2(0.f, 0.f);
                    if (has_base && gs < p.s_end) {
                        if (v0) base[q][0] = step_base<ADJ>(p.src, p.u, ny, nx, fwd1, j1, y0, gs);
                        if (v1) base[q][1] = step_base<ADJ>(p.src, p.u, ny, nx, fwd1, j1, y0 + 1, gs);
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int s = 8 * grp + 4 * h4 + q, gs = p.s0 + so + s;
                    const float4 cv = *reinterpret_cast<const float4 *>(cs + s * 64 + 2 * lane);
                    const float2 c0 = f2(cv.x, cv.y), c1 = f2(cv.z, cv.w);
                    float2 cm = f2(__shfl_up_sync(0xffffffffu, c1.x, 1), __shfl_up_sync(0xffffffffu, c1.y, 1));
                    float2 cp = f2(__shfl_down_sync(0xffffffffu, c0.x, 1), __shfl_down_sync(0xffffffffu, c0.y, 1));
                    if (lane == 0) cm = halo[s];
                    if (lane == 31) cp = halo[kCkMaxN + s];
                    float2 b0 = f2(0.f, 0.f), b1 = b0;
                    if (gs < p.s_end) {
                        if (v0) {
                            float2 acc = cmul(wc0, c0);
                            cfma(acc, wm0, cm);
                            cfma(acc, wp0, c1);
                            b0 = csub(base[q][0], acc);
                            if (wu) p.u[plane * gs + (size_t)ny * (j1 - 1) + y0] = b0;
                        }
                        if (v1) {
                            float2 acc = cmul(wc1, c1);
                            cfma(acc, wm1, c0);
                            cfma(acc, wp1, cp);
                            b1 = csub(base[q][1], acc);
                            if (wu) p.u[plane * gs + (size_t)ny * (j1 - 1) + y0 + 1] = b1;
                        }
                        if (out) {
                            float *re = out + (size_t)(so + s) * ny, *im = out + (size_t)(kCkMaxN + so + s) * ny;
                            if (v0) { __stcg(re + y0, b0.x); __stcg(im + y0, b0.y); }
                            if (v1) { __stcg(re + y0 + 1, b1.x); __stcg(im + y0 + 1, b1.y); }
                        }
                    }
                    if (BF) {
                        // rows yp0, yp0 + 1 of chunk yp0 / 32: four bf16 values (8 bytes)
                        if (pack && yp0 < kCkRowsPerChunk16 * kc) {
                            const int Q = yp0 / kCkRowsPerChunk16, ke = 2 * (yp0 % kCkRowsPerChunk16);
                            const uint32_t lo = (uint32_t)tc::to_bf16_bits(b0.x) | ((uint32_t)tc::to_bf16_bits(b0.y) << 16);
                            const uint32_t hi = (uint32_t)tc::to_bf16_bits(b1.x) | ((uint32_t)tc::to_bf16_bits(b1.y) << 16);
                            *reinterpret_cast<uint2 *>(bg + (size_t)Q * bbytes + tc::chunk_off16(s, ke)) = make_uint2(lo, hi);
                        }
                    } else {
                        bq[4 * h4 + q] = make_float4(to_tf32(b0.x), to_tf32(b0.y), to_tf32(b1.x), to_tf32(b1.y));
                    }
                }
            }
            if (pack && !BF) {
                float4 *reg = reinterpret_cast<float4 *>(cs + (size_t)grp * 8 * 64);   // 256 float4
                __syncwarp();
#pragma unroll
                for (int q = 0; q < 8; ++q) reg[lane * 8 + (q ^ (lane & 7))] = bq[q];
                __syncwarp();
                for (int Q = 0; Q < q_own; ++Q) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int idx = lane + 32 * h, kg = idx >> 3;
                        const float4 v = reg[(Q * 8 + kg) * 8 + ((idx & 7) ^ kg)];
                        *reinterpret_cast<float4 *>(bg + (size_t)(row0 / kCkRowsPerChunk + Q) * bbytes +
                                                    (size_t)grp * 1024 + (size_t)idx * 16) = v;
                    }
                }
            }
        }
    };

    if (tid == 0) {
        for (int q = 0; q < kCkStages; ++q) {
            tc::mbar_init(&full[q], 2);       // A copy + B copy
            tc::mbar_init(&empty[q], 1);      // MMAs of the stage retired
        }
        tc::mbar_init(done, 1);
        tc::mbar_fence_init();
    }
    const uint32_t tcols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;
    if (warp == 0) tc::tmem_alloc(tmem_slot, tcols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;

    // Accumulator (TMEM) -> staged state, own rows (rows beyond the grid 0).
    auto drain_tmem = [&]() {
        const int l = 32 * (warp & 3) + lane;
        const int part = l >> 6;                       // TMEM lanes 0-63: real parts, 64-127: imaginary
        const int row = l & 63;
        const bool row_ok = row0 + row < n;
        const int hc = ceil_div8(N / (kCkWarps / 4)), c0 = (warp >> 2) * hc;
        float *csf = reinterpret_cast<float *>(cs);
        const uint32_t tl = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
        int cb = 0;
        for (; cb + 32 <= hc && c0 + cb + 32 <= N; cb += 32) {
            float v[32];
            tc::tmem_ld32(tl + (uint32_t)(c0 + cb), v);
#pragma unroll
            for (int q = 0; q < 32; ++q) csf[((size_t)(c0 + cb + q) * 64 + row) * 2 + part] = row_ok ? v[q] : 0.f;
        }
        for (; cb < hc && c0 + cb < N; cb += 8) {
            float v[8];
            tc::tmem_ld8(tl + (uint32_t)(c0 + cb), v);
#pragma unroll
            for (int q = 0; q < 8; ++q) csf[((size_t)(c0 + cb + q) * 64 + row) * 2 + part] = row_ok ? v[q] : 0.f;
        }
    };
    // The state after step k: subtracting steps take old - value; write the
    // finished columns of u, and the state's edge rows (every row on the
    // chunk's last step) to the planes curp.
    auto finish = [&](int k, float *curp, bool last) {
        bool fwd = false;
        const int j = col_of(k, fwd);
        const bool sub = kind == K_BOUND || (!ADJ && !fwd);
        const bool wu = kind == K_EXACT && (!ADJ || !fwd);
        const float *oldp = kind == K_BOUND ? (ADJ ? p.sb : p.zst) + (size_t)(t0 + k) * sfl : nullptr;
        const bool old_u = sub && kind != K_BOUND && kind != K_PROP;
        const int yp0 = row0 + 2 * lane, y0 = yp0 + 1;
        const bool v0 = yp0 < n, v1 = yp0 + 1 < n;
        __syncthreads();
        for (int sb0 = warp; sb0 < N; sb0 += 4 * kCkWarps) {
            float2 o[4][2];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int s = sb0 + kCkWarps * q, gs = p.s0 + so + s;
                o[q][0] = o[q][1] = f2(0.f, 0.f);
                if (s < N && gs < p.s_end) {
                    if (old_u) {
                        const float2 *uc = p.u + plane * gs + (size_t)ny * j;
                        if (v0) o[q][0] = __ldcs(uc + y0);
                        if (v1) o[q][1] = __ldcs(uc + y0 + 1);
                    } else if (kind == K_BOUND) {
                        const float *ore = oldp + (size_t)(so + s) * ny, *oim = oldp + (size_t)(kCkMaxN + so + s) * ny;
                        if (v0) o[q][0] = f2(__ldcg(ore + y0), __ldcg(oim + y0));
                        if (v1) o[q][1] = f2(__ldcg(ore + y0 + 1), __ldcg(oim + y0 + 1));
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int s = sb0 + kCkWarps * q, gs = p.s0 + so + s;
                if (s >= N) break;                                   // warp-uniform
                float4 *cp4 = reinterpret_cast<float4 *>(cs + s * 64 + 2 * lane);
                float4 cv = *cp4;
                if (sub) {
                    cv = make_float4(o[q][0].x - cv.x, o[q][0].y - cv.y, o[q][1].x - cv.z, o[q][1].y - cv.w);
                    if (!v0) { cv.x = 0.f; cv.y = 0.f; }
                    if (!v1) { cv.z = 0.f; cv.w = 0.f; }
                    *cp4 = cv;
                }
                if (gs >= p.s_end) continue;
                if (wu) {                 // u streams through L2 (evict first), as the old column it replaces
                    float2 *uc = p.u + plane * gs + (size_t)ny * j;
                    if (v0) __stcs(uc + y0, f2(cv.x, cv.y));
                    if (v1) __stcs(uc + y0 + 1, f2(cv.z, cv.w));
                }
                if (lane == 0) __stcg(my_edges + s, f2(cv.x, cv.y));
                if (lane == 31 && v1) __stcg(my_edges + kCkMaxN + s, f2(cv.z, cv.w));
                if (last) {
                    float *re = curp + (size_t)(so + s) * ny, *im = curp + (size_t)(kCkMaxN + so + s) * ny;
                    if (v0) { __stcg(re + y0, cv.x); __stcg(im + y0, cv.y); }
                    if (v1) { __stcg(re + y0 + 1, cv.z); __stcg(im + y0 + 1, cv.w); }
                }
            }
        }
        if (kind == K_EXACT && ADJ && !fwd && t == 0) {
            // H^H backward: border rows of u(:, j) are zero
            for (int s = tid; s < N; s += kCkThreads) {
                const int gs = p.s0 + so + s;
                if (gs >= p.s_end) continue;
                p.u[plane * gs + (size_t)ny * j] = f2(0.f, 0.f);
                p.u[plane * gs + (size_t)ny * j + ny - 1] = f2(0.f, 0.f);
            }
        }
    };

    // Warps 1-7, while the MMAs run: pull into L2 the field columns that the
    // coming finish (old column of a subtracting step) and produce (base of
    // the next step) will read, own rows of every source.
    auto prefetch_cols = [&](int k) {
        const float2 *cols[2] = {nullptr, nullptr};
        bool fwd;
        const int j = col_of(k, fwd);
        if ((kind == K_EXACT || kind == K_LOCAL) && !ADJ && !fwd) cols[0] = p.u + (size_t)ny * j;
        if ((kind == K_EXACT || kind == K_LOCAL) && k + 1 < nsteps) {
            bool f1;
            const int j1 = col_of(k + 1, f1);
            if (ADJ && !f1) cols[1] = p.u + (size_t)ny * j1;
            else if (p.src.mode == SRC_DENSE && (!ADJ || j1 >= 2) && f1)
                cols[1] = p.src.dense + (size_t)ny * (ADJ ? j1 - 1 : j1);
        }
        const int y_first = row0 + 1, y_last = min(row0 + 64, n);
        for (int c = 0; c < 2; ++c) {
            if (!cols[c]) continue;
            for (int it = tid - 32; it < N * 5; it += kCkThreads - 32) {
                const int s = it / 5, q = it % 5, gs = p.s0 + so + s;
                if (gs >= p.s_end) continue;
                const char *first = reinterpret_cast<const char *>(cols[c] + plane * gs + y_first);
                const char *last = reinterpret_cast<const char *>(cols[c] + plane * gs + y_last);
                const uintptr_t line = ((uintptr_t)first >> 7) + (uintptr_t)q;
                if (line > ((uintptr_t)last >> 7)) continue;
                const char *a = q == 0 ? first : reinterpret_cast<const char *>(line << 7);
                tc::prefetch_l2(a);
            }
        }
    };

    // ---- bulk-copy ring; chunk ci = k * kc + q of step k --------------------
    // Two threads drive it: the copy thread (kCopyTid) refills each stage as
    // soon as the MMAs that read it have completed, and thread 0 issues each
    // chunk's MMAs as soon as its copies have landed, so neither waits on
    // the other's latency.  A chunk's stage is slot ci % kCkStages, used for
    // the (ci / kCkStages)-th time.
    uint32_t a_next = 0, b_next = 0, full_waited = 0;
    // the page stream passes through L2 once; the packed B is read by every
    // CTA of the group and should stay
    const uint64_t a_policy = tc::policy_evict_first();
    const uint64_t b_policy = tc::policy_evict_last();
    // copy thread: the A chunk a_next into its stage, once the MMAs of the
    // chunk that used the stage before have completed
    auto issue_a = [&]() -> bool {
        const uint32_t c = a_next;
        const int ks = (int)(c / kc), q = (int)(c % kc), slot = (int)(c % kCkStages);
        if (c >= (uint32_t)kCkStages && !tc::mbar_wait(&empty[slot], ((c / kCkStages) - 1) & 1u, p.timeout_ns))
            return false;
        tc::mbar_expect_tx(&full[slot], tc::kAChunk);
        tc::bulk_g2s_hint(sA + (size_t)slot * tc::kAChunk, apage(ks) + ((size_t)t * kc + q) * tc::kAChunk, tc::kAChunk,
                          &full[slot], a_policy);
        ++a_next;
        return true;
    };
    // copy thread, step k: every B chunk of the step (each after its A
    // chunk), then the next step's first A chunks as the stages free up
    auto copies = [&](int k) {
        bool good = true;
        const uint32_t end = (uint32_t)(k + 1) * (uint32_t)kc;
        while (good && b_next < end) {
            if (a_next <= b_next && !(good = issue_a())) break;
            const int q = (int)(b_next % kc), slot = (int)(b_next % kCkStages);
            tc::mbar_expect_tx(&full[slot], (uint32_t)bbytes);
            tc::bulk_g2s_hint(sB + (size_t)slot * kCkBSlot, bg + (size_t)q * bbytes, (uint32_t)bbytes, &full[slot],
                              b_policy);
            ++b_next;
        }
        const uint32_t a_end = min((uint32_t)min(k + 2, nsteps) * (uint32_t)kc, end + (uint32_t)kCkStages);
        while (good && a_next < a_end) good = issue_a();
        if (!good) atomicCAS(p.err, 0, SITE_COPY);
    };

    unsigned epoch = 0;
    bool ok = nsteps > 0;
    if (ok) {
        if (tid == kCopyTid)                                // the first A chunks of step 0
            while (a_next < (uint32_t)min(kCkStages, kc) && issue_a()) {
            }
        int in0 = IN_ZERO, mode0 = P_STENCIL;
        const float *pl0 = nullptr;
        if (kind == K_EXACT && chunk > 0) {
            in0 = IN_PLANES;
            pl0 = bstate(chunk - 1);
            if (ADJ) mode0 = P_IDENT;                      // the incoming state is this chunk's first B
        } else if (kind == K_EXACT && p.half == 1) {
            in0 = IN_UCOL;
        } else if (kind == K_PROP) {
            in0 = IN_IDENT;
        } else if (kind == K_BOUND) {
            in0 = IN_PLANES;
            pl0 = bstate(0);
            mode0 = P_IDENT;
        } else if (kind == K_LOCAL && ADJ) {
            mode0 = P_IDENT;                               // first B = 0
        }
        stage_in(in0, pl0);
        produce(0, mode0, nullptr, false);
        epoch += (unsigned)p.mt;
        ok = counter_sync(ctr, epoch, p.err, s_ok, p.timeout_ns, SITE_B);
    }
    float *cur = kind == K_BOUND ? nullptr : p.zst + (size_t)chunk * sfl;
    constexpr int kMmaPerChunk = tc::kChunkBytes / 32;
    const uint32_t idesc = tc::instr_desc<!BF>(tc::kTileRows, N);

#ifdef WUST_CHUNK_PROFILE
    long long prof_t = clock64();
    if (blockIdx.x == 0 && tid == 0) g_chunk_prof[p.pass][7] += (unsigned long long)nsteps;
#endif
    for (int k = 0; k < nsteps && ok; ++k) {
        CPROF(6);
        if (tid == kCopyTid) copies(k);
        if (tid == 0) {
            bool good = true;
            for (int q = 0; q < kc; ++q) {
                const uint32_t ci = (uint32_t)k * kc + q;
                const int slot = (int)(ci % kCkStages);
                if (!tc::mbar_wait(&full[slot], (ci / kCkStages) & 1u, p.timeout_ns)) { good = false; break; }
                full_waited = ci + 1;
                tc::fence_after();
#pragma unroll
                for (int kk = 0; kk < kMmaPerChunk; ++kk)
                    tc::mma<!BF>(tmem, tc::smem_desc(sA + (size_t)slot * tc::kAChunk + kk * 256),
                                  tc::smem_desc(sB + (size_t)slot * kCkBSlot + kk * 256), idesc,
                                  (q > 0 || kk > 0) ? 1u : 0u);
                tc::commit(&empty[slot]);
            }
            tc::commit(done);
            if (!good) atomicCAS(p.err, 0, SITE_COPY);
        }
        if (warp >= 1 && tid != kCopyTid) prefetch_cols(k);
        if (warp == 1 || warp == 2) {
            const bool next_b = k + 1 < nsteps || (ADJ && p.pass == CK_FIRST && chunk + 1 < p.C);
            if (next_b) {
                bool f1 = false;
                const int j1 = col_of(k + 1, f1);
                fill_weights(tid - 32, kind == K_BOUND, f1, j1);
            }
        }
        CPROF(0);
        if (!tc::mbar_wait(done, (uint32_t)(k & 1), p.timeout_ns)) atomicCAS(p.err, 0, SITE_MMA);
        tc::fence_after();
        if (tid == 0) *s_ok = (*(volatile int *)p.err == 0);
        __syncthreads();
        if (!*s_ok) {
            ok = false;
            break;
        }
        float *curp = kind == K_BOUND ? bstate(t0 + k) : cur;
        CPROF(1);
        drain_tmem();
        tc::fence_before();
        finish(k, curp, kind == K_BOUND || k + 1 == nsteps);
        CPROF(2);
        epoch += (unsigned)p.mt;
        if (!counter_sync(ctr, epoch, p.err, s_ok, p.timeout_ns, SITE_GROUP)) {
            ok = false;
            break;
        }
        tc::fence_after();
        CPROF(3);
        if (k + 1 < nsteps) {
            stage_halo();
            CPROF(5);
            produce(k + 1, kind == K_BOUND ? P_IDENT : P_STENCIL, nullptr, true);
            CPROF(4);
            epoch += (unsigned)p.mt;
            if (!counter_sync(ctr, epoch, p.err, s_ok, p.timeout_ns, SITE_B)) {
                ok = false;
                break;
            }
        } else if (kind == K_EXACT && ADJ && p.half == 0 && t0 + k == nx - 2) {
            stage_halo();
            produce(k, P_TURN, nullptr, false);
        } else if (ADJ && p.pass == CK_FIRST && chunk + 1 < p.C) {
            // outgoing B state of the chunk: the first B of the next chunk
            stage_halo();
            produce(k + 1, P_STENCIL, bstate(chunk), true);
        }
    }

    // copies issued but never waited for (a failure): stand in for the B
    // copies that will not come, then let them land (bounded)
    if (tid == kCopyTid) {
        s_ring[0] = a_next;
        s_ring[1] = b_next;
    }
    if (tid == 0) s_ring[2] = full_waited;
    __syncthreads();
    if (tid == 0) {
        for (uint32_t ci = s_ring[2]; ci < s_ring[0]; ++ci) {
            const int slot = (int)(ci % kCkStages);
            if (ci >= s_ring[1]) tc::mbar_arrive(&full[slot]);
            tc::mbar_wait(&full[slot], (ci / kCkStages) & 1u, p.timeout_ns);
        }
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, tcols);
}

// -Lambda_c (columns [s0, s_end) of the propagators of chunks 1 .. C-2, in
// the state planes) -> packed [Ar -Ai; Ai Ar] A pages of the boundary steps
// (page c), and the rows [s0, s_end) of -Lambda_c^H -> the pages C-1-c of the
// H^H boundary steps.  BF: BF16 pages (32 complex columns per K chunk).
template <bool BF>
__global__ void pack_lambda_kernel(const float *zst, size_t sfl, int ny, int n, int mt, int kc, size_t page_bytes,
                                   int s0, int s_end, int C, uint8_t *lpack, uint8_t *lpack_h) {
    constexpr int RPC = BF ? kCkRowsPerChunk16 : kCkRowsPerChunk;   // complex columns per chunk
    constexpr int CPU = RPC / 8;                                      // complex columns per 16-byte unit
    const int i_s = threadIdx.x;                     // stacked row 0..127
    const int Q = blockIdx.x;                        // K chunk
    const int m = blockIdx.y;                        // M tile
    const int c = 1 + blockIdx.z;                    // chunk
    const int i = m * 64 + (i_s & 63);
    const bool imrow = i_s >= 64;
    const float *pl = zst + (size_t)c * sfl;
    auto store = [&](uint8_t *dst, int u, const float (&v)[2 * CPU]) {
        if (BF) {
            uint32_t w[CPU];
#pragma unroll
            for (int h = 0; h < CPU; ++h)
                w[h] = (uint32_t)tc::to_bf16_bits(v[2 * h]) | ((uint32_t)tc::to_bf16_bits(v[2 * h + 1]) << 16);
            *reinterpret_cast<uint4 *>(dst + tc::chunk_off16(i_s, 8 * u)) = make_uint4(w[0], w[1], w[2 % CPU], w[3 % CPU]);
        } else {
            *reinterpret_cast<float4 *>(dst + chunk_off(i_s, 4 * u)) =
                make_float4(to_tf32(v[0]), to_tf32(v[1]), to_tf32(v[2 % (2 * CPU)]), to_tf32(v[3 % (2 * CPU)]));
        }
    };
    // direct: A(i, k) = -Lambda(i, k) for K columns k in [s0, s_end)
    if ((Q * RPC < s_end || s_end >= n) && (Q + 1) * RPC > s0) {
        uint8_t *dst = lpack + (size_t)c * page_bytes + ((size_t)m * kc + Q) * tc::kAChunk;
#pragma unroll 2
        for (int u = 0; u < 8; ++u) {
            const int kk = Q * RPC + CPU * u;          // K columns kk .. kk+CPU-1 (the last tile also zeroes the padding)
            if (!(kk + CPU - 1 >= s0 && (kk < s_end || s_end >= n))) continue;
            float v[2 * CPU];
#pragma unroll
            for (int h = 0; h < CPU; ++h) {
                const int k = kk + h;
                float2 a = make_float2(0.f, 0.f);
                if (i < n && k >= s0 && k < s_end) {
                    const int sc = k - s0;
                    a = make_float2(-pl[(size_t)sc * ny + i + 1], -pl[(size_t)(kCkMaxN + sc) * ny + i + 1]);
                }
                v[2 * h] = imrow ? a.y : a.x;
                v[2 * h + 1] = imrow ? a.x : -a.y;
            }
            store(dst, u, v);
        }
    }
    // conjugate transpose: A(i, k) = -conj(Lambda(k, i)) for rows i in [s0, s_end)
    if (m * 64 >= s0 && m * 64 < s_end) {
        uint8_t *dst = lpack_h + (size_t)(C - 1 - c) * page_bytes + ((size_t)m * kc + Q) * tc::kAChunk;
#pragma unroll 2
        for (int u = 0; u < 8; ++u) {
            float v[2 * CPU];
#pragma unroll
            for (int h = 0; h < CPU; ++h) {
                const int k = Q * RPC + CPU * u + h;
                float2 a = make_float2(0.f, 0.f);
                if (i < n && i < s_end && k < n) {
                    const int sc = i - s0;
                    a = make_float2(-pl[(size_t)sc * ny + k + 1], pl[(size_t)(kCkMaxN + sc) * ny + k + 1]);
                }
                v[2 * h] = imrow ? a.y : a.x;
                v[2 * h + 1] = imrow ? a.x : -a.y;
            }
            store(dst, u, v);
        }
    }
}

// invT pages -> BF16 packed [Ar -Ai; Ai Ar] operands of invT_j and invT_j^H
// (32 complex columns per K chunk).  One thread per (row of the 128-row tile,
// chunk, M tile, page).
__global__ void pack_invT16_kernel(const float2 *__restrict__ invT, int ny, int n, int mt, int kc, size_t page_bytes,
                                   uint8_t *afwd, uint8_t *aadj) {
    const int i_s = threadIdx.x;
    const int c = blockIdx.x, m = blockIdx.y, j = blockIdx.z;
    const int i = m * 64 + (i_s & 63);
    const bool imrow = i_s >= 64;
    const size_t off = (size_t)j * page_bytes + ((size_t)m * kc + c) * tc::kAChunk;
    const float2 *page = invT + (size_t)j * ny * ny;
#pragma unroll 2
    for (int u = 0; u < 8; ++u) {
        uint32_t wf[4], wa[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int k = c * kCkRowsPerChunk16 + 4 * u + h;
            float2 af = make_float2(0.f, 0.f), aa = af;
            if (i < n && k < n) {
                af = page[(size_t)(i + 1) + (size_t)ny * (k + 1)];
                const float2 at = page[(size_t)(k + 1) + (size_t)ny * (i + 1)];
                aa = make_float2(at.x, -at.y);
            }
            const float f0 = imrow ? af.y : af.x, f1 = imrow ? af.x : -af.y;
            const float a0 = imrow ? aa.y : aa.x, a1 = imrow ? aa.x : -aa.y;
            wf[h] = (uint32_t)tc::to_bf16_bits(f0) | ((uint32_t)tc::to_bf16_bits(f1) << 16);
            wa[h] = (uint32_t)tc::to_bf16_bits(a0) | ((uint32_t)tc::to_bf16_bits(a1) << 16);
        }
        *reinterpret_cast<uint4 *>(afwd + off + tc::chunk_off16(i_s, 8 * u)) = make_uint4(wf[0], wf[1], wf[2], wf[3]);
        *reinterpret_cast<uint4 *>(aadj + off + tc::chunk_off16(i_s, 8 * u)) = make_uint4(wa[0], wa[1], wa[2], wa[3]);
    }
}

// Both packings in one pass: each thread reads the 32 complex values of its
// row in a BF16 K chunk and their transposes once, and writes the BF16 chunk
// and the two TF32 chunks (16 complex columns each) it covers, for invT_j
// and invT_j^H.  Same layouts as pack_invT_kernel and pack_invT16_kernel.
__global__ void pack_invT_both_kernel(const float2 *__restrict__ invT, int ny, int n, int mt, int kc, int kc16,
                                      size_t page_bytes16, uint8_t *afwd, uint8_t *aadj, uint8_t *afwd16,
                                      uint8_t *aadj16) {
    const int i_s = threadIdx.x;
    const int c16 = blockIdx.x, m = blockIdx.y, j = blockIdx.z;
    const int i = m * 64 + (i_s & 63);
    const bool imrow = i_s >= 64;
    const size_t off16 = (size_t)j * page_bytes16 + ((size_t)m * kc16 + c16) * tc::kAChunk;
    const float2 *page = invT + (size_t)j * ny * ny;
#pragma unroll 2
    for (int u = 0; u < 8; ++u) {                   // complex columns 4u .. 4u + 3 of the BF16 chunk
        uint32_t wf[4], wa[4];
        float vf[8], va[8];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int k = c16 * kCkRowsPerChunk16 + 4 * u + h;
            float2 af = make_float2(0.f, 0.f), aa = af;
            if (i < n && k < n) {
                af = page[(size_t)(i + 1) + (size_t)ny * (k + 1)];                  // invT(i, k)
                const float2 at = page[(size_t)(k + 1) + (size_t)ny * (i + 1)];     // invT(k, i)
                aa = make_float2(at.x, -at.y);                                      // invT^H(i, k)
            }
            const float f0 = imrow ? af.y : af.x, f1 = imrow ? af.x : -af.y;
            const float a0 = imrow ? aa.y : aa.x, a1 = imrow ? aa.x : -aa.y;
            wf[h] = (uint32_t)tc::to_bf16_bits(f0) | ((uint32_t)tc::to_bf16_bits(f1) << 16);
            wa[h] = (uint32_t)tc::to_bf16_bits(a0) | ((uint32_t)tc::to_bf16_bits(a1) << 16);
            vf[2 * h] = tc::to_tf32(f0);
            vf[2 * h + 1] = tc::to_tf32(f1);
            va[2 * h] = tc::to_tf32(a0);
            va[2 * h + 1] = tc::to_tf32(a1);
        }
        *reinterpret_cast<uint4 *>(afwd16 + off16 + tc::chunk_off16(i_s, 8 * u)) = make_uint4(wf[0], wf[1], wf[2], wf[3]);
        *reinterpret_cast<uint4 *>(aadj16 + off16 + tc::chunk_off16(i_s, 8 * u)) = make_uint4(wa[0], wa[1], wa[2], wa[3]);
        const int c = 2 * c16 + u / 4;               // TF32 chunk of these columns
        if (c < kc) {
            const size_t off = (((size_t)j * mt + m) * kc + c) * tc::kAChunk;
            const int ke = 8 * (u % 4);
            *reinterpret_cast<float4 *>(afwd + off + tc::chunk_off(i_s, ke)) = make_float4(vf[0], vf[1], vf[2], vf[3]);
            *reinterpret_cast<float4 *>(afwd + off + tc::chunk_off(i_s, ke + 4)) = make_float4(vf[4], vf[5], vf[6], vf[7]);
            *reinterpret_cast<float4 *>(aadj + off + tc::chunk_off(i_s, ke)) = make_float4(va[0], va[1], va[2], va[3]);
            *reinterpret_cast<float4 *>(aadj + off + tc::chunk_off(i_s, ke + 4)) = make_float4(va[4], va[5], va[6], va[7]);
        }
    }
}

void tc_pack_invT_both(const float2 *invT, int ny, int nx, const TcChunkGeom &g, uint8_t *afwd, uint8_t *aadj,
                       uint8_t *afwd16, uint8_t *aadj16, cudaStream_t st) {
    const dim3 grid(g.kc16, g.mt, nx);
    pack_invT_both_kernel<<<grid, 128, 0, st>>>(invT, ny, g.n, g.mt, g.kc, g.kc16, g.page_bytes16, afwd, aadj, afwd16,
                                                aadj16);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

void tc_pack_invT16(const float2 *invT, int ny, int nx, const TcChunkGeom &g, uint8_t *afwd16, uint8_t *aadj16,
                    cudaStream_t st) {
    const dim3 grid(g.kc16, g.mt, nx);
    pack_invT16_kernel<<<grid, 128, 0, st>>>(invT, ny, g.n, g.mt, g.kc16, g.page_bytes16, afwd16, aadj16);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

static void ck_configure() {
    // called before every launch: the attribute lives in the current
    // device's context, which a caller may switch or reset between calls
    WUST_CUDA(cudaFuncSetAttribute(tc_chunk_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCkSmem));
    WUST_CUDA(cudaFuncSetAttribute(tc_chunk_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCkSmem));
    WUST_CUDA(cudaFuncSetAttribute(tc_chunk_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCkSmem));
    WUST_CUDA(cudaFuncSetAttribute(tc_chunk_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCkSmem));
}

int tc_chunk_max_ctas() {
    ck_configure();
    int dev = 0, sms = 0, per_sm = 0;
    WUST_CUDA(cudaGetDevice(&dev));
    WUST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WUST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc_chunk_kernel<false, false>, kCkThreads, kCkSmem));
    return sms * per_sm;
}

static ChunkParams base_params(const Coefs<float2> &co, const TcChunkGeom &g, const TcChunkBuffers &b) {
    ChunkParams p{};
    p.page_bytes = g.page_bytes;
    p.co = co;
    p.bglob = b.bglob;
    p.zst = b.zst;
    p.sb = b.sb;
    p.edges = b.edges;
    p.group_ctr = b.sync;
    p.err = b.err;
    p.ny = co.ny;
    p.nx = co.nx;
    p.n = g.n;
    p.mt = g.mt;
    p.kc = g.kc;
    p.C = g.C;
    p.timeout_ns = 1000000000ull;
    return p;
}

// Chunk bounds (first step within the half) of one substitution.  The
// forward substitutions cut the columns at F[c] = c (nx-1) / C; the backward
// ones mirror the cuts so that the composed propagators of the H^H
// substitutions (which carry B states) are the conjugate transposes of those
// of the H substitutions: H backward chunk C-1-c covers the pages of the H^H
// forward chunk c, H^H backward chunk C-1-c the columns of H forward chunk c.
static void set_bounds(ChunkParams &p, int C, bool adjoint, int half) {
    const int steps = p.nx - 1;
    auto F = [&](int c) { return (int)((long long)c * steps / C); };
    for (int c = 0; c <= C; ++c) {
        if (half == 0) p.bounds[c] = F(c);
        else if (!adjoint) p.bounds[c] = steps - F(C - c);
        else p.bounds[c] = (c == 0 || c == C) ? (c == 0 ? 0 : steps) : steps - 1 - F(C - c);
    }
}

static void ck_launch(ChunkParams &p, bool adjoint, bool bf16, int pass, int groups, cudaStream_t st) {
    if (groups <= 0) return;
    p.pass = pass;
    WUST_CUDA(cudaMemsetAsync(p.group_ctr, 0, sizeof(unsigned) * groups, st));
    void *args[] = {&p};
    const dim3 grid(groups * p.mt), block(kCkThreads);
    void *fn = adjoint ? (bf16 ? (void *)tc_chunk_kernel<true, true> : (void *)tc_chunk_kernel<true, false>)
                       : (bf16 ? (void *)tc_chunk_kernel<false, true> : (void *)tc_chunk_kernel<false, false>);
    WUST_CUDA(cudaLaunchCooperativeKernel(fn, grid, block, args, kCkSmem, st));
    ++g_kernel_launches;
}

static uint8_t *lpack_of(const TcChunkGeom &g, uint8_t *lpack, bool adjoint, int half, size_t page_bytes) {
    return lpack + (size_t)((adjoint ? 2 : 0) + half) * g.C * page_bytes;
}

void tc_chunk_prepare(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcChunkGeom &g,
                      const TcChunkBuffers &b, cudaStream_t st) {
    (void)aadj;
    ck_configure();
    if (g.C < 3) return;
    ChunkParams p = base_params(co, g, b);
    const size_t sfl = tc_chunk_state_floats(co.ny);
    p.apack = afwd;
    for (int half = 0; half < 2; ++half) {
        p.half = half;
        set_bounds(p, g.C, false, half);
        uint8_t *lp = lpack_of(g, b.lpack, false, half, g.page_bytes);
        uint8_t *lph = lpack_of(g, b.lpack, true, 1 - half, g.page_bytes);
        for (int s0 = 0, N = 0; s0 < g.n; s0 += N) {
            // source tiles of whole 64-row M tiles (the transposed pack fills M tiles)
            N = std::min(kCkMaxN, ceil_div(g.n - s0, 64) * 64);
            p.s0 = s0;
            p.s_end = std::min(g.n, s0 + N);
            p.N = N;
            ck_launch(p, false, false, CK_PROP, g.C - 2, st);
            const dim3 grid(g.kc, g.mt, g.C - 2);
            pack_lambda_kernel<false><<<grid, 128, 0, st>>>(b.zst, sfl, co.ny, g.n, g.mt, g.kc, g.page_bytes, s0,
                                                            p.s_end, g.C, lp, lph);
            ++g_kernel_launches;
            if (b.lpack16) {
                const dim3 grid16(g.kc16, g.mt, g.C - 2);
                pack_lambda_kernel<true><<<grid16, 128, 0, st>>>(
                    b.zst, sfl, co.ny, g.n, g.mt, g.kc16, g.page_bytes16, s0, p.s_end, g.C,
                    lpack_of(g, b.lpack16, false, half, g.page_bytes16), lpack_of(g, b.lpack16, true, 1 - half, g.page_bytes16));
                ++g_kernel_launches;
            }
        }
    }
    WUST_LAUNCH_CHECK();
}

void tc_chunk_solve(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcChunkGeom &g,
                    const TcChunkBuffers &b, const SrcView &src, int S, bool adjoint, float2 *u, bool bf16,
                    cudaStream_t st) {
    ck_configure();
    const int ny = co.ny, nx = co.nx;
    WUST_CUDA(cudaMemsetAsync(u, 0, sizeof(float2) * (size_t)ny * nx * S, st));
    ChunkParams p = base_params(co, g, b);
    p.apack = adjoint ? aadj : afwd;
    if (bf16) {
        p.kc = g.kc16;
        p.page_bytes = g.page_bytes16;
    }
    p.src = src;
    p.u = u;
    for (int s0 = 0; s0 < S; s0 += kCkMaxN) {
        p.s0 = s0;
        p.s_end = std::min(S, s0 + kCkMaxN);
        p.N = ceil_div(p.s_end - s0, 16) * 16;
        for (int half = 0; half < 2; ++half) {
            p.half = half;
            set_bounds(p, g.C, adjoint, half);
            p.lpack = bf16 ? lpack_of(g, b.lpack16, adjoint, half, g.page_bytes16)
                           : lpack_of(g, b.lpack, adjoint, half, g.page_bytes);
            ck_launch(p, adjoint, bf16, CK_FIRST, g.C, st);
            if (g.C >= 3) {
                // the chain of C - 2 dense steps on up to C groups, each
                // carrying a 16-multiple slice of the sources (one group
                // would leave all but mt SMs idle for the whole chain)
                const int N = p.N;
                const int per = ceil_div(ceil_div(N, g.C), 16) * 16;
                p.N = per;
                ck_launch(p, adjoint, bf16, CK_BOUNDARY, ceil_div(N, per), st);
                p.N = N;
            }
            if (g.C >= 2) ck_launch(p, adjoint, bf16, CK_SECOND, g.C - 1, st);
        }
    }
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
