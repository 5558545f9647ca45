// Schur inverses of decompBlockLU (Runtime/solver/decompBlockLU.cu:337-368)
// by Newton-Schulz iteration on the tensor cores, for the refined TF32
// profile (whose FP64-residual refinement absorbs the TF32 error of the
// factor, as it does that of the sweeps).
//
// Adjacent Schur complements of the Helmholtz operator differ little: with
// X_0 = invT_{j-1}, the residual R_0 = I - T_j X_0 of the interior columns
// has an RMS singular value of 1e-3 (homogeneous medium) to 0.3 (tissue
// texture).  Newton-Schulz squares it every iteration:
//     R_k = I - T_j X_k,     X_{k+1} = X_k + X_k R_k,     R_{k+1} = R_k^2,
// so one to four iterations (two complex GEMMs each) replace the O(n)
// sequential pivot steps of Gauss-Jordan.  Per column, with r_k the RMS of
// R_k (||R_k||_F / sqrt(n), summed in a fixed order so every CTA decides
// alike):
//     r_k <= kAccept                      accept X_k
//     r_k <= kLastUpdate(First), stalled  one more update, accept
//     r_k <= kCubicLast                   one cubic update, accept
//     diverging / not contracting         give the column back (Gauss-Jordan)
// The cubic update X_{k+1} = X_k (I + R_k + R_k^2), residual R_k^3, takes two
// dependent GEMMs (Y = X_k R_k, then X_k + Y + Y R_k) where the quadratic
// route takes three (X_{k+1}, R_{k+1}, X_{k+2}): from r_k <= 0.04 its
// residual 6.4e-5 is well below the TF32 floor of the products (3.5e-4).  On
// a textured medium most first residuals lie between 2e-2 and 4e-2 (median
// 2.8e-2, 90th percentile 3.4e-2 at 552^2, 1.2 MHz), so most pages cost 3
// GEMMs instead of 4.  (With a limit of 0.06 the pages next to the PML of a
// textured 330^2 grid came out 5.0e-3 off the Gauss-Jordan pages.)
// Columns where X_{j-1} is no start (the Dirichlet columns, the first
// columns after them) go to the Gauss-Jordan kernel; the host driver
// alternates between the two.
//
// Both products are n x n x n complex GEMMs, split into one real GEMM with
// re/im interleaved along K (rows 0-63 of a 128-row A tile give the real
// parts of 64 complex rows, rows 64-127 the imaginary parts):
//     A = [Yr -Yi; Yi Yr] packed per (64-row tile, 16-column K chunk),
//     B = complex columns of Z packed per (112-column tile, K chunk).
// Grid: 64-row tiles x 112-column tiles x ks K slices, one CTA per SM,
// launched cooperatively; operands stream through a shared-memory ring with
// cp.async.bulk.  The ks CTAs of a tile form one thread-block cluster: each
// keeps its TF32 partial tile in its own shared memory and, after a bounded
// cluster barrier, each sums one row slice of the tile from the cluster's
// shared memory in rank order and writes the epilogue (R in B layout, or X
// in A and B layouts and into its resident slice).  A solver confined to a
// partition of the SMs runs the same kernel without clusters: partials
// through L2, a grid barrier after every GEMM.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace wust {

using tc::chunk_off;
using tc::to_tf32;

namespace {

constexpr int NTN = 112;                           // MMA N: complex columns per tile
constexpr int kRows = 64;                          // complex rows per M tile
constexpr int kKRows = 16;                         // complex K rows per chunk
constexpr int kStages = 5;
constexpr int kNsThreads = 512;
constexpr int kPartCols = (NTN / (kNsThreads / 128) + 7) / 8 * 8;   // TMEM columns per warp of the partial tile
constexpr int kBChunkNs = NTN * tc::kChunkBytes;   // 14 KB
constexpr int kStageBytes = tc::kAChunk + kBChunkNs;
constexpr int kSP = NTN + 1;                       // pitch (float2) of a staged slice row
constexpr int kSliceRows = ((kRows + 2) / 3 + 1) & ~1;   // rows of the largest slice (ks >= 3)
// ring, barriers and scalars, then this CTA's resident X and Y slices
constexpr size_t kNsSmem = (size_t)kStages * kStageBytes + 512 + 2 * (size_t)kSliceRows * kSP * sizeof(float2);
static_assert(kNsSmem <= 232448, "shared memory of one CTA");
constexpr int kTmemCols = 128;
constexpr int kNsCopyTid = 96;                     // the ring's copy thread (warp 3, lane 0)

constexpr float kAccept = 2e-4f;        // residual small enough: keep X_k
// One more update, then accept: from the page's first residual (the
// previous page's inverse as the start) when r_0 <= kLastUpdateFirst (the
// accepted page then has r ~ 4e-4, at the TF32 floor of ~3.5e-4), from a
// later residual when r_k <= kLastUpdate.  Measured at 552^2, 256 sources,
// 1.2 MHz: (3e-2, 1e-2) saves 8 ms of factorization on a half-textured
// medium but the fully textured one then needs a third refinement
// correction; (2e-2, 1e-2) keeps two corrections on both and saves 2.3 ms.
constexpr float kLastUpdateFirst = 2e-2f;
constexpr float kLastUpdate = 1e-2f;
constexpr float kCubicLast = 0.04f;     // one cubic update, then accept
constexpr float kFirstFail = 0.8f;      // X_{j-1} is no start for this column
constexpr float kStallAccept = 0.05f;   // stalled at this level: finish with one update

enum { NS_SITE_COPY = 21, NS_SITE_MMA = 22, NS_SITE_SYNC = 23, NS_SITE_CLUSTER = 24, NS_SITE_SHAPE = 25 };

// Cluster launch: the K slices of one tile form a thread-block cluster; each
// CTA keeps its partial tile in its own shared memory (pitch kPartPitch
// floats: 16-byte rows whose float4 stores from 8 consecutive TMEM lanes hit
// distinct banks) at kPartOff, in the operand ring, which is idle from the
// end of a GEMM to the grid barrier before the next one.
constexpr int kPartPitch = NTN + 4;
constexpr size_t kPartOff = 65536;
static_assert(kPartOff + 128 * kPartPitch * sizeof(float) <= (size_t)kStages * kStageBytes, "partial tile in the ring");

// Generic address of the same shared-memory location in cluster rank `rank`.
template <typename T>
__device__ __forceinline__ const T *peer_shared(const T *local, uint32_t rank) {
    uint64_t out;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(out) : "l"(local), "r"(rank));
    return reinterpret_cast<const T *>(out);
}

// Hardware barrier of all threads of the cluster (unbounded: used only where
// every thread of every CTA of the cluster arrives unconditionally).
__device__ __forceinline__ void cluster_barrier_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Bounded barrier of the cluster's CTAs on a counter in rank 0's shared
// memory (ctr: its shared::cluster address); false on an expired wait or a
// reported error.
__device__ __forceinline__ bool cluster_sync(uint32_t ctr, unsigned target, int *err, int *s_ok,
                                             unsigned long long timeout_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("fence.acq_rel.cluster;" ::: "memory");
        asm volatile("red.release.cluster.shared::cluster.add.u32 [%0], %1;" ::"r"(ctr), "r"(1u) : "memory");
        int ok = 1;
        const unsigned long long t0 = global_timer_ns();
        for (unsigned spin = 0;; ++spin) {
            unsigned v;
            asm volatile("ld.acquire.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(ctr) : "memory");
            if ((int)(v - target) >= 0) break;
            if ((spin & 15u) == 15u) {
                if (*(volatile int *)err) { ok = 0; break; }
                if (global_timer_ns() - t0 > timeout_ns) {
                    atomicCAS(err, 0, NS_SITE_CLUSTER);
                    ok = 0;
                    break;
                }
            }
        }
        asm volatile("fence.acq_rel.cluster;" ::: "memory");
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

}  // namespace

// Optional phase timer (SM cycles of CTA 0, summed), profiling builds only.
#ifdef WUST_NS_PROFILE
__device__ unsigned long long g_ns_prof[16];
#define NSPROF(k)                                                                                  \
    do {                                                                                           \
        if (bid == 0 && threadIdx.x == 0) {                                                        \
            const long long t_ = clock64();                                                        \
            g_ns_prof[k] += (unsigned long long)(t_ - prof_t);                                     \
            prof_t = t_;                                                                           \
        }                                                                                          \
    } while (0)
extern "C" int wust_ns_profile_read(unsigned long long *out) {
    return (int)cudaMemcpyFromSymbol(out, g_ns_prof, sizeof(g_ns_prof));
}
extern "C" int wust_ns_profile_reset() {
    unsigned long long z[16] = {};
    return (int)cudaMemcpyToSymbol(g_ns_prof, z, sizeof(z));
}
#else
#define NSPROF(k) ((void)0)
#endif

struct NsParams {
    Coefs<float2> co;
    float2 *invT;            // [ny, ny, nx] column-major pages
    float2 *xf0, *xf1;       // X, fp32 complex, column-major n x n: an update reads one and writes the other
    float2 *xy;              // Y = X_k R_k of a cubic update, same layout
    uint8_t *aT;             // A-packed T_j: [mt][kc] x 16 KB
    uint8_t *aX0, *aX1;      // A-packed X, same layout, with xf0 / xf1 (an update reads one and writes the other)
    uint8_t *bX, *bR;        // B-packed X and R:   [ntn][kc] x 14 KB
    float *part;             // [tile][ks][128][NTN]
    double *rn;              // [nblocks] per-CTA sums of |R|^2
    unsigned *ctr;           // grid barrier counter
    int *err;                // wait-site code
    int *status;             // [0] failed column or -1, [1] GEMMs, [2] updates, [3] columns done
    int ny, nx, n, mt, ntn, kc, ks, per;
    int j0, j1, max_iter;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ bool ns_sync(unsigned *ctr, unsigned target, int *err, int *s_ok,
                                        unsigned long long timeout_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        asm volatile("fence.proxy.async.global;" ::: "memory");
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
                    atomicCAS(err, 0, NS_SITE_SYNC);
                    ok = 0;
                    break;
                }
            }
        }
        asm volatile("fence.proxy.async.global;" ::: "memory");
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// X(r, c) into the A layout (two stacked rows) and the B layout.
__device__ __forceinline__ void put_x_packed(const NsParams &p, uint8_t *aX, uint8_t *bX, int r, int c, float2 v) {
    const float xr = to_tf32(v.x), xi = to_tf32(v.y);
    uint8_t *ac = aX + ((size_t)(r / kRows) * p.kc + c / kKRows) * tc::kAChunk;
    const int ke = 2 * (c % kKRows);
    *reinterpret_cast<float2 *>(ac + chunk_off(r % kRows, ke)) = make_float2(xr, -xi);
    *reinterpret_cast<float2 *>(ac + chunk_off(r % kRows + kRows, ke)) = make_float2(xi, xr);
    uint8_t *bc = bX + ((size_t)(c / NTN) * p.kc + r / kKRows) * kBChunkNs;
    *reinterpret_cast<float2 *>(bc + chunk_off(c % NTN, 2 * (r % kKRows))) = make_float2(xr, xi);
}

// CL: launched as clusters of the ks K slices of each tile (partials in
// shared memory, read across the cluster); otherwise partials through L2.
template <bool CL>
__global__ void __launch_bounds__(kNsThreads, 1) ns_factor_kernel(NsParams p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *misc = smem + (size_t)kStages * kStageBytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(misc);
    uint64_t *empty = full + kStages;
    uint64_t *done = empty + kStages;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(misc + 128);
    int *s_ok = reinterpret_cast<int *>(misc + 132);
    int *s_dec = reinterpret_cast<int *>(misc + 136);        // decision, r_k
    double *s_red = reinterpret_cast<double *>(misc + 192);  // one per warp
    unsigned *s_cctr = reinterpret_cast<unsigned *>(misc + 384);   // cluster barrier counter (rank 0's is used)
    float *spart = reinterpret_cast<float *>(smem + kPartOff);     // [128][kPartPitch] partial tile (CL)
    // this CTA's slice of the current X and of a cubic update's Y, resident
    // across the GEMMs (outside the ring); global memory keeps only the
    // values other CTAs' windows read
    float2 *sxk = reinterpret_cast<float2 *>(misc + 512);          // [kSliceRows][kSP]
    float2 *syk = sxk + (size_t)kSliceRows * kSP;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = blockIdx.x, nb = blockIdx.y, ks = blockIdx.z;
    const int KS = p.ks;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int ny = p.ny, n = p.n;
    const size_t page_sz = (size_t)ny * ny;
    const int tile = mt + p.mt * nb;
    const int c0 = ks * p.per;
    const int nch = max(0, min(p.kc, c0 + p.per) - c0);
    const int gthreads = nblocks * kNsThreads;
    const int gtid = bid * kNsThreads + tid;
    unsigned epoch = 0;
#ifdef WUST_NS_PROFILE
    long long prof_t = clock64();
#endif

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        *s_cctr = 0u;
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, kTmemCols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;
    // every CTA of the cluster has started (and zeroed its counter) before
    // any shared memory of another is touched
    if (CL) cluster_barrier_all();
    const uint32_t cctr0 = CL ? (uint32_t)__cvta_generic_to_shared(s_cctr) : 0u;
    uint32_t cctr = 0;
    if (CL) asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(cctr) : "r"(cctr0), "r"(0u));
    unsigned ctarget = 0;

    uint32_t u_issue = 0, u_cons = 0;    // ring counters (copy thread, thread 0)
    uint32_t n_gemm = 0;                 // GEMMs run (done-barrier phase)
    bool ok = true;
    if (CL) {
        // the K slices of this tile must be this cluster, in rank order;
        // launched in any other shape (the same in every CTA), no CTA does
        // any work or touches another's shared memory, and the host reruns
        // the pages with the classic kernel
        uint32_t ncta, rank;
        asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncta));
        asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
        if (ncta != (uint32_t)KS || rank != (uint32_t)ks) {
            if (tid == 0) atomicCAS(p.err, 0, NS_SITE_SHAPE);
            ok = false;
        }
    }

    // One GEMM C = Apack * Bpack^T over this CTA's K slice into TMEM, then
    // the partial tile into L2 (or, CL, into this CTA's shared memory, and
    // with `edges` the tile's first and last rows and columns also into L2,
    // where the neighbouring tiles read their windows' halos).  Returns false
    // on an expired wait.  The copy thread (kNsCopyTid) refills each stage as
    // soon as the MMAs that read it have completed; thread 0 issues each
    // chunk's MMAs as soon as its copies have landed.  Both count the chunks
    // of every GEMM (u_issue, u_cons), so a stage's parity carries over from
    // one GEMM to the next.
    auto gemm = [&](const uint8_t *Apack, const uint8_t *Bpack, bool edges) -> bool {
        NSPROF(14);
        if (tid == kNsCopyTid) {
            const uint8_t *ab = Apack + ((size_t)mt * p.kc + c0) * tc::kAChunk;
            const uint8_t *bb = Bpack + ((size_t)nb * p.kc + c0) * kBChunkNs;
            bool good = true;
            for (int c = 0; c < nch && good; ++c) {
                const uint32_t s = u_issue % kStages, f = u_issue / kStages;
                if (f >= 1 && !tc::mbar_wait(&empty[s], (f - 1) & 1u, p.timeout_ns)) {
                    good = false;
                    break;
                }
                uint8_t *st = smem + (size_t)s * kStageBytes;
                tc::mbar_expect_tx(&full[s], kStageBytes);
                tc::bulk_g2s(st, ab + (size_t)c * tc::kAChunk, tc::kAChunk, &full[s]);
                tc::bulk_g2s(st + tc::kAChunk, bb + (size_t)c * kBChunkNs, kBChunkNs, &full[s]);
                ++u_issue;
            }
            if (!good) atomicCAS(p.err, 0, NS_SITE_COPY);
        }
        if (tid == 0) {
            bool good = true;
            constexpr uint32_t kIdesc = tc::instr_desc<true>(tc::kTileRows, NTN);
            for (int c = 0; c < nch; ++c) {
                const uint32_t s = u_cons % kStages, f = u_cons / kStages;
                if (!tc::mbar_wait(&full[s], f & 1u, p.timeout_ns)) { good = false; }
                if (c == 0) NSPROF(11);
                ++u_cons;
                tc::fence_after();
                const uint8_t *st = smem + (size_t)s * kStageBytes;
#pragma unroll
                for (int k = 0; k < tc::kChunkBytes / 32; ++k)
                    tc::mma<true>(tmem, tc::smem_desc(st + k * 256), tc::smem_desc(st + tc::kAChunk + k * 256), kIdesc,
                                  (c > 0 || k > 0) ? 1u : 0u);
                tc::commit(&empty[s]);
            }
            tc::commit(done);
            if (!good) atomicCAS(p.err, 0, NS_SITE_COPY);
        }
        NSPROF(1);
        if (!tc::mbar_wait(done, n_gemm & 1u, p.timeout_ns)) atomicCAS(p.err, 0, NS_SITE_MMA);
        NSPROF(2);
        ++n_gemm;
        tc::fence_after();
        // partial tile: warp w reads TMEM lanes 32(w%4).., columns
        // [kPartCols (w/4), kPartCols (w/4 + 1)) within the tile
        const int row = 32 * (warp & 3) + lane;
        const int cb0 = kPartCols * (warp >> 2);
        float *mypart = p.part + ((size_t)(tile * KS + ks) * 128 + row) * NTN + cb0;
        float *myspart = spart + (size_t)row * kPartPitch + cb0;
        const bool edge_row = (row & (kRows - 1)) == 0 || (row & (kRows - 1)) == kRows - 1;
#pragma unroll
        for (int cb = 0; cb < kPartCols; cb += 8) {
            if (cb0 + cb >= NTN) break;                // warp-uniform
            float t[8];
            if (nch > 0) {
                tc::tmem_ld8(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(cb0 + cb), t);
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) t[q] = 0.f;
            }
            if (CL) {
                *reinterpret_cast<float4 *>(myspart + cb) = make_float4(t[0], t[1], t[2], t[3]);
                *reinterpret_cast<float4 *>(myspart + cb + 4) = make_float4(t[4], t[5], t[6], t[7]);
                if (edges) {
                    if (edge_row) {
                        __stcg(reinterpret_cast<float4 *>(mypart + cb), make_float4(t[0], t[1], t[2], t[3]));
                        __stcg(reinterpret_cast<float4 *>(mypart + cb + 4), make_float4(t[4], t[5], t[6], t[7]));
                    } else {
                        if (cb0 + cb == 0) __stcg(mypart + cb, t[0]);
                        if (cb0 + cb + 8 == NTN) __stcg(mypart + cb + 7, t[7]);
                    }
                }
            } else {
                __stcg(reinterpret_cast<float4 *>(mypart + cb), make_float4(t[0], t[1], t[2], t[3]));
                __stcg(reinterpret_cast<float4 *>(mypart + cb + 4), make_float4(t[4], t[5], t[6], t[7]));
            }
        }
        tc::fence_before();
        NSPROF(3);
        bool synced = true;
        // CL: the cluster's barrier publishes the shared partials; a GEMM
        // with edges needs the grid barrier, whose gpu-scope release and
        // acquire cover the cluster's shared memory too
        if (CL && !edges) {
            ctarget += (unsigned)KS;
            synced = cluster_sync(cctr, ctarget, p.err, s_ok, p.timeout_ns);
            NSPROF(4);
            return synced;
        }
        epoch += (unsigned)nblocks;
        synced = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns) && synced;
        NSPROF(4);
        return synced;
    };

    // Rows of this tile whose split-K sum this CTA forms.
    const int rows_per = ((kRows + KS - 1) / KS + 1) & ~1;   // even: B-layout units hold row pairs
    const int rbeg = ks * rows_per, rend = min(kRows, rbeg + rows_per);
    // This CTA's epilogue items: item m of thread tid is it = tid + kNsThreads m over
    // the (rend - rbeg) x NTN slice; their split-K sums, with every load of a
    // rank in flight at once.
    constexpr int kEpi = ((kRows + 2) / 3 * NTN + kNsThreads - 1) / kNsThreads;   // bound for ks >= 3
    const int n_items = (rend - rbeg) * NTN;
    auto tile_values = [&](float2 (&v)[kEpi]) {
        const float *pt = p.part + (size_t)tile * KS * 128 * NTN;
#pragma unroll
        for (int m = 0; m < kEpi; ++m) v[m] = make_float2(0.f, 0.f);
        for (int q = 0; q < KS; ++q) {
            if (CL) {                       // rank q of the cluster holds K slice q
                const float *pq = peer_shared(spart, (uint32_t)q);
#pragma unroll
                for (int m = 0; m < kEpi; ++m) {
                    const int it = tid + kNsThreads * m;
                    if (it < n_items) {
                        const int rl = rbeg + it / NTN, cl = it % NTN;
                        v[m].x += pq[rl * kPartPitch + cl];
                        v[m].y += pq[(rl + kRows) * kPartPitch + cl];
                    }
                }
                continue;
            }
            const float *pq = pt + (size_t)q * 128 * NTN;
#pragma unroll
            for (int m = 0; m < kEpi; ++m) {
                const int it = tid + kNsThreads * m;
                if (it < n_items) {
                    const int rl = rbeg + it / NTN, cl = it % NTN;
                    v[m].x += __ldcg(pq + (size_t)rl * NTN + cl);
                    v[m].y += __ldcg(pq + (size_t)(rl + kRows) * NTN + cl);
                }
            }
        }
    };

    // Staging of this CTA's slice (rows rbeg..rend-1 of the M tile, all NTN
    // columns) in the operand ring, which is idle between GEMMs; from there
    // every packed layout is written in whole 16-byte units.
    constexpr int SP = kSP;                                      // staged row pitch (float2)
    float2 *sx = reinterpret_cast<float2 *>(smem);               // [rows_per][SP]
    float2 *xw = reinterpret_cast<float2 *>(smem + 32768);       // Schur window [rows_per + 2][SP + 2]
    const int nr = rend - rbeg;
    const int grow0 = mt * kRows + rbeg;                         // global row of slice row 0
    const int gcol0 = nb * NTN;
    // A layout (rows i_s = r % 64 and r % 64 + 64, K units of two columns)
    auto write_a = [&](uint8_t *Apack, const float2 *src) {
        for (int u = tid; u < nr * (NTN / 2); u += kNsThreads) {
            const int rl = u % nr, cp = u / nr;
            const int r = grow0 + rl, c = gcol0 + 2 * cp;
            if (r >= n || c >= n) continue;
            const float2 y0 = src[rl * SP + 2 * cp];
            const float2 y1 = c + 1 < n ? src[rl * SP + 2 * cp + 1] : make_float2(0.f, 0.f);
            uint8_t *ac = Apack + ((size_t)mt * p.kc + c / kKRows) * tc::kAChunk;
            const int ke = 2 * (c % kKRows);
            *reinterpret_cast<float4 *>(ac + chunk_off(r % kRows, ke)) =
                make_float4(to_tf32(y0.x), -to_tf32(y0.y), to_tf32(y1.x), -to_tf32(y1.y));
            *reinterpret_cast<float4 *>(ac + chunk_off(r % kRows + kRows, ke)) =
                make_float4(to_tf32(y0.y), to_tf32(y0.x), to_tf32(y1.y), to_tf32(y1.x));
        }
    };
    // B layout (column cl, K units of two rows)
    auto write_b = [&](uint8_t *Bpack, const float2 *src) {
        for (int u = tid; u < (nr / 2) * NTN; u += kNsThreads) {
            const int cl = u % NTN, rp = u / NTN;
            const int r = grow0 + 2 * rp, c = gcol0 + cl;
            if (r >= n || c >= n) continue;
            const float2 z0 = src[(2 * rp) * SP + cl];
            const float2 z1 = r + 1 < n ? src[(2 * rp + 1) * SP + cl] : make_float2(0.f, 0.f);
            uint8_t *bc = Bpack + ((size_t)nb * p.kc + r / kKRows) * kBChunkNs;
            *reinterpret_cast<float4 *>(bc + chunk_off(cl, 2 * (r % kKRows))) =
                make_float4(to_tf32(z0.x), to_tf32(z0.y), to_tf32(z1.x), to_tf32(z1.y));
        }
    };
    // column-major copy (leading dimension ld, element (r, c) at base[r + ld c])
    auto write_cm = [&](float2 *base, size_t ld, const float2 *src) {
        for (int u = tid; u < nr * NTN; u += kNsThreads) {
            const int rl = u % nr, cl = u / nr;
            const int r = grow0 + rl, c = gcol0 + cl;
            if (r < n && c < n) base[(size_t)r + ld * c] = src[rl * SP + cl];
        }
    };
    // the values of the slice that other CTAs' windows read (its first and
    // last rows, the tile's first and last columns) into an n x n
    // column-major array
    auto write_edges = [&](float2 *base, const float2 *src) {
        for (int u = tid; u < 2 * NTN + 2 * nr; u += kNsThreads) {
            int rl, cl;
            if (u < NTN) { rl = 0; cl = u; }
            else if (u < 2 * NTN) { rl = nr - 1; cl = u - NTN; }
            else if (u < 2 * NTN + nr) { rl = u - 2 * NTN; cl = 0; }
            else { rl = u - 2 * NTN - nr; cl = NTN - 1; }
            const int r = grow0 + rl, c = gcol0 + cl;
            if (r < n && c < n) base[(size_t)r + (size_t)n * c] = src[rl * SP + cl];
        }
    };

    // ---- start: X = invT_{j0-1} into the fp32 and packed copies; zero the
    //      borders of the pages this launch writes ----------------------------
    if (ok) {
        const float2 *X = p.invT + (size_t)(p.j0 - 1) * page_sz;
        for (int idx = gtid; idx < n * n; idx += gthreads) {
            const int r = idx % n, c = idx / n;
            const float2 v = X[(size_t)(r + 1) + (size_t)ny * (c + 1)];
            p.xf0[idx] = v;
            put_x_packed(p, p.aX0, p.bX, r, c, v);
        }
        for (size_t idx = gtid; idx < (size_t)(p.j1 - p.j0) * 4 * ny; idx += gthreads) {
            const size_t page = p.j0 + idx / (4 * (size_t)ny);
            const int rem = (int)(idx % (4 * (size_t)ny));
            const int which = rem / ny, k = rem % ny;
            const size_t off = which == 0 ? (size_t)ny * k
                             : which == 1 ? (size_t)(ny - 1) + (size_t)ny * k
                             : which == 2 ? (size_t)k
                                          : (size_t)k + (size_t)ny * (ny - 1);
            p.invT[page * page_sz + off] = make_float2(0.f, 0.f);
        }
        for (int u = tid; u < nr * NTN; u += kNsThreads) {
            const int rl = u / NTN, cl = u % NTN;
            const int r = grow0 + rl, c = gcol0 + cl;
            sxk[rl * SP + cl] = r < n && c < n ? X[(size_t)(r + 1) + (size_t)ny * (c + 1)] : make_float2(0.f, 0.f);
        }
        epoch += (unsigned)nblocks;
        ok = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns);
    }

    // ---- T_jt = D_jt - L_{jt-1} X U_{jt-1} (interior, A layout) of this
    //      CTA's slice, with X = X_{jt-1}.  fill_window puts X's window (the
    //      slice's rows and columns, one more on each side) into xw; its
    //      loads are issued after the coefficient loads, so both are in flight
    const int wr = nr + 2, wc = NTN + 2;
    float2 *cw_ = xw + (size_t)(kRows / 3 + 3) * (SP + 2);   // [3][NTN] column coefs ud, uu, ul
    float2 *rw_ = cw_ + 3 * NTN;                            // [6][rows] row coefs ld, ll, lu, dd, dl, du
    auto build_T = [&](int jt, auto &&fill_window) {
        const int jm = jt - 1;
        // coefficients: items [0, 3 NTN) columns, [3 NTN, 3 NTN + 6 nr) rows
        float2 cf[2];
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int q = tid + kNsThreads * m;
            float2 v2 = make_float2(0.f, 0.f);
            if (q < 3 * NTN) {
                const int which = q / NTN, cl = q % NTN, C = gcol0 + cl + 1;
                if (C <= n) v2 = which == 0 ? p.co.ud(C, jm) : which == 1 ? p.co.uu(C - 1, jm) : p.co.ul(C, jm);
            } else if (q < 3 * NTN + 6 * nr) {
                const int rt = q - 3 * NTN, which = rt / nr, rl = rt % nr, R = grow0 + rl + 1;
                if (R <= n) {
                    if (which == 0) v2 = p.co.ld(R, jm);
                    else if (which == 1) v2 = p.co.ll(R - 1, jm);
                    else if (which == 2) v2 = p.co.lu(R, jm);
                    else if (which == 3) v2 = p.co.dd(R, jt);
                    else if (which == 4) v2 = p.co.dl(R, jt);        // element (R+1, R)
                    else if (R >= 2) v2 = p.co.du(R - 1, jt);        // element (R-1, R)
                }
            }
            cf[m] = v2;
        }
        fill_window();
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int q = tid + kNsThreads * m;
            if (q < 3 * NTN + 6 * nr) cw_[q] = cf[m];       // rw_ follows cw_ directly
        }
        __syncthreads();
        for (int u = tid; u < nr * NTN; u += kNsThreads) {
            const int cl = u % NTN, rl = u / NTN;
            const int r = grow0 + rl, c = gcol0 + cl;
            float2 v = make_float2(0.f, 0.f);
            if (r < n && c < n) {
                // D_jt(R, C): dd on the diagonal, dl(C) below (R = C+1), du(R) above (C = R+1)
                if (r == c) v = rw_[3 * nr + rl];
                else if (r == c + 1) v = rw_[4 * nr + (rl - 1 >= 0 ? rl - 1 : 0)];
                else if (r + 1 == c) v = rw_[5 * nr + (rl + 1 < nr ? rl + 1 : rl)];
                if (r == c + 1 && rl == 0) v = p.co.dl(c + 1, jt);         // pair leaves the slice
                if (r + 1 == c && rl + 1 >= nr) v = p.co.du(r + 1, jt);
                const float2 udc = cw_[cl], uuc = cw_[NTN + cl], ulc = cw_[2 * NTN + cl];
                float2 right[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {               // rows r-1, r, r+1 (window row rl + d)
                    const float2 *xr = xw + (rl + d) * (SP + 2) + cl;    // columns c-1, c, c+1
                    float2 acc = cmul(xr[1], udc);
                    cfma(acc, xr[0], uuc);
                    cfma(acc, xr[2], ulc);
                    right[d] = acc;
                }
                float2 lr = cmul(rw_[rl], right[1]);
                cfma(lr, rw_[nr + rl], right[0]);
                cfma(lr, rw_[2 * nr + rl], right[2]);
                v = csub(v, lr);
            }
            sx[rl * SP + cl] = v;
        }
        __syncthreads();
        write_a(p.aT, sx);
    };
    // window of an X held whole in global memory (all loads of a thread in flight)
    // window of the current X: the slice from sxk, the halo ring from the
    // edges its owners wrote to X (global)
    auto window_from = [&](const float2 *X) {
        const int n_halo = 2 * wc + 2 * nr;
        if (tid < n_halo) {
            const int h = tid;
            int hrw, hcw;
            if (h < wc) { hrw = 0; hcw = h; }
            else if (h < 2 * wc) { hrw = nr + 1; hcw = h - wc; }
            else if (h < 2 * wc + nr) { hrw = 1 + (h - 2 * wc); hcw = 0; }
            else { hrw = 1 + (h - 2 * wc - nr); hcw = NTN + 1; }
            const int r = grow0 - 1 + hrw, c = gcol0 - 1 + hcw;
            xw[hrw * (SP + 2) + hcw] =
                r >= 0 && r < n && c >= 0 && c < n ? X[(size_t)r + (size_t)n * c] : make_float2(0.f, 0.f);
        }
        for (int u = tid; u < nr * NTN; u += kNsThreads) {
            const int rl = u / NTN, cl = u % NTN;
            const bool in = grow0 + rl < n && gcol0 + cl < n;
            xw[(rl + 1) * (SP + 2) + cl + 1] = in ? sxk[rl * SP + cl] : make_float2(0.f, 0.f);
        }
    };
    // window of X_{k+1} = X_k + (X_k R_k) right after an update: the slice is
    // in sxk; each halo value is its owner's sum, formed here the same way
    // (X_k from Xold plus the split-K partials of the owner's tile, in rank
    // order), so no barrier is needed before the next Schur complement
    auto window_after_update = [&](const float2 *Xold, const float2 *Yadd) {
        const int n_halo = 2 * wc + 2 * nr;
        float2 hv = make_float2(0.f, 0.f);
        int hrw = 0, hcw = 0;
        if (tid < n_halo) {
            const int h = tid;
            if (h < wc) { hrw = 0; hcw = h; }
            else if (h < 2 * wc) { hrw = nr + 1; hcw = h - wc; }
            else if (h < 2 * wc + nr) { hrw = 1 + (h - 2 * wc); hcw = 0; }
            else { hrw = 1 + (h - 2 * wc - nr); hcw = NTN + 1; }
            const int r = grow0 - 1 + hrw, c = gcol0 - 1 + hcw;
            if (r >= 0 && r < n && c >= 0 && c < n) {
                const float *pt = p.part + (size_t)((r / kRows) + p.mt * (c / NTN)) * KS * 128 * NTN;
                const int rl = r % kRows, cl = c % NTN;
                float vx = 0.f, vy = 0.f;
                if (CL && r / kRows == mt && c / NTN == nb) {     // this tile: the cluster's shared partials
                    for (int q = 0; q < KS; ++q) {
                        const float *pq = peer_shared(spart, (uint32_t)q);
                        vx += pq[rl * kPartPitch + cl];
                        vy += pq[(rl + kRows) * kPartPitch + cl];
                    }
                } else {                    // another tile's edge (CL: written to L2 by its last GEMM)
                    for (int q = 0; q < KS; ++q) {
                        vx += __ldcg(pt + ((size_t)q * 128 + rl) * NTN + cl);
                        vy += __ldcg(pt + ((size_t)q * 128 + rl + kRows) * NTN + cl);
                    }
                }
                float2 xo = Xold[(size_t)r + (size_t)n * c];
                if (Yadd) {
                    const float2 yo = __ldcg(Yadd + (size_t)r + (size_t)n * c);
                    xo = make_float2(xo.x + yo.x, xo.y + yo.y);
                }
                hv = make_float2(xo.x + vx, xo.y + vy);
            }
        }
        for (int u = tid; u < nr * NTN; u += kNsThreads) {
            const int rl = u / NTN, cl = u % NTN;
            const bool in = grow0 + rl < n && gcol0 + cl < n;
            xw[(rl + 1) * (SP + 2) + cl + 1] = in ? sxk[rl * SP + cl] : make_float2(0.f, 0.f);
        }
        if (tid < n_halo) xw[hrw * (SP + 2) + hcw] = hv;
    };

    int n_gemms = 0, n_updates = 0, failed = -1, cols_done = 0;
    int cur = 0;                 // xf0 or xf1 holds the current X
    bool t_ready = false;        // aT already holds the next page's Schur complement
    for (int j = p.j0; j < p.j1 && ok && failed < 0; ++j) {
        // ---- T_j (unless the last update of page j-1 formed it already) ---
        NSPROF(0);
        if (!t_ready) {
            build_T(j, [&] { window_from(cur ? p.xf1 : p.xf0); });
            NSPROF(5);
            epoch += (unsigned)nblocks;
            if (!(ok = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns))) break;
            NSPROF(6);
        }
        t_ready = false;

        float r_prev = 0.f;
        bool accepted = false;
        for (int k = 0; ok && !accepted && failed < 0; ++k) {
            // ---- R_k = I - T X_k (B layout) and its squared norm -----------
            if (!(ok = gemm(p.aT, p.bX, false))) break;
            ++n_gemms;
            double acc2 = 0.0;
            NSPROF(0);
            float2 pvs[kEpi];
            tile_values(pvs);
#pragma unroll
            for (int m = 0; m < kEpi; ++m) {
                const int it = tid + kNsThreads * m;
                if (it >= n_items) break;
                const int rl = it / NTN, cl = it % NTN;
                const int r = grow0 + rl, c = gcol0 + cl;
                float2 rv = make_float2(0.f, 0.f);
                if (r < n && c < n) {
                    const float2 pv = pvs[m];
                    rv = make_float2((r == c ? 1.f : 0.f) - pv.x, -pv.y);
                    acc2 += (double)rv.x * rv.x + (double)rv.y * rv.y;
                }
                sx[rl * SP + cl] = rv;
            }
            __syncthreads();
            write_b(p.bR, sx);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc2 += __shfl_xor_sync(0xffffffffu, acc2, o);
            if (lane == 0) s_red[warp] = acc2;
            __syncthreads();
            if (tid == 0) {
                double t = 0.0;
                for (int w = 0; w < kNsThreads / 32; ++w) t += s_red[w];
                p.rn[bid] = t;
            }
            NSPROF(7);
            epoch += (unsigned)nblocks;
            if (!(ok = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns))) break;
            NSPROF(8);
            // ---- decision (identical in every CTA: same sums, same order) ----
            {   // sum of the per-CTA norms: fixed tree, identical in every CTA
                double v = 0.0;
                for (int b2 = tid; b2 < nblocks; b2 += kNsThreads) v += __ldcg(p.rn + b2);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) s_red[warp] = v;
                __syncthreads();
            }
            if (tid == 0) {
                double t = 0.0;
                for (int w = 0; w < kNsThreads / 32; ++w) t += s_red[w];
                const float r_k = (float)sqrt(t / (double)n);
                int dec;                          // 0 accept, 1 last update, 2 update, 3 fail, 4 cubic last update
                if (!(r_k == r_k) || r_k > 1e30f) dec = 3;
                else if (r_k <= kAccept) dec = 0;
                else if (r_k <= (k == 0 ? kLastUpdateFirst : kLastUpdate)) dec = 1;
                else if (k > 0 && r_k >= r_prev) dec = 3;
                else if (r_k <= kCubicLast) dec = 4;
                else if (k > 0 && r_k > 0.3f * r_prev && r_k < kStallAccept) dec = 1;
                else if ((k == 0 && r_k > kFirstFail) || k >= p.max_iter) dec = 3;
                else dec = 2;
                s_dec[0] = dec;
                reinterpret_cast<float *>(s_dec)[1] = r_k;
            }
            __syncthreads();
            const int dec = s_dec[0];
            r_prev = reinterpret_cast<float *>(s_dec)[1];
            __syncthreads();
            if (dec == 3) {
                failed = j;
                break;
            }
            if (dec == 0) {
                // X_k stays: copy it into page j.  No barrier: nothing of the
                // next page's Schur complement writes what another CTA reads
                float2 *page = p.invT + (size_t)j * page_sz;
                write_cm(page + ny + 1, (size_t)ny, sxk);
                accepted = true;
                break;
            }
            if (dec == 4) {
                // ---- cubic last update: Y = X_k R_k (the slice into syk, its
                //      edges into xy, A layout into aT, whose T_j is no longer
                //      read), then X_{k+1} = X_k + Y + Y R_k -------------------
                if (!(ok = gemm(cur ? p.aX1 : p.aX0, p.bR, false))) break;
                ++n_gemms;
                NSPROF(0);
                {
                    float2 pv[kEpi];
                    tile_values(pv);
#pragma unroll
                    for (int m = 0; m < kEpi; ++m) {
                        const int it = tid + kNsThreads * m;
                        if (it >= n_items) break;
                        const int rl = it / NTN, cl = it % NTN;
                        const bool in = grow0 + rl < n && gcol0 + cl < n;
                        syk[rl * SP + cl] = in ? pv[m] : make_float2(0.f, 0.f);
                    }
                }
                __syncthreads();
                write_edges(p.xy, syk);
                write_a(p.aT, syk);
                NSPROF(9);
                epoch += (unsigned)nblocks;
                if (!(ok = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns))) break;
                NSPROF(10);
                if (!(ok = gemm(p.aT, p.bR, j + 1 < p.j1))) break;
                ++n_gemms;
                ++n_updates;
                NSPROF(0);
                float2 *page = p.invT + (size_t)j * page_sz;
                const float2 *xold = cur ? p.xf1 : p.xf0;
                float2 *xnew = cur ? p.xf0 : p.xf1;
                float2 pvx[kEpi];
                tile_values(pvx);
#pragma unroll
                for (int m = 0; m < kEpi; ++m) {     // X_{k+1} = X_k + Y + Y R_k, in place
                    const int it = tid + kNsThreads * m;
                    if (it >= n_items) break;
                    const int rl = it / NTN, cl = it % NTN;
                    float2 &x = sxk[rl * SP + cl];
                    const float2 y = syk[rl * SP + cl];
                    x = make_float2(x.x + y.x + pvx[m].x, x.y + y.y + pvx[m].y);
                }
                __syncthreads();
                NSPROF(12);
                write_edges(xnew, sxk);
                write_cm(page + ny + 1, (size_t)ny, sxk);
                write_a(cur ? p.aX0 : p.aX1, sxk);
                write_b(p.bX, sxk);
                NSPROF(13);
                if (j + 1 < p.j1) {
                    __syncthreads();
                    build_T(j + 1, [&] { window_after_update(xold, p.xy); });
                    t_ready = true;
                }
                NSPROF(15);
                cur ^= 1;
                NSPROF(9);
                epoch += (unsigned)nblocks;
                if (!(ok = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns))) break;
                NSPROF(10);
                accepted = true;
                break;
            }
            // ---- X_{k+1} = X_k + X_k R_k ------------------------------------
            if (!(ok = gemm(cur ? p.aX1 : p.aX0, p.bR, dec == 1 && j + 1 < p.j1))) break;
            ++n_gemms;
            ++n_updates;
            const bool last = (dec == 1);
            NSPROF(0);
            float2 *page = p.invT + (size_t)j * page_sz;
            const float2 *xold = cur ? p.xf1 : p.xf0;
            float2 *xnew = cur ? p.xf0 : p.xf1;
            float2 pvx[kEpi];
            tile_values(pvx);
#pragma unroll
            for (int m = 0; m < kEpi; ++m) {         // X_{k+1} = X_k + X_k R_k, in place
                const int it = tid + kNsThreads * m;
                if (it >= n_items) break;
                const int rl = it / NTN, cl = it % NTN;
                float2 &x = sxk[rl * SP + cl];
                x = make_float2(x.x + pvx[m].x, x.y + pvx[m].y);
            }
            __syncthreads();
            NSPROF(12);
            write_edges(xnew, sxk);
            if (last) write_cm(page + ny + 1, (size_t)ny, sxk);
            write_a(cur ? p.aX0 : p.aX1, sxk);
            write_b(p.bX, sxk);
            NSPROF(13);
            if (last && j + 1 < p.j1) {
                // the next page's Schur complement from X_{k+1} (window
                // formed without a barrier), ready at this update's barrier
                __syncthreads();
                build_T(j + 1, [&] { window_after_update(xold, nullptr); });
                t_ready = true;
            }
            NSPROF(15);
            cur ^= 1;
            NSPROF(9);
            epoch += (unsigned)nblocks;
            if (!(ok = ns_sync(p.ctr, epoch, p.err, s_ok, p.timeout_ns))) break;
            NSPROF(10);
            accepted = last;
        }
        if (accepted) ++cols_done;
    }

    if (bid == 0 && tid == 0) {
        p.status[0] = failed;
        p.status[1] = n_gemms;
        p.status[2] = n_updates;
        p.status[3] = cols_done;
    }
    // drain: every issued copy was consumed and every MMA committed (the
    // ring waits even after an expired wait), so TMEM can go.  CL: no CTA
    // leaves while another of its cluster may still read its shared memory
    // (every wait above is bounded, so all of them get here)
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, kTmemCols);
    if (CL) cluster_barrier_all();
}

// ---------------------------------------------------------------------------
// Cluster launches unless WUST_NS_CLUSTER=0 (the classic path, partials
// through L2, for comparison), or once a launch ran without its clusters.
static std::atomic<bool> g_ns_cluster_off{false};

static bool ns_cluster_enabled() {
    const char *e = std::getenv("WUST_NS_CLUSTER");
    return !(e && e[0] == '0');
}

// How many clusters of ks CTAs (one per SM) the device holds at once.
static int ns_max_clusters(int mt, int ntn, int ks) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(mt, ntn, ks);
    cfg.blockDim = dim3(kNsThreads);
    cfg.dynamicSmemBytes = kNsSmem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 1;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = ks;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, ns_factor_kernel<true>, &cfg) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return n;
}

NsGeom ns_geom(int ny, int max_ctas, bool allow_cluster) {
    NsGeom g{};
    g.n = ny - 2;
    g.mt = ceil_div(g.n, kRows);
    g.ntn = ceil_div(g.n, NTN);
    g.kc = ceil_div(g.n, kKRows);
    const int tiles = g.mt * g.ntn;
    g.ks = std::max(1, std::min(max_ctas / std::max(tiles, 1), 8));
    g.ks = std::min(g.ks, g.kc);
    if (g.ks < 3) g.ks = 0;                   // outside the epilogue bound: Gauss-Jordan only
    // the largest K split whose clusters all fit at once (a cluster's CTAs
    // share one GPC, so fewer clusters of 8 fit than 148 / 8)
    g.cluster = 0;
    if (g.ks > 0 && allow_cluster && ns_cluster_enabled()) {
        for (int ks = g.ks; ks >= 3; --ks) {
            if (ns_max_clusters(g.mt, g.ntn, ks) >= tiles) {
                g.ks = ks;
                g.cluster = 1;
                break;
            }
        }
    }
    g.per = g.ks > 0 ? ceil_div(g.kc, g.ks) : 0;
    g.a_bytes = (size_t)g.mt * g.kc * tc::kAChunk;
    g.b_bytes = (size_t)g.ntn * g.kc * kBChunkNs;
    g.part_bytes = (size_t)tiles * std::max(g.ks, 1) * 128 * NTN * sizeof(float);
    g.scratch_bytes = 3 * g.a_bytes + 2 * g.b_bytes + g.part_bytes + 3 * (size_t)g.n * g.n * sizeof(float2) +
                      (size_t)max_ctas * sizeof(double) + 256;
    return g;
}

int ns_max_ctas() {
    int dev = 0, sms = 0, per_sm = 0;
    WUST_CUDA(cudaGetDevice(&dev));
    // the attributes live in the current device's context (set every time: a
    // caller may switch devices or reset one between calls)
    WUST_CUDA(cudaFuncSetAttribute(ns_factor_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kNsSmem));
    WUST_CUDA(cudaFuncSetAttribute(ns_factor_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kNsSmem));
    WUST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    WUST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ns_factor_kernel<false>, kNsThreads, kNsSmem));
    return sms * per_sm;
}

// Launch the Newton-Schulz pages [j0, j1); returns the first page it gave
// back (or -1) and adds its GEMM/update counts to stats; *cluster_used
// (nullable) says whether it ran as clusters.
static int ns_launch(const Coefs<float2> &co, float2 *invT, const NsGeom &g, uint8_t *scratch, int j0, int j1,
                     cudaStream_t st, long long *stats, int *cluster_used) {
    NsParams p;
    p.co = co;
    p.invT = invT;
    uint8_t *q = scratch;
    p.aT = q; q += g.a_bytes;
    p.aX0 = q; q += g.a_bytes;
    p.aX1 = q; q += g.a_bytes;
    p.bX = q; q += g.b_bytes;
    p.bR = q; q += g.b_bytes;
    p.part = reinterpret_cast<float *>(q); q += g.part_bytes;
    p.xf0 = reinterpret_cast<float2 *>(q); q += (size_t)g.n * g.n * sizeof(float2);
    p.xf1 = reinterpret_cast<float2 *>(q); q += (size_t)g.n * g.n * sizeof(float2);
    p.xy = reinterpret_cast<float2 *>(q); q += (size_t)g.n * g.n * sizeof(float2);
    p.rn = reinterpret_cast<double *>(q); q += (size_t)g.mt * g.ntn * g.ks * sizeof(double);
    int *tail = reinterpret_cast<int *>(scratch + g.scratch_bytes - 256);
    p.ctr = reinterpret_cast<unsigned *>(tail);
    p.err = tail + 1;
    p.status = tail + 2;
    p.ny = co.ny;
    p.nx = co.nx;
    p.n = g.n;
    p.mt = g.mt;
    p.ntn = g.ntn;
    p.kc = g.kc;
    p.ks = g.ks;
    p.per = g.per;
    p.j0 = j0;
    p.j1 = j1;
    p.max_iter = 8;
    p.timeout_ns = 2000000000ull;
    // packed operands: padding entries must be zero (never written later)
    WUST_CUDA(cudaMemsetAsync(scratch, 0, 3 * g.a_bytes + 2 * g.b_bytes, st));
    WUST_CUDA(cudaMemsetAsync(tail, 0, 8 * sizeof(int), st));
    int h[6];
    auto read_tail = [&] {
        WUST_CUDA(cudaMemcpyAsync(h, tail, sizeof(h), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
    };
    bool launched = false;
    if (g.cluster && !g_ns_cluster_off.load()) {
        // cooperative (every CTA resident at once) and clustered (the K
        // slices of a tile in one cluster); a runtime that refuses the pair
        // gets the classic kernel on the same geometry
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g.mt, g.ntn, g.ks);
        cfg.blockDim = dim3(kNsThreads);
        cfg.dynamicSmemBytes = kNsSmem;
        cfg.stream = st;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 1;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = g.ks;
        at[1].id = cudaLaunchAttributeCooperative;
        at[1].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 2;
        if (cudaLaunchKernelEx(&cfg, ns_factor_kernel<true>, p) == cudaSuccess) {
            launched = true;
            ++g_kernel_launches;
            WUST_LAUNCH_CHECK();
            read_tail();
            if (h[1] == NS_SITE_SHAPE) {
                // the launch did not get its clusters (the kernel did nothing):
                // the classic kernel from here on in this process
                g_ns_cluster_off.store(true);
                launched = false;
                WUST_CUDA(cudaMemsetAsync(tail, 0, 8 * sizeof(int), st));
            }
        } else {
            (void)cudaGetLastError();
        }
    }
    if (cluster_used) *cluster_used = launched ? 1 : 0;
    if (!launched) {
        void *args[] = {&p};
        WUST_CUDA(cudaLaunchCooperativeKernel((void *)ns_factor_kernel<false>, dim3(g.mt, g.ntn, g.ks),
                                              dim3(kNsThreads), args, kNsSmem, st));
        ++g_kernel_launches;
        WUST_LAUNCH_CHECK();
        read_tail();
    }
    if (h[1]) fail(WUST_ERR_DEVICE_TIMEOUT, "Newton-Schulz factorization: device wait expired (site %d)", h[1]);
    if (stats) {
        stats[0] += h[3];
        stats[1] += h[4];
        stats[2] += h[5];
    }
    return h[2];
}

// Page j of invT in closed form when T_j is the identity: the Dirichlet
// columns of the operator, whose rows hold only a unit diagonal
// (ninePointCoefficients.m:33-34).  T_0 = D_0 has no predecessor; for j > 0,
// T_j = D_j - L_{j-1} X U_{j-1} = D_j when the coupling L_{j-1} is zero.  The
// kernel writes the identity page and clears ok[0] if D_j is not the
// identity (unit diagonal, zero off-diagonals) or L_{j-1} is not zero; the
// caller then inverts the page by Gauss-Jordan.
__global__ void identity_page_kernel(Coefs<float2> co, float2 *invT, int j, int *ok) {
    const int ny = co.ny;
    const size_t page_sz = (size_t)ny * ny;
    float2 *P = invT + (size_t)j * page_sz;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
    for (size_t i = tid; i < page_sz; i += nth) {
        const int r = (int)(i % ny), c = (int)(i / ny);
        P[i] = make_float2(r == c && r >= 1 && r <= ny - 2 ? 1.f : 0.f, 0.f);
    }
    auto zero = [](float2 v) { return v.x == 0.f && v.y == 0.f; };
    bool good = true;
    for (size_t y = tid; y < (size_t)ny; y += nth) {
        const int yy = (int)y;
        const float2 d = co.dd(yy, j);
        if (yy >= 1 && yy <= ny - 2 && !(d.x == 1.f && d.y == 0.f)) good = false;
        if (yy <= ny - 2 && !(zero(co.dl(yy, j)) && zero(co.du(yy, j)))) good = false;
        if (j > 0) {
            if (!zero(co.ld(yy, j - 1))) good = false;
            if (yy <= ny - 2 && !(zero(co.ll(yy, j - 1)) && zero(co.lu(yy, j - 1)))) good = false;
        }
    }
    if (!good) atomicExch(ok, 0);
}

void ns_factor(const Coefs<float2> &co, float2 *invT, const NsGeom &g, void *ns_scratch, void *gj_scratch,
               size_t gj_scratch_bytes, cudaStream_t st, long long *stats, int *head_hint, int max_ctas,
               int *cluster_used) {
    const int nx = co.nx;
    int hstat[3];
    auto gj = [&](int a, int b) {
        factor_launch(co, invT, gj_scratch, gj_scratch_bytes, st, 10.0, hstat, a, b, max_ctas);
        if (hstat[2]) fail(WUST_ERR_DEVICE_TIMEOUT, "factorization barrier timed out (site %d)", hstat[2]);
        if (hstat[0])
            fail(WUST_ERR_SINGULAR_SCHUR_BLOCK, "Schur block %d is singular (pivot %d)", hstat[0] - 1, hstat[1]);
        if (stats) stats[3] += b - a;
    };
    // the Dirichlet columns' pages in closed form (Gauss-Jordan if the check fails)
    int *ok = reinterpret_cast<int *>(static_cast<uint8_t *>(ns_scratch) + g.scratch_bytes - 256) + 8;
    auto identity = [&](int j) -> bool {
        const int one = 1;
        int h = 0;
        WUST_CUDA(cudaMemcpyAsync(ok, &one, sizeof(int), cudaMemcpyHostToDevice, st));
        identity_page_kernel<<<(int)std::min<size_t>(((size_t)co.ny * co.ny + 255) / 256, 1184), 256, 0, st>>>(
            co, invT, j, ok);
        ++g_kernel_launches;
        WUST_LAUNCH_CHECK();
        WUST_CUDA(cudaMemcpyAsync(&h, ok, sizeof(int), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        if (h && stats) stats[3] += 1;
        return h != 0;
    };
    // the first pages (Dirichlet column and the PML start) and the last one
    // (Dirichlet column) have no usable predecessor.  head_hint carries, from
    // one factorization of a solver to the next, how far past them the
    // iteration kept failing on the first page of each launch (the outer PML
    // columns of this grid): those pages join the head's Gauss-Jordan launch.
    const int base = std::min(nx, 3);
    if (g.ks <= 0 || nx <= base + 1) {
        gj(0, nx);
        return;
    }
    const int head = std::max(base, std::min(head_hint ? *head_hint : base, nx - 2));
    gj(identity(0) ? 1 : 0, head);
    int j = head, fallbacks = 0, learned = head;
    bool leading = true;                        // every launch so far failed on its first page
    while (j < nx - 1) {
        if (fallbacks >= 16) {                  // not this operator's regime: finish with Gauss-Jordan
            gj(j, nx - 1);
            j = nx - 1;
            break;
        }
        const int bad = ns_launch(co, invT, g, (uint8_t *)ns_scratch, j, nx - 1, st, stats, cluster_used);
        leading = leading && bad == j;
        if (leading) learned = bad + 1;
        if (bad < 0) {
            j = nx - 1;
        } else {
            gj(bad, bad + 1);
            ++fallbacks;
            j = bad + 1;
        }
    }
    if (head_hint) *head_hint = std::min(learned, base + 16);
    if (!identity(nx - 1)) gj(nx - 1, nx);
}

}  // namespace wust
