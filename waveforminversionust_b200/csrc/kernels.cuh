// Host-side launchers shared between the translation units of libwust_b200.
#pragma once

#include "common.cuh"

namespace wust {

// ---- factor.cu -------------------------------------------------------------
constexpr int kFactorTile = 48;
// padded interior size of a working page (multiple of the output tile)
constexpr size_t factor_pad(int ny) { return ((size_t)(ny - 2) + kFactorTile - 1) / kFactorTile * kFactorTile; }
// two ping-pong working pages + barrier/status words
constexpr size_t factor_scratch_bytes_for(int ny) { return 2 * factor_pad(ny) * factor_pad(ny) * 8 + 256; }
size_t factor_scratch_bytes(int ny);
// host_status (nullable, int[3]): {1+bad page, pivot, barrier timeout site};
// when non-null the call synchronizes the stream.  Pages [j0, j1) are
// factored (j1 < 0: through the last page); page j0 - 1 must already be in invT.
// max_ctas > 0 caps the cooperative grid (a solver confined to part of the GPU).
void factor_launch(const Coefs<float2> &co, float2 *invT, void *scratch, size_t scratch_bytes,
                   cudaStream_t stream, double timeout_s, int *host_status, int j0 = 0, int j1 = -1,
                   int max_ctas = 0);
int barrier_selftest(double timeout_s, int *site_out);

// ---- sweep.cu --------------------------------------------------------------
// u (ny*nx*S) is overwritten; tmp needs ny*S elements.
void sweep_solve(const Coefs<float2> &co, const float2 *invT, const SrcView &src, int S, bool adjoint,
                 float2 *u, float2 *tmp, cudaStream_t st);

// ---- tcsweep.cu (tensor-core sweeps, TF32 inputs) --------------------------
struct TcSweepGeom {
    int n;            // interior size ny - 2
    int mt;           // 64-row complex tiles of the interior
    int kc;           // K chunks: 16 complex interior rows (32 interleaved re/im values) each
    int ks;           // K split: CTAs sharing one output tile
    int per;          // K chunks per CTA
    int nt;           // 64-source tiles per launch (source batch = 64 nt)
    size_t page_bytes;    // packed operand bytes per page
    size_t part_bytes;    // split-K partial tiles of one launch
    size_t b_bytes;       // packed B chunks of one launch
    int sync_words;       // group counters
};
// max_ctas: CTAs that can be co-resident (cooperative launch, one per SM).
TcSweepGeom tc_sweep_geom(int ny, int S, int max_ctas);
int tc_sweep_max_ctas();
// invT pages -> packed [Ar -Ai; Ai Ar] operands of invT_j and invT_j^H
void tc_pack_invT(const float2 *invT, int ny, int nx, const TcSweepGeom &g, uint8_t *afwd, uint8_t *aadj,
                  cudaStream_t st);
// Same contract as sweep_solve: u (ny*nx*S) is overwritten.  Scratch:
// bglob (g.b_bytes), part (g.part_bytes), sync (g.sync_words); err receives
// the site of an expired device wait.
void tc_sweep_solve(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcSweepGeom &g,
                    const SrcView &src, int S, bool adjoint, float2 *u, uint8_t *bglob, float *part, unsigned *sync,
                    int *err, cudaStream_t st);

// ---- tcchunk.cu (column-chunked tensor-core sweeps, TF32 inputs) -----------
struct TcChunkGeom {
    int n, mt, kc;        // interior size, 64-row M tiles, 16-row K chunks (same packing as TcSweepGeom)
    int kc16;             // 32-row K chunks of the BF16 operands
    int C;                // column chunks per substitution
    size_t page_bytes;    // packed operand bytes per page
    size_t page_bytes16;  // BF16 packed operand bytes per page
    size_t lpack_bytes;   // packed -Lambda_c pages: 4 substitutions x C pages
    size_t lpack16_bytes; // the same, BF16
    size_t b_bytes;       // packed B chunks of C groups
    size_t state_bytes;   // C column states (re, im planes of 256 sources x ny rows)
    size_t edge_bytes;    // first and last state row of every CTA of C groups
    int sync_words;       // group counters
};
struct TcChunkBuffers {
    uint8_t *lpack, *bglob;
    uint8_t *lpack16;     // nullable: BF16 propagator pages
    float *zst, *sb;      // zero-initialised once (border rows are never written)
    float2 *edges;
    unsigned *sync;
    int *err;
};
// chunks > 0 asks for that many column chunks (clamped to what fits).
TcChunkGeom tc_chunk_geom(int ny, int nx, int max_ctas, int chunks = 0);
int tc_chunk_max_ctas();
size_t tc_chunk_state_floats(int ny);
// Composed propagators of the chunks of all four substitutions (after tc_pack_invT).
void tc_chunk_prepare(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcChunkGeom &g,
                      const TcChunkBuffers &b, cudaStream_t st);
// invT pages -> the TF32 packed operands (as tc_pack_invT) and the BF16 ones
// (as tc_pack_invT16) in one pass over the pages
void tc_pack_invT_both(const float2 *invT, int ny, int nx, const TcChunkGeom &g, uint8_t *afwd, uint8_t *aadj,
                       uint8_t *afwd16, uint8_t *aadj16, cudaStream_t st);
// invT pages -> BF16 packed operands of invT_j and invT_j^H (g.page_bytes16 per page)
void tc_pack_invT16(const float2 *invT, int ny, int nx, const TcChunkGeom &g, uint8_t *afwd16, uint8_t *aadj16,
                    cudaStream_t st);
// Same contract as tc_sweep_solve: u (ny*nx*S) is overwritten.  bf16: afwd /
// aadj are the BF16 pages and the BF16 propagators are used.
void tc_chunk_solve(const Coefs<float2> &co, const uint8_t *afwd, const uint8_t *aadj, const TcChunkGeom &g,
                    const TcChunkBuffers &b, const SrcView &src, int S, bool adjoint, float2 *u, bool bf16,
                    cudaStream_t st);

// ---- ncg.cu (NCG update, FP64) -------------------------------------------------
constexpr int kNcgMaxBlocks = 592;    // partials per reduction (<= 3 values each)
void ncg_roi_launch(const double *g, const uint8_t *mask, double *roi, size_t n, cudaStream_t st);
void ncg_mask_scale_launch(double *z, const uint8_t *mask, double scale, size_t n, cudaStream_t st);
void ncg_butterworth_launch(double2 *spec, int nx, int ny, double dx, double dy, double kc2, double order,
                            cudaStream_t st);
// the launchers below return the number of block partials written
int ncg_dot2_launch(const double *a, const double *b, const double *c, size_t n, double *part, cudaStream_t st);
int ncg_dot_launch(const double *a, const double *b, size_t n, double *part, cudaStream_t st);
int ncg_direction_launch(const double *z, const double *g, double beta, double *d, size_t n, double *part,
                         cudaStream_t st);
int ncg_project_launch(double *c, const double *d, double step, double max_update, double c_min, double c_max,
                       const uint8_t *mask, size_t n, double *part, cudaStream_t st);

// ---- prepare.cu (DTFT of the RF preparation) --------------------------------
// time_s, freq, K (nf x nt): device; rf [nt, n_rx, n_tx] float or double;
// active [n_tx, n_rx] bytes; Y [n_tx, n_rx, nf]; *bad set on a nonfinite active sample.
void dtft_launch(const double *time_s, const double *freq, int nt, int nf, double dt, const void *rf, bool rf_double,
                 int n_rx, int n_tx, const uint8_t *active, double2 *K, float2 *Y, int *bad, cudaStream_t st);

// ---- nsfactor.cu (Newton-Schulz Schur inverses, TF32 tensor cores) ---------
struct NsGeom {
    int n, mt, ntn, kc, ks, per;   // ks == 0: the grid does not fit; Gauss-Jordan only
    int cluster;                   // 1: launched as clusters of the ks K slices of a tile
    size_t a_bytes, b_bytes, part_bytes, scratch_bytes;
};
// allow_cluster: the solver has the whole device (a solver confined to a
// partition of the SMs runs the classic kernel: clusters need whole GPCs'
// worth of free SMs, which partitions running side by side need not leave).
NsGeom ns_geom(int ny, int max_ctas, bool allow_cluster);
int ns_max_ctas();
// All pages of invT: Newton-Schulz where the previous page is a good start,
// the Gauss-Jordan kernel elsewhere (gj_scratch as for factor_launch).
// stats (nullable, long long[4]): GEMMs, X updates, Newton-Schulz pages,
// Gauss-Jordan pages (accumulated).
// head_hint (in/out, may be null): the first page of the Newton-Schulz run
// (at least 3); the pages before it go to one Gauss-Jordan launch.  Updated
// from this factorization for the next one of the same solver.
// cluster_used (out, may be null): 1 if the Newton-Schulz launches ran as
// clusters, 0 if as the classic kernel; untouched without one.
void ns_factor(const Coefs<float2> &co, float2 *invT, const NsGeom &g, void *ns_scratch, void *gj_scratch,
               size_t gj_scratch_bytes, cudaStream_t st, long long *stats, int *head_hint, int max_ctas = 0,
               int *cluster_used = nullptr);

// ---- assemble.cu -----------------------------------------------------------
struct AssemblyInput {
    int ny, nx;
    double f, sgn, a0, L;
    double xmin, xmax, ymin, ymax;
    double h, g;
    double b, d, e;
    int ldr9;
    double dt, cr;
};
// vel, atten: device ny*nx (atten may be null). Outputs: 9 c128 + 9 c64
// blocks in the reference layout and the c128 virtual-source multiplier.
void assemble_launch(const AssemblyInput &in, const double *vel, const double *atten,
                     const double *ex_col, const double *ey_row,   // device, 2*(n-1)+1 imaginary parts
                     double2 *const co128[9], float2 *const co64[9], double2 *mult, int *status,
                     cudaStream_t st);
void stencil_opt_params(double vmin, double vmax, double f, double h, double g, double *b, double *d,
                        double *e);

// ---- objective.cu ----------------------------------------------------------
struct FitParams {
    const float2 *u;          // forward fields [ny, nx, nb]
    const double2 *u64;       // nullable: FP64 refined fields (gathered instead of u)
    const int32_t *rx_lin;    // 0-based
    const float2 *Y;          // [n_tx, n_rx] observations of this frequency
    const uint8_t *mask;      // [n_tx, n_rx]
    int n_tx, n_rx, first_tx, nb, ny, nx;
    float2 *residual;         // [n_rx, nb] adjoint sources (c64)
    double2 *scale;           // [nb]
    double *loss_per_src;     // [nb]
    int *status;              // [0] = 1 + first failing source
};
void fit_launch(const FitParams &p, cudaStream_t st);

// g(y,x) += sum_s -Re(conj(scale_s * mult * u_s) * (M^T lam_s))   (wust_oracle.m:66-68)
void gradient_launch(const float2 *u, const float2 *lam, const double2 *mult, const double2 *scale, int ny,
                     int nx, int nb, double d, double e, double *grad, cudaStream_t st);
// out = massApply(v, adjoint) for plain fields (HelmholtzSolver.m:205-220)
void mass_apply_launch(const float2 *v, float2 *out, int ny, int nx, int n, double d, double e, bool adjoint,
                       cudaStream_t st);
// out = massApply(mult .* u .* direction, false): curvature sources
void curvature_source_launch(const float2 *u, const double2 *mult, const double *direction, float2 *out, int ny,
                             int nx, int nb, double d, double e, cudaStream_t st);
// per-source sum |u(rx) * scale * mask|^2 -> out[nb]
void curvature_reduce_launch(const float2 *u, const int32_t *rx_lin, const uint8_t *mask, const double2 *scale,
                             int n_tx, int n_rx, int first_tx, int nb, int ny, int nx, double *out,
                             cudaStream_t st);
// q(r, s) = -a_s u_s(rx_r) on unmasked receivers (zero elsewhere) into
// resid[r + n_rx s], the linearized residual J d of the Gauss-Newton
// product, and sum_r |q|^2 per source into out[s]
void linearized_residual_launch(const float2 *u, const int32_t *rx_lin, const uint8_t *mask, const double2 *scale,
                                int n_tx, int n_rx, int first_tx, int nb, int ny, int nx, float2 *resid, double *out,
                                cudaStream_t st);
// virt = mult .* u
void virtual_source_launch(const float2 *u, const double2 *mult, float2 *virt, int ny, int nx, int n,
                           cudaStream_t st);

// ---- refine.cu -------------------------------------------------------------
// Interleaved nine-point weights [x][y][9] of H (w9f) and H^H (w9a), complex128.
struct RefineWeights {
    const double2 *w9f, *w9a;
    int ny, nx;
};
void refine_weights_launch(const Coefs<double2> &co, double2 *w9f, double2 *w9a, cudaStream_t st);
// First refinement step: r = b - H u (or H^H) on rows y in [1, ny-2], zero on
// rows 0 and ny-1, as c64 for the correction solve; per-source squared
// interior norms of r and (if bnorm2) of b.
void refine_first_launch(const RefineWeights &w, const SrcView &b, const float2 *u, int S, bool adjoint,
                         float2 *r32, double *rnorm2, double *bnorm2, cudaStream_t st);
// Later steps: x_new = x_old + d in FP64 and r = b - H x_new, with norms of r,
// d and x_new.  The first correction passes the solve's c64 field as x_old32
// and no out; later ones pass the FP64 iterate as x_old and get its c64 copy
// in out.  x_new must differ from x_old.
void refine_step_launch(const RefineWeights &w, const SrcView &b, const float2 *d, const float2 *x_old32,
                        const double2 *x_old, int S, bool adjoint, double2 *x_new, float2 *out, float2 *r32,
                        double *rnorm2, double *dnorm2, double *xnorm2, cudaStream_t st);
// u = c64(x)
void refine_demote_launch(const double2 *x, float2 *u, size_t n, cudaStream_t st);


// RF simulation (simulate.cu): host inputs, device output rf [ly][nrx][ntx]
// column-major (ly = ceil(nt / decimation)).
struct SimulateArgs {
    const double *c;          // [ny][nx] column-major sound speed (m/s)
    int ny, nx;
    double dy, dx, dt;        // grid spacing (m) along y (first axis) and x, time step (s)
    int nt;
    const double *source;     // [nt] Dirichlet source pressure
    const int *tx_index;      // [ntx] 1-based column-major
    int ntx;
    const int *rx_index;      // [nrx]
    int nrx;
    int pml;                  // PML cells outside the grid on every side
    double c_ref, rho0;
    int decimation;           // >= 1
    int tx_batch;             // transmitters per batch (0: all)
};
void simulate_rf(const SimulateArgs &a, float *rf, cudaStream_t st);

}  // namespace wust
