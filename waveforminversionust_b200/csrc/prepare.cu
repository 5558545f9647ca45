// The DTFT of the RF preparation, Runtime/matlab/wust_prepare.m:30-37:
//     Y(tx, rx, k) = single( sum_t exp(-2 pi i f_k t) dt * rf(t, rx, tx) )
// over the sample times t of the record, FP64 phases and accumulation, with
// the traces of inactive channels taken as zero (the reference zeroes them
// before the product, so non-finite samples there do not matter).
//
// It is one real x complex GEMM, Y^T (traces x nf) = RF^T (traces x nt) K^T,
// memory-bound on the RF stream: a block takes 64 traces, stages 32-sample
// slabs of them and of the phase matrix K (nf x nt, built once per call on
// the device) in shared memory, and every thread accumulates 2 traces x 4
// frequencies in complex double.  Frequencies beyond 32 are done in further
// passes over the traces (the block's slab stays in L2).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"

namespace wust {

constexpr int kDtTraces = 64;      // traces per block
constexpr int kDtSamples = 32;     // samples per slab
constexpr int kDtFreqs = 32;       // frequencies per pass
constexpr int kDtThreads = 256;    // 32 trace pairs x 8 frequency quads

// K(k, t) = exp(-2 pi i f_k t) * dt, arguments formed as ((-2 pi) f_k) t
__global__ void dtft_phase_kernel(const double *time_s, const double *freq, int nt, int nf, double dt, double2 *K) {
    const size_t total = (size_t)nf * nt;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(i / nt), t = (int)(i % nt);
        const double arg = (-2.0 * M_PI * freq[k]) * time_s[t];
        double s, c;
        sincos(arg, &s, &c);
        K[i] = make_double2(c * dt, s * dt);
    }
}

template <typename T>
__global__ void __launch_bounds__(kDtThreads) dtft_kernel(const T *rf, const uint8_t *active, const double2 *K, int nt,
                                                         int nf, int n_rx, int n_tx, float2 *Y, int *bad) {
    __shared__ double sp[kDtSamples][kDtTraces + 1];        // rf(t, trace)
    __shared__ double2 sk[kDtSamples][kDtFreqs];            // K(k, t)
    const int n_tr = n_rx * n_tx;
    const int tr0 = blockIdx.x * kDtTraces;
    const int k0 = blockIdx.y * kDtFreqs;
    const int tid = threadIdx.x;
    const int tp = tid & 31, fq = tid >> 5;                // traces 2 tp, 2 tp + 1; frequencies 4 fq .. 4 fq + 3
    double2 acc[2][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = make_double2(0.0, 0.0);
    int nonfinite = 0;
    for (int t0 = 0; t0 < nt; t0 += kDtSamples) {
        // rf slab: 64 traces x 32 samples, samples fastest (coalesced)
        for (int e = tid; e < kDtTraces * kDtSamples; e += kDtThreads) {
            const int ts = e % kDtSamples, tr = e / kDtSamples;
            const int t = t0 + ts, g = tr0 + tr;
            double v = 0.0;
            if (t < nt && g < n_tr && active[(g / n_rx) + (size_t)n_tx * (g % n_rx)]) {
                v = (double)rf[(size_t)t + (size_t)nt * g];
                if (!isfinite(v)) {
                    nonfinite = 1;
                    v = 0.0;
                }
            }
            sp[ts][tr] = v;
        }
        for (int e = tid; e < kDtFreqs * kDtSamples; e += kDtThreads) {
            const int ts = e % kDtSamples, kk = e / kDtSamples;
            const int t = t0 + ts, k = k0 + kk;
            sk[ts][kk] = (t < nt && k < nf) ? K[(size_t)k * nt + t] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 4
        for (int ts = 0; ts < kDtSamples; ++ts) {
            const double p0 = sp[ts][2 * tp], p1 = sp[ts][2 * tp + 1];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const double2 kv = sk[ts][4 * fq + b];
                acc[0][b].x += kv.x * p0;
                acc[0][b].y += kv.y * p0;
                acc[1][b].x += kv.x * p1;
                acc[1][b].y += kv.y * p1;
            }
        }
        __syncthreads();
    }
    if (nonfinite) atomicExch(bad, 1);
    // Y(tx, rx, k), tx fastest; trace g = rx + n_rx tx
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int g = tr0 + 2 * tp + a;
        if (g >= n_tr) continue;
        const int rx = g % n_rx, tx = g / n_rx;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int k = k0 + 4 * fq + b;
            if (k < nf)
                Y[tx + (size_t)n_tx * (rx + (size_t)n_rx * k)] = make_float2((float)acc[a][b].x, (float)acc[a][b].y);
        }
    }
}

void dtft_launch(const double *time_s, const double *freq, int nt, int nf, double dt, const void *rf, bool rf_double,
                 int n_rx, int n_tx, const uint8_t *active, double2 *K, float2 *Y, int *bad, cudaStream_t st) {
    const size_t nk = (size_t)nf * nt;
    dtft_phase_kernel<<<(int)std::min<size_t>((nk + 255) / 256, 4096), 256, 0, st>>>(time_s, freq, nt, nf, dt, K);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
    const dim3 grid(ceil_div((long long)n_rx * n_tx, kDtTraces), ceil_div(nf, kDtFreqs));
    if (rf_double)
        dtft_kernel<double><<<grid, kDtThreads, 0, st>>>(static_cast<const double *>(rf), active, K, nt, nf, n_rx,
                                                         n_tx, Y, bad);
    else
        dtft_kernel<float><<<grid, kDtThreads, 0, st>>>(static_cast<const float *>(rf), active, K, nt, nf, n_rx, n_tx,
                                                        Y, bad);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
