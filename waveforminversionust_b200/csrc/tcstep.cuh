// Column-step semantics of the block-tridiagonal sweeps shared by the
// tensor-core sweep kernels (tcsweep.cu: one group per solve, tcchunk.cu:
// one group per column chunk), and the bounded inter-CTA counter barrier.
#pragma once

#include "common.cuh"

namespace wust {

// Device-wait sites reported through *err.
enum { SITE_COPY = 1, SITE_MMA = 2, SITE_GROUP = 4, SITE_B = 5 };

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// Arrive on a monotonic counter and wait until it reaches target (bounded).
// __syncthreads on both sides; the result is uniform over the CTA and false
// when this or another CTA gave up.  Global writes made before the call are
// visible to the other CTAs' generic and async-proxy (bulk copy) reads after it.
__device__ __forceinline__ bool counter_sync(unsigned *ctr, unsigned target, int *err, int *s_ok,
                                             unsigned long long timeout_ns, int site) {
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
                    atomicCAS(err, 0, site);
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

// Column index of step i and its direction.
__device__ __forceinline__ int step_col(int i, int nx, bool &fwd) {
    fwd = i < nx - 1;
    return fwd ? 1 + i : (nx - 2) - (i - (nx - 1));
}

// B of step (fwd, j) at grid row y:  B(y) = base(y) - (wc c(y) + wm c(y-1) + wp c(y+1)),
// c = the column the step depends on (the previous step's GEMM result):
//   !ADJ fwd: c = u(:, j-1), L_{j-1}            base = SRC_j
//   !ADJ bwd: c = u(:, j+1), -U_j               base = 0
//   ADJ fwd:  c = tmp_{j-1}, U_{j-2}^H          base = SRC_{j-1}   (j == 1: B = u(:, 0) = 0)
//   ADJ bwd:  c = u(:, j+1), L_j^H              base = u(:, j)
// (applyBlockLU.cu:433-467; the ADJ forward value B is also u(:, j-1)).
// Weights that would reach outside the grid are zero.
template <bool ADJ>
__device__ __forceinline__ void step_weights(const Coefs<float2> &co, bool fwd, int j, int y, float2 &wc, float2 &wm,
                                             float2 &wp) {
    const int ny = co.ny;
    const float2 z = f2(0.f, 0.f);
    wc = z; wm = z; wp = z;
    if (!ADJ && fwd) {
        wc = co.ld(y, j - 1); wm = co.ll(y - 1, j - 1); wp = co.lu(y, j - 1);
    } else if (!ADJ) {
        const float2 a = co.ud(y, j), b = co.ul(y - 1, j), c = co.uu(y, j);
        wc = f2(-a.x, -a.y); wm = f2(-b.x, -b.y); wp = f2(-c.x, -c.y);
    } else if (fwd) {
        if (j >= 2) {
            wc = cconj(co.ud(y, j - 2));
            if (y > 0) wm = cconj(co.uu(y - 1, j - 2));
            if (y < ny - 1) wp = cconj(co.ul(y, j - 2));
        } else {
            wc = f2(-1.f, 0.f);
        }
    } else {
        wc = cconj(co.ld(y, j)); wm = cconj(co.lu(y - 1, j)); wp = cconj(co.ll(y, j));
    }
}
template <bool ADJ>
__device__ __forceinline__ float2 step_base(const SrcView &src, const float2 *u, int ny, int nx, bool fwd, int j, int y,
                                            int s) {
    if (!ADJ && fwd) return src.get(y, j, s, ny, nx);
    if (!ADJ) return f2(0.f, 0.f);
    if (fwd) return j >= 2 ? src.get(y, j - 1, s, ny, nx) : f2(0.f, 0.f);
    return __ldcg(u + (size_t)ny * nx * s + (size_t)ny * j + y);
}

}  // namespace wust
