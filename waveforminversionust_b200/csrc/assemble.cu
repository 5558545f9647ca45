// Nine-point PML Helmholtz operator assembly on the GPU, in FP64:
//   complex wavenumber and staggered PML ratios  HelmholtzSolver.m:66-90,101
//   nine coefficient arrays                      ninePointCoefficients.m:1-74
//   optional k-Wave LDR9 wavenumber              kwaveLdr9WavenumberSquared.m:11-61
// The reference builds these on the host in MATLAB and uploads nine casts
// (HelmholtzSolver.m:112-113,152-160); here one thread per grid point writes
// every coefficient owned by that point in c128 (FP64 residuals) and c64
// (factor and sweeps), plus the virtual-source multiplier C * dq/ds.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace wust {

// ---------------------------------------------------------------------------
// stencilOptParams.m:9-38 -- 1000 x 2 least squares with b = 5/6.
// Solved by modified Gram-Schmidt QR in double.
// ---------------------------------------------------------------------------
void stencil_opt_params(double vmin, double vmax, double f, double h, double g, double *b_out, double *d_out,
                        double *e_out) {
    const int na = 100, nw = 10;
    const double pi = 3.14159265358979323846;
    const double gmin = vmin / (f * h), gmax = vmax / (f * h);
    const double b = 5.0 / 6.0;
    std::vector<double> a1, a2, y;
    a1.reserve(na * nw); a2.reserve(na * nw); y.reserve(na * nw);
    for (int m = 0; m < na; ++m) {              // columns of the meshgrid (theta)
        const double th = m * pi / (4.0 * (na - 1));
        for (int n = 0; n < nw; ++n) {          // rows (G); column-major flattening
            const double G = 1.0 / (1.0 / gmax + ((double)n / (nw - 1)) * (1.0 / gmin - 1.0 / gmax));
            const double P = std::cos(g * 2 * pi * std::cos(th) / G);
            const double Q = std::cos(2 * pi * std::sin(th) / G);
            const double S1 = (1 + 1 / (g * g)) * (G * G) * (1 - P - Q + P * Q);
            const double S2 = (pi * pi) * (2 - P - Q);
            const double S3 = (2 * pi * pi) * (1 - P * Q);
            const double S4 = 2 * pi * pi + (G * G) * ((1 + 1 / (g * g)) * P * Q - P - Q / (g * g));
            a1.push_back(S2); a2.push_back(S3); y.push_back(S4 - b * S1);
        }
    }
    const size_t N = a1.size();
    double r11 = 0; for (size_t i = 0; i < N; ++i) r11 += a1[i] * a1[i];
    r11 = std::sqrt(r11);
    std::vector<double> q1(N), q2(N);
    for (size_t i = 0; i < N; ++i) q1[i] = a1[i] / r11;
    double r12 = 0; for (size_t i = 0; i < N; ++i) r12 += q1[i] * a2[i];
    for (size_t i = 0; i < N; ++i) q2[i] = a2[i] - r12 * q1[i];
    double r12b = 0; for (size_t i = 0; i < N; ++i) r12b += q1[i] * q2[i];   // re-orthogonalise
    for (size_t i = 0; i < N; ++i) q2[i] -= r12b * q1[i];
    r12 += r12b;
    double r22 = 0; for (size_t i = 0; i < N; ++i) r22 += q2[i] * q2[i];
    r22 = std::sqrt(r22);
    for (size_t i = 0; i < N; ++i) q2[i] /= r22;
    double c1 = 0, c2 = 0;
    for (size_t i = 0; i < N; ++i) { c1 += q1[i] * y[i]; c2 += q2[i] * y[i]; }
    const double e = c2 / r22;
    const double d = (c1 - r12 * e) / r11;
    *b_out = b; *d_out = d; *e_out = e;
}

struct AsmDev {
    AssemblyInput in;
    const double *vel, *atten, *exi, *eyi;
    int *status;
};

__device__ __forceinline__ double2 zdivr(double2 a, double s) { return make_double2(a.x / s, a.y / s); }

// ex/ey at staggered index (imaginary part precomputed on the host)
__device__ __forceinline__ double2 ex_at(const AsmDev &p, int i) { return make_double2(1.0, p.exi[i]); }
__device__ __forceinline__ double2 ey_at(const AsmDev &p, int i) { return make_double2(1.0, p.eyi[i]); }

__device__ __forceinline__ double2 A_at(const AsmDev &p, int y, int x) { return zdiv(ey_at(p, 2 * y), ex_at(p, 2 * x + 1)); }
__device__ __forceinline__ double2 B_at(const AsmDev &p, int y, int x) { return zdiv(ex_at(p, 2 * x), ey_at(p, 2 * y + 1)); }
__device__ __forceinline__ double2 C_at(const AsmDev &p, int y, int x) { return zmul(ex_at(p, 2 * x), ey_at(p, 2 * y)); }

// LDR9 effective q and dq/ds at one pixel (kwaveLdr9WavenumberSquared.m:11-56).
__device__ void ldr9_point(const AsmDev &p, double c, double *q_out, double *dq_out) {
    const double nodes[8] = {-0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
                             0.1834346424956498,  0.5255324099163290,  0.7966664774136267,  0.9602898564975363};
    const double wts[8] = {0.1012285362903763, 0.2223810344533745, 0.3137066458778873, 0.3626837833783620,
                           0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
    const double pi = 3.14159265358979323846;
    const double b = p.in.b, d = p.in.d, e = p.in.e, h = p.in.h, dt = p.in.dt, cr = p.in.cr;
    const double omega = 2 * pi * p.in.f;
    const double ts = sin(omega * dt / 2);
    const double z = (cr / c) * ts;
    if (!(fabs(z) < 1.0)) { atomicCAS(p.status, 0, 2); *q_out = 1; *dq_out = 0; return; }
    const double K = (2 * h / (cr * dt)) * asin(z);
    double N = 0, D = 0, Np = 0, Dp = 0;
    for (int jn = 0; jn < 8; ++jn) {
        const double th = (nodes[jn] + 1) * (pi / 8);
        const double ct = cos(th), st = sin(th);
        const double xx = K * ct, yy = K * st;
        const double cx = cos(xx), cy = cos(yy), sx = sin(xx), sy = sin(yy);
        const double lam = -4 * b + 2 * (2 * b - 1) * (cx + cy) + 4 * (1 - b) * cx * cy;
        const double mass = 1 - d - e + (d / 2) * (cx + cy) + e * cx * cy;
        const double lamp = -2 * (2 * b - 1) * (sx * ct + sy * st) - 4 * (1 - b) * (sx * ct * cy + cx * sy * st);
        const double massp = -(d / 2) * (sx * ct + sy * st) - e * (sx * ct * cy + cx * sy * st);
        const double w = 0.5 * wts[jn];
        N += w * lam * mass;
        D += w * mass * mass;
        Np += w * (lamp * mass + lam * massp);
        Dp += w * (2 * mass * massp);
    }
    const double Q = -N / D;
    const double Qp = -(Np * D - N * Dp) / (D * D);
    const double q = Q / (h * h);
    const double dKds = (2 * h * ts) / (dt * sqrt(1 - z * z));
    const double dq = (Qp / (h * h)) * dKds;
    if (!(isfinite(q) && q > 0 && isfinite(dq))) atomicCAS(p.status, 0, 3);
    *q_out = q;
    *dq_out = dq;
}

// k^2 (or q for LDR9) at a grid point
__device__ __forceinline__ double2 k2_at(const AsmDev &p, int y, int x) {
    const size_t idx = (size_t)y + (size_t)p.in.ny * x;
    const double c = p.vel[idx];
    if (p.in.ldr9) {
        double q, dq;
        ldr9_point(p, c, &q, &dq);
        const double k = sqrt(q);
        return make_double2(k * k, 0.0);
    }
    const double pi = 3.14159265358979323846;
    const double SI = p.atten ? p.atten[idx] / (2 * pi) : 0.0;
    const double2 den = make_double2(1.0 / c, SI * p.in.sgn);
    const double2 velocity = zdiv(make_double2(1.0, 0.0), den);
    const double2 k = zdiv(make_double2(2 * pi * p.in.f, 0.0), velocity);
    return zmul(k, k);
}

struct CoefTables {
    double2 *d128[9];
    float2 *d64[9];
};

__global__ void assemble_kernel(AsmDev p, CoefTables tab, double2 *mult) {
    const int ny = p.in.ny, nx = p.in.nx;
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (y >= ny || x >= nx) return;
    const double b = p.in.b, d = p.in.d, e = p.in.e;
    const double h2 = p.in.h * p.in.h, g2 = p.in.g * p.in.g;
    const double hb = (1 - b) / 2;
    const double pi = 3.14159265358979323846;
    const size_t idx = (size_t)y + (size_t)ny * x;
    {
        const double c = p.vel[idx];
        if (!(c > 0 && isfinite(c))) atomicCAS(p.status, 0, 1);
    }
    auto put = [&](int which, int ld, int yy, int xx, double2 v) {
        const size_t o = (size_t)yy + (size_t)ld * xx;
        tab.d128[which][o] = v;
        tab.d64[which][o] = c_from(v);
    };
    const double2 zero = make_double2(0.0, 0.0);
    const bool yin = (y >= 1 && y <= ny - 2), xin = (x >= 1 && x <= nx - 2);

    // Dd (:33-40)
    {
        double2 v;
        if (!yin || !xin) v = make_double2(1.0, 0.0);
        else {
            double2 sum = zadd(zadd(zadd(A_at(p, y, x), A_at(p, y, x - 1)), zdivr(B_at(p, y, x), g2)),
                               zdivr(B_at(p, y - 1, x), g2));
            double2 mass = zmul(zscale(1 - d - e, C_at(p, y, x)), k2_at(p, y, x));
            v = zsub(mass, zdivr(zscale(b, sum), h2));
        }
        put(0, ny, y, x, v);
    }
    if (y <= ny - 2) {
        // Dl (:43-45): rows 0..ny-3, x interior
        double2 v = zero;
        if (y <= ny - 3 && xin) {
            double2 t = zsub(zdivr(zscale(b, B_at(p, y, x)), g2), zscale(hb, zadd(A_at(p, y, x), A_at(p, y, x - 1))));
            v = zadd(zdivr(t, h2), zmul(zscale(d / 4, C_at(p, y, x)), k2_at(p, y, x)));
        }
        put(1, ny - 1, y, x, v);
        // Du (:46-48): rows 1..ny-2
        v = zero;
        if (yin && xin) {
            double2 t = zsub(zdivr(zscale(b, B_at(p, y, x)), g2),
                             zscale(hb, zadd(A_at(p, y + 1, x), A_at(p, y + 1, x - 1))));
            v = zadd(zdivr(t, h2), zmul(zscale(d / 4, C_at(p, y + 1, x)), k2_at(p, y + 1, x)));
        }
        put(2, ny - 1, y, x, v);
    }
    if (x <= nx - 2) {
        // Ld (:51-53): rows 1..ny-2, xl = 0..nx-3
        double2 v = zero;
        if (yin && x <= nx - 3) {
            double2 t = zsub(zscale(b, A_at(p, y, x)),
                             zscale(hb, zadd(zdivr(B_at(p, y, x), g2), zdivr(B_at(p, y - 1, x), g2))));
            v = zadd(zdivr(t, h2), zmul(zscale(d / 4, C_at(p, y, x)), k2_at(p, y, x)));
        }
        put(3, ny, y, x, v);
        // Ud (:63-65): rows 1..ny-2, xu = 1..nx-2
        v = zero;
        if (yin && x >= 1) {
            double2 t = zsub(zscale(b, A_at(p, y, x)),
                             zscale(hb, zadd(zdivr(B_at(p, y, x + 1), g2), zdivr(B_at(p, y - 1, x + 1), g2))));
            v = zadd(zdivr(t, h2), zmul(zscale(d / 4, C_at(p, y, x + 1)), k2_at(p, y, x + 1)));
        }
        put(6, ny, y, x, v);
        if (y <= ny - 2) {
            // Ll (:54-56): rows 0..ny-3
            v = zero;
            if (y <= ny - 3 && x <= nx - 3) {
                double2 t = zscale(hb, zadd(A_at(p, y, x), zdivr(B_at(p, y, x), g2)));
                v = zadd(zdivr(t, h2), zmul(zscale(e / 4, C_at(p, y, x)), k2_at(p, y, x)));
            }
            put(4, ny - 1, y, x, v);
            // Lu (:57-60): rows 1..ny-2
            v = zero;
            if (yin && x <= nx - 3) {
                double2 t = zscale(hb, zadd(A_at(p, y + 1, x), zdivr(B_at(p, y, x), g2)));
                v = zadd(zdivr(t, h2), zmul(zscale(e / 4, C_at(p, y + 1, x)), k2_at(p, y + 1, x)));
            }
            put(5, ny - 1, y, x, v);
            // Ul (:66-68): rows 0..ny-3, xu = 1..nx-2
            v = zero;
            if (y <= ny - 3 && x >= 1) {
                double2 t = zscale(hb, zadd(A_at(p, y, x), zdivr(B_at(p, y, x + 1), g2)));
                v = zadd(zdivr(t, h2), zmul(zscale(e / 4, C_at(p, y, x + 1)), k2_at(p, y, x + 1)));
            }
            put(7, ny - 1, y, x, v);
            // Uu (:69-72): rows 1..ny-2
            v = zero;
            if (yin && x >= 1) {
                double2 t = zscale(hb, zadd(A_at(p, y + 1, x), zdivr(B_at(p, y, x + 1), g2)));
                v = zadd(zdivr(t, h2), zmul(zscale(e / 4, C_at(p, y + 1, x + 1)), k2_at(p, y + 1, x + 1)));
            }
            put(8, ny - 1, y, x, v);
        }
    }
    // virtual-source multiplier C .* dq/ds (HelmholtzSolver.m:101,139,146-147)
    {
        double2 ds;
        if (p.in.ldr9) {
            double q, dq;
            ldr9_point(p, p.vel[idx], &q, &dq);
            ds = make_double2(dq, 0.0);
        } else {
            const double SI = p.atten ? p.atten[idx] / (2 * pi) : 0.0;
            const double2 den = make_double2(1.0 / p.vel[idx], SI * p.in.sgn);
            const double2 velocity = zdiv(make_double2(1.0, 0.0), den);
            ds = zdiv(make_double2(8 * pi * pi * p.in.f * p.in.f, 0.0), velocity);
        }
        mult[idx] = zmul(C_at(p, y, x), ds);
    }
}

void assemble_launch(const AssemblyInput &in, const double *vel, const double *atten, const double *ex_col,
                     const double *ey_row, double2 *const co128[9], float2 *const co64[9], double2 *mult,
                     int *status, cudaStream_t st) {
    AsmDev p;
    p.in = in;
    p.vel = vel;
    p.atten = atten;
    p.exi = ex_col;
    p.eyi = ey_row;
    p.status = status;
    CoefTables t;
    for (int i = 0; i < 9; ++i) { t.d128[i] = co128[i]; t.d64[i] = co64[i]; }
    dim3 grid(ceil_div(in.ny, 128), in.nx);
    assemble_kernel<<<grid, 128, 0, st>>>(p, t, mult);
    ++g_kernel_launches;
    WUST_LAUNCH_CHECK();
}

}  // namespace wust
