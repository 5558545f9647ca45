"""FP64 CPU oracle for the WUST Helmholtz gradient path.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package imports this module;
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker or
the timed CPU baseline.

What it is: a NumPy/SciPy restatement, in float64/complex128, of the
reference's Helmholtz path (WaveformInversionUST, MATLAB + MEX):

* ``stencil_opt_params``        Runtime/solver/stencilOptParams.m:1-38
* ``pml_fields``                Runtime/solver/HelmholtzSolver.m:56-101
* ``nine_point_coefficients``   Runtime/solver/ninePointCoefficients.m:1-74
* ``assemble_sparse``           Runtime/solver/HelmholtzSolver.m:114-138
* ``HelmholtzSolverFP64``       Runtime/solver/HelmholtzSolver.m:32-220 (cpu backend:
                                sparse LU, SciPy ``splu`` stands in for MATLAB
                                ``decomposition(H,'lu')``)
* ``block_lu_factor`` / ``block_lu_apply``
                                Runtime/solver/decompBlockLU.cu:337-368 and
                                Runtime/solver/applyBlockLU.cu:433-467 restated in
                                complex128 (same recursion and sweeps, any dtype)
* ``wust_oracle``               Runtime/matlab/wust_oracle.m:1-86
* ``directional_curvature``     Runtime/matlab/directional_curvature.m:1-26
* ``gauss_newton_product``      Re(J^H J d): the product behind directional_curvature.m's
                                quadratic form (its J d, wust_oracle.m:62-68's J^H)
* NCG scalars                   Runtime/matlab/wust_ncg_direction.m, linearized_step_length.m,
                                wust_roi_gradient.m, wust_project_slowness_update.m
* ``ringing_removal_filt``      Runtime/solver/ringingRemovalFilt.m:1-45
* ``kwave_ldr9``                Runtime/solver/kwaveLdr9WavenumberSquared.m:1-73
* ``geometry``                  Runtime/matlab/wust_geometry.m:1-31

Parity status: PARTIALLY PINNED.  The reference is MATLAB (+ MEX needing
MATLAB's mxGPUArray runtime) and cannot run in this environment, and it ships
no golden vectors.  The oracle is pinned by the reference's own known-answer
and property tests (Runtime/tests/test_runtime.m): exact NCG/projection values
(beta = 4/3, gz = 4, projected 1512 m/s), ringingRemovalFilt(cutoff=0) as the
identity, central finite difference vs adjoint gradient (< 1e-4 in FP64),
loss-only vs loss+gradient equality, batch invariance (< 1e-4), and descent
of the 4-update reconstruction.  Values at the LU boundary are otherwise
unpinned; the block-LU restatement is cross-checked against the sparse LU.

Array conventions follow MATLAB: 2-D fields are ``(Ny, Nx)`` arrays indexed
``[y, x]``; RHS stacks are ``(Ny, Nx, S)``; linear grid indices are 1-based
column-major (``y + Ny * (x - 1)``), as produced by ``sub2ind``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class WustError(RuntimeError):
    """Error carrying a MATLAB-style identifier (``WUST:InvalidInput`` ...)."""

    def __init__(self, identifier: str, message: str):
        super().__init__(f"{identifier}: {message}")
        self.identifier = identifier


# ---------------------------------------------------------------------------
# Stencil parameters and PML (HelmholtzSolver.m:53-101, stencilOptParams.m)
# ---------------------------------------------------------------------------

def stencil_opt_params(vmin: float, vmax: float, f: float, h: float, g: float):
    """Optimal nine-point mass weights, stencilOptParams.m:9-38.

    b is fixed at 5/6 (:32); d, e solve the 1000x2 least-squares problem (:35).
    """
    angle_samples, wavelength_samples = 100, 10
    gmin = vmin / (f * h)
    gmax = vmax / (f * h)
    m = np.arange(1, angle_samples + 1)
    n = np.arange(1, wavelength_samples + 1)
    theta = (m - 1) * np.pi / (4 * (angle_samples - 1))
    G = 1.0 / (1.0 / gmax + ((n - 1) / (wavelength_samples - 1)) * (1.0 / gmin - 1.0 / gmax))
    TH, GG = np.meshgrid(theta, G)            # (10, 100) like MATLAB meshgrid
    P = np.cos(g * 2 * np.pi * np.cos(TH) / GG)
    Q = np.cos(2 * np.pi * np.sin(TH) / GG)
    S1 = (1 + 1 / g**2) * GG**2 * (1 - P - Q + P * Q)
    S2 = np.pi**2 * (2 - P - Q)
    S3 = (2 * np.pi**2) * (1 - P * Q)
    S4 = 2 * np.pi**2 + GG**2 * ((1 + 1 / g**2) * P * Q - P - Q / g**2)
    b = 5.0 / 6.0
    A = np.stack([S2.ravel(order="F"), S3.ravel(order="F")], axis=1)
    y = S4.ravel(order="F") - b * S1.ravel(order="F")
    params, *_ = np.linalg.lstsq(A, y, rcond=None)
    return b, float(params[0]), float(params[1])


def _matlab_linspace(a: float, b: float, n: int) -> np.ndarray:
    return np.linspace(a, b, n)


@dataclass
class PmlFields:
    A: np.ndarray        # (Ny, Nx-1) complex128
    B: np.ndarray        # (Ny-1, Nx) complex128
    C: np.ndarray        # (Ny, Nx) complex128
    k: np.ndarray        # (Ny, Nx) complex128 wavenumber
    dslow: np.ndarray    # (Ny, Nx) complex128, 8 pi^2 f^2 / velocity
    h: float
    g: float


def pml_fields(x, y, vel, atten, f, sign_convention, a0, L_pml) -> PmlFields:
    """Complex wavenumber and staggered PML ratios, HelmholtzSolver.m:56-101."""
    x = np.asarray(x, dtype=np.float64).ravel()
    y = np.asarray(y, dtype=np.float64).ravel()
    vel = np.asarray(vel, dtype=np.float64)
    atten = np.asarray(atten, dtype=np.float64)
    h = float(np.mean(np.diff(x)))
    gh = float(np.mean(np.diff(y)))
    g = gh / h
    xmin, xmax, ymin, ymax = x.min(), x.max(), y.min(), y.max()
    Nx, Ny = x.size, y.size
    sgn = float(np.sign(sign_convention))
    SI = atten / (2 * np.pi)
    velocity = 1.0 / (1.0 / vel + 1j * SI * sgn)
    k = 2 * np.pi * f / velocity
    xe = _matlab_linspace(xmin, xmax, 2 * (Nx - 1) + 1)
    ye = _matlab_linspace(ymin, ymax, 2 * (Ny - 1) + 1)
    Xe, Ye = np.meshgrid(xe, ye)
    xctr, xspan = (xmin + xmax) / 2, (xmax - xmin) / 2
    yctr, yspan = (ymin + ymax) / 2, (ymax - ymin) / 2
    sx = 2 * np.pi * a0 * f * (np.maximum(np.abs(Xe - xctr) - xspan + L_pml, 0) / L_pml) ** 2
    sy = 2 * np.pi * a0 * f * (np.maximum(np.abs(Ye - yctr) - yspan + L_pml, 0) / L_pml) ** 2
    ex = 1 + 1j * sx * sgn / (2 * np.pi * f)
    ey = 1 + 1j * sy * sgn / (2 * np.pi * f)
    A = (ey / ex)[0::2, 1::2]
    B = (ex / ey)[1::2, 0::2]
    C = (ex * ey)[0::2, 0::2]
    dslow = 8 * np.pi**2 * f**2 / velocity
    return PmlFields(A=A, B=B, C=C, k=k.astype(np.complex128), dslow=dslow.astype(np.complex128), h=h, g=g)


# ---------------------------------------------------------------------------
# Nine-point coefficients (ninePointCoefficients.m:1-74), 0-based restatement
# ---------------------------------------------------------------------------

COEF_NAMES = ("Dd", "Dl", "Du", "Ld", "Ll", "Lu", "Ud", "Ul", "Uu")


def nine_point_coefficients(A, B, C, k, b, d, e, h, g, Nx, Ny, q=None):
    """The nine coefficient arrays of H = K + M_mass diag(C q).

    ``q`` defaults to k**2 (continuum); the LDR9 option passes q directly
    (HelmholtzSolver.m:102-110 sets k = sqrt(q), so k.*k == q up to rounding).
    """
    k2 = (k * k) if q is None else np.asarray(q, dtype=np.complex128)
    h2 = h * h
    g2 = g * g
    Dd = np.zeros((Ny, Nx), np.complex128)
    Dl = np.zeros((Ny - 1, Nx), np.complex128)
    Du = np.zeros((Ny - 1, Nx), np.complex128)
    Ld = np.zeros((Ny, Nx - 1), np.complex128)
    Ll = np.zeros((Ny - 1, Nx - 1), np.complex128)
    Lu = np.zeros((Ny - 1, Nx - 1), np.complex128)
    Ud = np.zeros((Ny, Nx - 1), np.complex128)
    Ul = np.zeros((Ny - 1, Nx - 1), np.complex128)
    Uu = np.zeros((Ny - 1, Nx - 1), np.complex128)
    # Dirichlet rows (:33-34)
    Dd[[0, Ny - 1], :] = 1
    Dd[1:Ny - 1, [0, Nx - 1]] = 1
    y = slice(1, Ny - 1)          # interior rows 1..Ny-2
    ym = slice(0, Ny - 2)         # y-1
    yp = slice(2, Ny)             # y+1
    x = slice(1, Nx - 1)          # interior columns
    xm = slice(0, Nx - 2)         # x-1
    r0 = slice(0, Ny - 2)         # MATLAB 1:Ny-2
    # Dd (:38-40)
    Dd[y, x] = ((1 - d - e) * C[y, x] * k2[y, x]
                - b * (A[y, x] + A[y, xm] + B[y, x] / g2 + B[ym, x] / g2) / h2)
    # Dl, Du (:43-48)
    Dl[r0, x] = ((b * B[r0, x] / g2 - ((1 - b) / 2) * (A[r0, x] + A[r0, xm])) / h2
                 + (d / 4) * C[r0, x] * k2[r0, x])
    Du[y, x] = ((b * B[y, x] / g2 - ((1 - b) / 2) * (A[yp, x] + A[yp, xm])) / h2
                + (d / 4) * C[yp, x] * k2[yp, x])
    # Lower block (:51-60): rows in x+1, columns in x, xl = 0..Nx-3
    xl = slice(0, Nx - 2)
    Ld[y, xl] = ((b * A[y, xl] - ((1 - b) / 2) * (B[y, xl] / g2 + B[ym, xl] / g2)) / h2
                 + (d / 4) * C[y, xl] * k2[y, xl])
    Ll[r0, xl] = (((1 - b) / 2) * (A[r0, xl] + B[r0, xl] / g2) / h2
                  + (e / 4) * C[r0, xl] * k2[r0, xl])
    Lu[y, xl] = (((1 - b) / 2) * (A[yp, xl] + B[y, xl] / g2) / h2
                 + (e / 4) * C[yp, xl] * k2[yp, xl])
    # Upper block (:63-72): rows in x, columns in x+1, xu = 1..Nx-2
    xu = slice(1, Nx - 1)
    xu1 = slice(2, Nx)
    Ud[y, xu] = ((b * A[y, xu] - ((1 - b) / 2) * (B[y, xu1] / g2 + B[ym, xu1] / g2)) / h2
                 + (d / 4) * C[y, xu1] * k2[y, xu1])
    Ul[r0, xu] = (((1 - b) / 2) * (A[r0, xu] + B[r0, xu1] / g2) / h2
                  + (e / 4) * C[r0, xu1] * k2[r0, xu1])
    Uu[y, xu] = (((1 - b) / 2) * (A[yp, xu] + B[y, xu1] / g2) / h2
                 + (e / 4) * C[yp, xu1] * k2[yp, xu1])
    return dict(Dd=Dd, Dl=Dl, Du=Du, Ld=Ld, Ll=Ll, Lu=Lu, Ud=Ud, Ul=Ul, Uu=Uu)


def assemble_sparse(coefs, Ny, Nx) -> sp.csc_matrix:
    """9-point CSC matrix with identity Dirichlet rows, HelmholtzSolver.m:114-138."""
    N = Ny * Nx
    yy, xx = np.meshgrid(np.arange(Ny), np.arange(Nx), indexing="ij")
    lin = yy + Ny * xx                      # 0-based column-major
    interior = (yy > 0) & (yy < Ny - 1) & (xx > 0) & (xx < Nx - 1)
    rows, cols, vals = [], [], []
    b_idx = lin[~interior]
    rows.append(b_idx); cols.append(b_idx); vals.append(np.ones(b_idx.size, np.complex128))
    iy, ix = yy[interior], xx[interior]
    row = lin[interior]
    c = coefs
    entries = [
        (0, c["Dd"][iy, ix]),
        (-1, c["Dl"][iy - 1, ix]),
        (+1, c["Du"][iy, ix]),
        (-Ny, c["Ld"][iy, ix - 1]),
        (-Ny - 1, c["Ll"][iy - 1, ix - 1]),
        (-Ny + 1, c["Lu"][iy, ix - 1]),
        (+Ny, c["Ud"][iy, ix]),
        (+Ny - 1, c["Ul"][iy - 1, ix]),
        (+Ny + 1, c["Uu"][iy, ix]),
    ]
    for off, val in entries:
        rows.append(row); cols.append(row + off); vals.append(val)
    rows = np.concatenate(rows); cols = np.concatenate(cols); vals = np.concatenate(vals)
    return sp.csc_matrix((vals, (rows, cols)), shape=(N, N))


# ---------------------------------------------------------------------------
# Mass stencil (HelmholtzSolver.m:205-220)
# ---------------------------------------------------------------------------

def mass_kernel(d: float, e: float) -> np.ndarray:
    return np.array([[e / 4, d / 4, e / 4], [d / 4, 1 - d - e, d / 4], [e / 4, d / 4, e / 4]])


def _conv_same_3x3(v: np.ndarray, ker: np.ndarray) -> np.ndarray:
    """convn(v, ker, 'same') over the first two axes with zero padding."""
    Ny, Nx = v.shape[:2]
    pad = np.zeros((Ny + 2, Nx + 2) + v.shape[2:], dtype=np.result_type(v, ker))
    pad[1:-1, 1:-1] = v
    out = np.zeros_like(pad[1:-1, 1:-1])
    # convolution flips the kernel; the mass kernel is symmetric so this is exact
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            w = ker[1 - dy, 1 - dx]
            out += w * pad[1 + dy:1 + dy + Ny, 1 + dx:1 + dx + Nx]
    return out


def mass_apply(v: np.ndarray, d: float, e: float, adjoint: bool) -> np.ndarray:
    """massApply: forward zeroes the ring after the convolution, adjoint before."""
    v = np.array(v, copy=True)
    if adjoint:
        v[[0, -1], ...] = 0
        v[:, [0, -1], ...] = 0
    out = _conv_same_3x3(v, mass_kernel(d, e))
    if not adjoint:
        out[[0, -1], ...] = 0
        out[:, [0, -1], ...] = 0
    return out


# ---------------------------------------------------------------------------
# LDR9 wavenumber (kwaveLdr9WavenumberSquared.m) -- optional continuum alternative
# ---------------------------------------------------------------------------

_GL8_NODES = np.array([-0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
                       0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363])
_GL8_WEIGHTS = 0.5 * np.array([0.1012285362903763, 0.2223810344533745, 0.3137066458778873, 0.3626837833783620,
                               0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763])


def kwave_ldr9(c, f, h, b, d, e, dt, cr):
    """q_eff and dq/ds, kwaveLdr9WavenumberSquared.m:11-61 (8-node Gauss-Legendre)."""
    c = np.asarray(c, np.float64)
    omega = 2 * np.pi * f
    ts = np.sin(omega * dt / 2)
    z = (cr / c) * ts
    if np.any(np.abs(z) >= 1):
        raise WustError("WUST:InvalidInput", "k-Wave local dispersion target is evanescent")
    K = (2 * h / (cr * dt)) * np.arcsin(z)
    theta = (_GL8_NODES + 1) * (np.pi / 8)
    N = np.zeros_like(K); D = np.zeros_like(K); Np_ = np.zeros_like(K); Dp = np.zeros_like(K)
    for th, w in zip(theta, _GL8_WEIGHTS):
        ct, st = np.cos(th), np.sin(th)
        xx, yy = K * ct, K * st
        cx, cy, sx, sy = np.cos(xx), np.cos(yy), np.sin(xx), np.sin(yy)
        lam = -4 * b + 2 * (2 * b - 1) * (cx + cy) + 4 * (1 - b) * cx * cy
        mass = 1 - d - e + (d / 2) * (cx + cy) + e * cx * cy
        lamp = -2 * (2 * b - 1) * (sx * ct + sy * st) - 4 * (1 - b) * (sx * ct * cy + cx * sy * st)
        massp = -(d / 2) * (sx * ct + sy * st) - e * (sx * ct * cy + cx * sy * st)
        N += w * lam * mass
        D += w * mass * mass
        Np_ += w * (lamp * mass + lam * massp)
        Dp += w * (2 * mass * massp)
    Q = -N / D
    Qp = -(Np_ * D - N * Dp) / (D * D)
    q = Q / (h * h)
    dKds = (2 * h * ts) / (dt * np.sqrt(1 - z * z))
    dq = (Qp / (h * h)) * dKds
    if np.any(~np.isfinite(q) | (q <= 0)) or np.any(~np.isfinite(dq)):
        raise WustError("WUST:NumericalFailure", "LDR-9 produced invalid wavenumber or derivative")
    return q, dq


# ---------------------------------------------------------------------------
# Block LU restatement (decompBlockLU.cu:337-368, applyBlockLU.cu:433-467)
# ---------------------------------------------------------------------------

def _tri(dg, lo, up):
    return np.diag(dg) + np.diag(lo, -1) + np.diag(up, 1)


def block_lu_factor(coefs, dtype=np.complex128, invert=None):
    """invT[:, :, j] = inv(T_j interior) with T_{j+1} = D_{j+1} - L_j invT_j U_j.

    Border rows/columns of every page stay zero (decompBlockLU.cu:337-368).
    ``invert`` may replace ``np.linalg.inv`` (used to emulate reduced precision).
    """
    c = {k: np.asarray(v, dtype) for k, v in coefs.items()}
    Ny, Nx = c["Dd"].shape
    inv = invert or np.linalg.inv
    invT = np.zeros((Ny, Ny, Nx), dtype)
    T = _tri(c["Dd"][:, 0], c["Dl"][:, 0], c["Du"][:, 0])
    for j in range(1, Nx + 1):
        invT[1:-1, 1:-1, j - 1] = inv(T[1:-1, 1:-1])
        if j == Nx:
            break
        D = _tri(c["Dd"][:, j], c["Dl"][:, j], c["Du"][:, j])
        L = _tri(c["Ld"][:, j - 1], c["Ll"][:, j - 1], c["Lu"][:, j - 1])
        U = _tri(c["Ud"][:, j - 1], c["Ul"][:, j - 1], c["Uu"][:, j - 1])
        T = D - L @ invT[:, :, j - 1] @ U
    return invT


def block_lu_apply(src, coefs, invT, adjoint: bool):
    """Forward or adjoint block-tridiagonal sweeps of applyBlockLU.cu:433-467.

    ``src`` is (Ny, Nx, S).  u starts at zero (applyBlockLU.cu:404-409).
    """
    dtype = invT.dtype
    c = {k: np.asarray(v, dtype) for k, v in coefs.items()}
    src = np.asarray(src, dtype)
    if src.ndim == 2:
        src = src[:, :, None]
    Ny, Nx, S = src.shape
    u = np.zeros_like(src)

    def Lm(j):
        return _tri(c["Ld"][:, j], c["Ll"][:, j], c["Lu"][:, j])

    def Um(j):
        return _tri(c["Ud"][:, j], c["Ul"][:, j], c["Uu"][:, j])

    if adjoint:
        for j in range(1, Nx):
            tmp = invT[:, :, j - 1].conj().T @ u[:, j - 1, :]
            u[:, j, :] = src[:, j, :] - Um(j - 1).conj().T @ tmp
        for j in range(Nx - 2, -1, -1):
            tmp = u[:, j, :] - Lm(j).conj().T @ u[:, j + 1, :]
            u[:, j, :] = invT[:, :, j].conj().T @ tmp
    else:
        for j in range(1, Nx):
            tmp = src[:, j, :] - Lm(j - 1) @ u[:, j - 1, :]
            u[:, j, :] = invT[:, :, j] @ tmp
        for j in range(Nx - 2, -1, -1):
            tmp = Um(j) @ u[:, j + 1, :]
            u[:, j, :] = u[:, j, :] - invT[:, :, j] @ tmp
    return u


# ---------------------------------------------------------------------------
# HelmholtzSolver (cpu backend)
# ---------------------------------------------------------------------------

@dataclass
class SolverOptions:
    stencil_bounds: tuple
    dispersion: dict | None = None


class HelmholtzSolverFP64:
    """HelmholtzSolver.m with backend='cpu': sparse complex128 LU of the 9-point operator."""

    def __init__(self, x, y, vel, atten, f, sign_convention, a0, L_pml, options, factor=True):
        if options is None or "stencil_bounds" not in options or "backend" not in options:
            raise WustError("WUST:InvalidInput", "Explicit backend and fixed stencil_bounds are required")
        bounds = options["stencil_bounds"]
        if (bounds is None or np.size(bounds) != 2 or not np.all(np.isfinite(bounds))
                or bounds[0] <= 0 or bounds[1] <= bounds[0]):
            raise WustError("WUST:InvalidInput", "stencil_bounds must be a positive ordered [min,max] pair")
        vel = np.asarray(vel, np.float64)
        x = np.asarray(x, np.float64).ravel(); y = np.asarray(y, np.float64).ravel()
        if vel.shape != (y.size, x.size) or min(vel.shape) < 3 or np.any(~np.isfinite(vel)) or np.any(vel <= 0):
            raise WustError("WUST:InvalidInput", "Expected a positive finite [ny,nx] medium")
        self.Ny, self.Nx = vel.shape
        pf = pml_fields(x, y, vel, atten, f, sign_convention, a0, L_pml)
        b, d, e = stencil_opt_params(float(bounds[0]), float(bounds[1]), f, pf.h, pf.g)
        self.b, self.d, self.e = b, d, e
        q = None
        dslow = pf.dslow
        disp = options.get("dispersion")
        if disp:
            q, dq = kwave_ldr9(vel, f, pf.h, b, d, e, disp["time_step_s"], disp["reference_speed_mps"])
            dslow = dq.astype(np.complex128)
            k = np.sqrt(q.astype(np.complex128))
        else:
            k = pf.k
        self.k = k
        self.pml = pf
        self.coefs = nine_point_coefficients(pf.A, pf.B, pf.C, k, b, d, e, pf.h, pf.g, self.Nx, self.Ny,
                                             q=None if q is None else (k * k))
        self.virtual_source_multiplier = pf.C * dslow
        self.H = assemble_sparse(self.coefs, self.Ny, self.Nx)
        self.lu = spla.splu(self.H) if factor else None

    def solve(self, src, adjoint=False, want_virtual=False):
        src = np.asarray(src, np.complex128)
        squeeze = src.ndim == 2
        if squeeze:
            src = src[:, :, None]
        Ny, Nx, S = src.shape
        rhs = src.reshape(Ny * Nx, S, order="F")
        sol = self.lu.solve(rhs, trans="H" if adjoint else "N")
        u = sol.reshape(Ny, Nx, S, order="F")
        if squeeze:
            u = u[:, :, 0]
        if want_virtual:
            mult = self.virtual_source_multiplier
            v = u * (mult if u.ndim == 2 else mult[:, :, None])
            return u, v
        return u

    def mass_apply(self, v, adjoint):
        return mass_apply(v, self.d, self.e, adjoint)


# ---------------------------------------------------------------------------
# Geometry (wust_geometry.m) and observations
# ---------------------------------------------------------------------------

def grid_centres(shape_yx, origin_yx, spacing_yx):
    ny, nx = shape_yx
    y = origin_yx[0] + (np.arange(ny) + 0.5) * spacing_yx[0]
    x = origin_yx[1] + (np.arange(nx) + 0.5) * spacing_yx[1]
    return x, y


def snap(xy, x, y):
    """Nearest-sample snapping; ties take the first index (wust_geometry.m:20-31).

    Returns 1-based column-major linear indices.
    """
    xy = np.asarray(xy, np.float64)
    if xy.ndim != 2 or xy.shape[1] != 2 or xy.shape[0] == 0 or not np.all(np.isfinite(xy)):
        raise WustError("WUST:InvalidInput", "Positions must be finite [N,2] physical [x,y]")
    if not np.all((xy[:, 0] >= x[0]) & (xy[:, 0] <= x[-1]) & (xy[:, 1] >= y[0]) & (xy[:, 1] <= y[-1])):
        raise WustError("WUST:InvalidInput", "Array outside grid sampling coordinates")
    ix = np.argmin(np.abs(x[:, None] - xy[None, :, 0]), axis=0)   # first minimum on ties
    iy = np.argmin(np.abs(y[:, None] - xy[None, :, 1]), axis=0)
    index = (iy + 1) + y.size * ix
    if np.unique(index).size != index.size:
        raise WustError("WUST:InvalidInput", "Distinct elements in one array collapse onto a grid sample")
    return index.astype(np.int64)


@dataclass
class Observations:
    """The subset of wust.measurements the oracle consumes (wust_prepare_observations.m:69-80)."""
    x_m: np.ndarray
    y_m: np.ndarray
    tx_index: np.ndarray          # 1-based linear indices
    rx_index: np.ndarray
    frequencies_hz: np.ndarray
    Y: np.ndarray                 # (n_tx, n_rx, n_f) complex
    mask: np.ndarray              # (n_tx, n_rx, n_f) bool
    shape_yx: tuple = field(default=None)

    def __post_init__(self):
        if self.shape_yx is None:
            self.shape_yx = (self.y_m.size, self.x_m.size)
        self.Y = np.where(self.mask, self.Y, 0)

    @property
    def n_tx(self):
        return self.tx_index.size

    @property
    def frequency_data_norm(self):
        return np.sum(np.abs(self.Y.astype(np.complex128)) ** 2, axis=(0, 1))


@dataclass
class OracleConfig:
    pml_m: float
    pml_strength: float = 10.0
    stencil_bounds: tuple = (1400.0, 1700.0)
    source_batch_size: int = 10**9
    wavenumber: str = "continuum"
    dispersion: dict | None = None
    backend: str = "cpu"


def point_sources(tx_index, ids, ny, nx, dtype=np.complex128):
    src = np.zeros((ny, nx, len(ids)), dtype)
    flat = src.reshape(ny * nx, len(ids), order="F")
    for j, t in enumerate(ids):
        flat[tx_index[t] - 1, j] = 1
    return flat.reshape(ny, nx, len(ids), order="F")


# ---------------------------------------------------------------------------
# wust_oracle / directional_curvature (wust_oracle.m, directional_curvature.m)
# ---------------------------------------------------------------------------

def make_solver(c, obs: Observations, fi: int, cfg: OracleConfig, factor=True):
    ny, nx = obs.shape_yx
    disp = cfg.dispersion if cfg.wavenumber == "kwave-ldr9" else None
    return HelmholtzSolverFP64(obs.x_m, obs.y_m, np.asarray(c, np.float64), np.zeros((ny, nx)),
                               float(obs.frequencies_hz[fi]), -1, cfg.pml_strength, cfg.pml_m,
                               dict(backend="cpu", stencil_bounds=cfg.stencil_bounds, dispersion=disp),
                               factor=factor)


def wust_oracle(c, obs: Observations, fi: int, cfg: OracleConfig, need_gradient=True, retain_state=False,
                solver=None):
    """Source-projected least squares at one frequency, wust_oracle.m:1-86.

    Returns (loss, gradient or None, cache or None).  ``fi`` is 0-based.
    """
    ny, nx = obs.shape_yx
    nt = obs.n_tx
    if solver is None:
        solver = make_solver(c, obs, fi, cfg)
    gradient = np.zeros((ny, nx)) if need_gradient else None
    loss = 0.0
    virtual, scales, fields = [], [], []
    rx0 = obs.rx_index - 1
    for first in range(0, nt, cfg.source_batch_size):
        ids = list(range(first, min(first + cfg.source_batch_size, nt)))
        nb = len(ids)
        source = point_sources(obs.tx_index, ids, ny, nx)
        u, v = solver.solve(source, adjoint=False, want_virtual=True)
        uf = u.reshape(ny * nx, nb, order="F")
        predicted = uf[rx0, :]
        mask = obs.mask[ids, :, fi].T.astype(np.float64)
        observed = obs.Y[ids, :, fi].T.astype(np.complex128)
        predicted = predicted * mask
        observed = observed * mask
        den = np.sum(np.abs(predicted) ** 2, axis=0)
        num = np.sum(np.conj(predicted) * observed, axis=0)
        if not (np.all(np.isfinite(den) & (den > np.finfo(np.float64).tiny)) and np.all(np.isfinite(num))):
            raise WustError("WUST:NumericalFailure", "Unusable source-scale denominator/numerator")
        scale = num / den
        if not np.all(np.isfinite(scale)):
            raise WustError("WUST:NumericalFailure", "Nonfinite source scale")
        residual = (predicted * scale[None, :] - observed) * mask
        loss += 0.5 * float(np.sum(np.abs(residual) ** 2))
        if need_gradient:
            rhs = np.zeros((ny * nx, nb), np.complex128)
            rhs[rx0, :] = residual
            lam = solver.solve(rhs.reshape(ny, nx, nb, order="F"), adjoint=True)
            lam = solver.mass_apply(lam, adjoint=True)
            gradient += np.sum(-np.real(np.conj(v * scale[None, None, :]) * lam), axis=2)
        if retain_state:
            virtual.append(v); scales.append(scale); fields.append(u)
    if not np.isfinite(loss) or (need_gradient and not np.all(np.isfinite(gradient))):
        raise WustError("WUST:NumericalFailure", "Nonfinite objective/gradient")
    cache = dict(solver=solver, virtual=virtual, scales=scales, fields=fields) if retain_state else None
    return loss, gradient, cache


def directional_curvature(state, direction, rx_index, receiver_mask):
    """Gauss-Newton curvature with frozen source scales, directional_curvature.m:1-26.

    ``receiver_mask`` is (n_tx, n_rx) for the frequency.
    """
    solver = state["solver"]
    curvature = 0.0
    offset = 0
    rx0 = np.asarray(rx_index) - 1
    for v, a in zip(state["virtual"], state["scales"]):
        nb = a.size
        ids = list(range(offset, offset + nb))
        offset += nb
        source = solver.mass_apply(v * direction[:, :, None], adjoint=False)
        u = solver.solve(source, adjoint=False)
        uf = u.reshape(-1, nb, order="F")
        deriv = -uf[rx0, :] * a[None, :] * receiver_mask[ids, :].T
        curvature += float(np.sum(np.abs(deriv) ** 2))
    return curvature


def gauss_newton_product(state, direction, rx_index, receiver_mask):
    """Re(J^H J d) with the source scales frozen: the Hessian-vector product
    whose quadratic form d' (J^H J d) is directional_curvature.m:1-26.

    J d is the curvature's ``derivative`` (directional_curvature.m:14-19);
    J^H q is the adjoint solve and accumulation of the oracle's gradient
    (wust_oracle.m:62-68) with q in place of the residual.  Returns
    (product, curvature)."""
    solver = state["solver"]
    ny, nx = direction.shape
    out = np.zeros((ny, nx))
    curvature = 0.0
    offset = 0
    rx0 = np.asarray(rx_index) - 1
    for v, a in zip(state["virtual"], state["scales"]):
        nb = a.size
        ids = list(range(offset, offset + nb))
        offset += nb
        source = solver.mass_apply(v * direction[:, :, None], adjoint=False)
        uf = solver.solve(source, adjoint=False).reshape(-1, nb, order="F")
        q = -uf[rx0, :] * a[None, :] * receiver_mask[ids, :].T
        curvature += float(np.sum(np.abs(q) ** 2))
        rhs = np.zeros((ny * nx, nb), np.complex128)
        rhs[rx0, :] = q
        lam = solver.solve(rhs.reshape(ny, nx, nb, order="F"), adjoint=True)
        lam = solver.mass_apply(lam, adjoint=True)
        out += np.sum(-np.real(np.conj(v * a[None, None, :]) * lam), axis=2)
    return out, curvature


# ---------------------------------------------------------------------------
# NCG helpers
# ---------------------------------------------------------------------------

def ncg_direction(g, z, prev_z, prev_gz, previous_direction, same_frequency):
    """Clipped PR/FR, wust_ncg_direction.m:1-17."""
    g = np.asarray(g, np.float64); z = np.asarray(z, np.float64)
    gz = float(np.sum(g * z))
    beta = 0.0
    if same_frequency and prev_gz > 0:
        beta_fr = gz / prev_gz
        beta_pr = float(np.sum(g * (z - np.asarray(prev_z)))) / prev_gz
        beta = min(max(beta_pr, 0.0), beta_fr)
    direction = -z + beta * np.asarray(previous_direction, np.float64)
    if float(np.sum(g * direction)) >= 0:
        direction = -z
        beta = 0.0
    if not (np.all(np.isfinite(direction)) and np.isfinite(gz) and gz >= 0):
        raise WustError("WUST:NumericalFailure", "Invalid preconditioned gradient")
    return direction, beta, gz


def linearized_step_length(slope, curvature):
    """alpha = max(0, -slope/curvature), linearized_step_length.m:1-11."""
    if not (np.isfinite(slope) and np.isfinite(curvature) and curvature >= 0):
        raise WustError("WUST:NumericalFailure", "Nonfinite slope/curvature")
    if not (curvature > 0 or slope == 0):
        raise WustError("WUST:NumericalFailure", "Zero curvature with nonzero directional slope")
    return max(0.0, -slope / curvature) if curvature > 0 else 0.0


def ringing_removal_filt(xin, yin, img, c0, f, cutoff, order):
    """Radial Butterworth low-pass, ringingRemovalFilt.m:1-45 (cutoff 0 = identity)."""
    if cutoff == 0:
        return img
    nx, ny = len(xin), len(yin)
    dx = float(np.mean(np.diff(xin))); dy = float(np.mean(np.diff(yin)))
    kx = np.fft.fftshift((np.arange(nx) / nx) / dx)
    kx[kx >= 1 / (2 * dx)] -= 1 / dx
    ky = np.fft.fftshift((np.arange(ny) / ny) / dy)
    ky[ky >= 1 / (2 * dy)] -= 1 / dy
    KX, KY = np.meshgrid(kx, ky)
    kc = (2 * f / c0) * cutoff
    filt = 1.0 / (1.0 + ((KX**2 + KY**2) / kc**2) ** order)
    return np.real(np.fft.ifft2(np.fft.ifftshift(filt * np.fft.fftshift(np.fft.fft2(img)))))


def roi_gradient(g, mask, x_m, y_m, c0, frequency_hz, cutoff, order):
    """M F M g, wust_roi_gradient.m:1-10."""
    roi = np.where(mask, g, 0.0)
    z = roi
    if cutoff > 0:
        z = ringing_removal_filt(x_m, y_m, z, c0, frequency_hz, cutoff, order)
    z = np.where(mask, z, 0.0)
    return roi, z


def project_slowness_update(c, direction, alpha, max_update_mps, bounds_mps, step_damping, update_mask):
    """Slowness-space clip, wust_project_slowness_update.m:1-10."""
    c = np.asarray(c, np.float64)
    c_lo = np.maximum(c - max_update_mps, bounds_mps[0])
    c_hi = np.minimum(c + max_update_mps, bounds_mps[1])
    trial = 1.0 / c + step_damping * alpha * np.asarray(direction, np.float64)
    if not np.all(np.isfinite(trial)):
        raise WustError("WUST:NumericalFailure", "Nonfinite slowness trial")
    s_new = np.maximum(1.0 / c_hi, np.minimum(1.0 / c_lo, trial))
    c_new = 1.0 / s_new
    return np.where(update_mask, c_new, c)
