"""Gradients/s of the WUST Helmholtz path on B200 (512^2 interior + 20-cell PML = 552^2, 256 TX).

One step = one gradient: GPU assembly of the nine-point PML operator, block-LU
factorization (552 Schur pages), forward solve of all 256 transmitters,
receiver gather, source fit, misfit, adjoint solve, mass-stencil adjoint and
FP64 gradient accumulation -- i.e. one wust_oracle call with two outputs.

  value  inputs already resident in HBM (device pointers into the C ABI)
  e2e    the same call with HOST buffers (medium, observations, gradient):
         host<->device copies are inside the timed region
Timing: W untimed warm-up steps, then K steps bracketed by barrier +
cudaDeviceSynchronize, CUDA events on the solver stream, max over ranks.
Every input (1.35 GB of Schur inverses, 0.6 GB fields per solve) is larger
than the 126 MB L2, so no explicit flush is needed.

``--impl reference`` times the reference's CPU path (sparse LU in FP64, the
oracle port of HelmholtzSolver's cpu backend) on a bounded sample.
Multi-GPU: replicas only (the Schur recursion does not shard); each rank runs
its own gradient and ``value`` sums the ranks' gradients over the max time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "config2": dict(n_tx=256, freq=1.2e6,
                    text="config2 gradient: 552x552 grid (512^2 + 20-cell PML), dx 0.25 mm, 256 TX x 256 RX ring "
                         "r = 55 mm, f = 1.2 MHz, breast-like phantom"),
    # mid-size case for ncu captures of the tensor-core kernels (same launch
    # shapes as 552^2 with 256 sources: 112-144 CTAs; a few GB on the device)
    "mid400": dict(n_tx=256, freq=0.9e6,
                   text="mid400: 400x400 grid (368^2 + 16-cell PML), dx 0.3 mm, 256 TX x 256 RX ring, f = 0.9 MHz"),
    # seconds-scale case used for ncu captures of the same kernels
    "config1": dict(n_tx=32, freq=0.5e6,
                    text="config1 gradient: 224x224 grid (192^2 + 16-cell PML), dx 0.4 mm, 32 TX x 128 RX ring "
                         "r = 35 mm, f = 0.5 MHz, three elliptical inclusions"),
}
WORKLOAD = "config2"
N_TX = WORKLOADS[WORKLOAD]["n_tx"]
FREQ = WORKLOADS[WORKLOAD]["freq"]


def flops_per_gradient(ny: int, nx: int, s: int) -> dict:
    f_fac = 8.0 * (ny - 2) ** 3 * nx
    f_apply = 2 * 8.0 * ny ** 2 * s * nx
    return dict(factor=f_fac, apply=f_apply, gradient=f_fac + 2 * f_apply)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int = 0, period_ms: int = 200):
        self.cmd = ["nvidia-smi", f"--id={index}",
                    "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                    "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                    "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", f"-lms={period_ms}"]
        self.lines: list[str] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(self.cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=[], samples=0)
        return dict(sm_mhz=float(np.median(sm)), sm_max_mhz=float(max(mx)), reasons=sorted(reasons),
                    samples=len(sm))


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """Max of a per-rank time over the process group (identity on one rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, steps: int, max_ms: float) -> float:
    """Whole-job gradients/s: every rank runs `steps` gradients (replicas),
    timed by the slowest rank."""
    return world * steps / (max_ms * 1e-3)


def make_problem(seed: int = 0):
    from waveforminversionust_b200 import synthetic
    if WORKLOAD == "config1":
        return synthetic.config1(seed=seed)
    if WORKLOAD == "mid400":
        return synthetic.small(seed=seed, n_interior=368, pml=16, dx=0.3e-3, n_elem=256, n_tx=256, freqs=(FREQ,))
    return synthetic.config2(seed=seed, freqs=[FREQ])


PARITY_TX = [0, 37, 73, 110, 146, 183, 219, 255]


def media(p) -> dict:
    """Media a gradient is evaluated at: the homogeneous start of the first NCG
    iteration, a textured NCG-like iterate halfway to the phantom (the
    headline), and a late iterate 90 % of the way (nearly the phantom's
    texture; the phantom itself would leave a zero residual, since the
    observations are simulated on it)."""
    return dict(homogeneous=p.c_init, halfway=0.5 * (p.c_init + p.c_true), late=0.1 * p.c_init + 0.9 * p.c_true)


HEADLINE_MEDIUM = "halfway"


def thread_env() -> dict:
    return {k: os.environ[k] for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")
            if k in os.environ}


def cpu_gradient(pool, p, c, Y, mask, keep=()) -> dict:
    """One full FP64 gradient (all transmitters; SuperLU per worker) on the host cores."""
    return pool.gradient(p.x_m, p.y_m, c, FREQ, p.pml_m, p.tx_index, p.rx_index, Y, mask, keep_fields=keep)


def cpu_sample_text(out) -> str:
    return (f"one full FP64 gradient (all {N_TX} transmitters forward + adjoint, nothing extrapolated): "
            f"SciPy SuperLU sparse LU in complex128, transmitters split over {out['workers']} spawned worker "
            f"processes with one BLAS thread each, every worker assembling and factoring its own operator "
            f"(factor {out['factor_seconds']:.1f} s, solves {out['solve_seconds']:.1f} s in the slowest worker)")


def run_reference(args):
    """The reference's CPU path for this workload (backend 'cpu' of
    HelmholtzSolver: FP64 sparse LU; MATLAB's UMFPACK is unavailable here, so
    the oracle port with SciPy SuperLU stands in), on all host cores: each
    timed step is one full gradient over every transmitter.  Warm-up steps
    run the same pool on the config-1 grid (224^2, 32 transmitters)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.parallel_fp64 import ParallelOracle, host_cores
    from waveforminversionust_b200 import synthetic
    p = make_problem()
    c_eval = media(p)[HEADLINE_MEDIUM]
    small = synthetic.config1(seed=0)
    with ParallelOracle() as pool:
        Y = pool.observe(p.x_m, p.y_m, p.c_true, FREQ, p.pml_m, p.tx_index, p.rx_index)
        mask = np.ones(Y.shape, bool)
        Ys = pool.observe(small.x_m, small.y_m, small.c_true, 0.5e6, small.pml_m, small.tx_index, small.rx_index)
        for _ in range(args.warmup):
            pool.gradient(small.x_m, small.y_m, small.c_init, 0.5e6, small.pml_m, small.tx_index, small.rx_index,
                          Ys, np.ones(Ys.shape, bool))
        secs = []
        last = None
        t0 = time.perf_counter()
        for _ in range(args.steps):
            last = cpu_gradient(pool, p, c_eval, Y, mask)
            secs.append(last["seconds"])
        wall = time.perf_counter() - t0
    ms = 1e3 * wall / args.steps
    v = 1e3 / ms
    ref_gpu = reference_gpu_c64(p, c_eval)
    line = dict(impl="reference", metric="gradients_per_second", value=v, unit="gradients/s", n_gpus=args.gpus,
                steps=args.steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="c128", data="synthetic",
                config=dict(workload=WORKLOADS[WORKLOAD]["text"], global_batch=N_TX, medium=HEADLINE_MEDIUM),
                cpu_baseline=dict(value=v, unit="gradients/s", cores=last["workers"], kind="port",
                                  sample=cpu_sample_text(last)),
                e2e=dict(value=v, unit="gradients/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
                host=dict(cpu_count=os.cpu_count(), affinity_cores=host_cores(), thread_env=thread_env()),
                seconds_per_step=secs, wall_seconds=wall)
    if ref_gpu:
        line["reference_gpu_c64"] = ref_gpu
    print(json.dumps(line), flush=True)


def reference_gpu_c64(p, c, repeats: int = 3) -> dict | None:
    """The reference's GPU path on this device, beside its CPU path: the
    nine-point blocks assembled on the host in FP64 and cast to complex single
    (HelmholtzSolver.m:112-113, 152-160), then the reference's own MEX kernels
    -- decompBlockLU (pivoted cuSOLVER LU per Schur page) and applyBlockLU
    (cuBLAS Cgemm3m sweeps), forward over all transmitters and adjoint over
    as many receiver-residual sources -- compiled unchanged and called through
    the MEX runtime stand-in.  The source fit and gradient (MATLAB gpuArray
    element-wise code in the reference) are not included.  None when no GPU is
    present or the kernels were not built."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        from oracle import helmholtz_fp64 as o
        from oracle.mexshim import driver
        if not driver.reference_available():
            return None
    except Exception:
        return None
    rt = driver.runtime()
    ker = driver.reference_kernels()
    ny, nx = p.shape

    def colmajor(a, dtype=torch.complex64):
        t = torch.as_tensor(np.ascontiguousarray(np.asarray(a).T)).to(device="cuda", dtype=dtype)
        return rt.gpu(t.permute(*reversed(range(t.dim()))), dims=np.asarray(a).shape)

    names = ("Ld", "Ll", "Lu", "Dd", "Dl", "Du", "Ud", "Ul", "Uu")
    src = torch.zeros((N_TX, nx, ny), dtype=torch.complex64, device="cuda")
    src.view(N_TX, -1)[torch.arange(N_TX, device="cuda"), torch.as_tensor(p.tx_index - 1, device="cuda")] = 1
    rng = np.random.default_rng(0)
    res = torch.zeros_like(src)
    vals = rng.standard_normal((N_TX, p.rx_index.size)) + 1j * rng.standard_normal((N_TX, p.rx_index.size))
    res.view(N_TX, -1)[:, torch.as_tensor(p.rx_index - 1, device="cuda")] = torch.as_tensor(
        vals.astype(np.complex64), device="cuda")
    src_mx = rt.gpu(src.permute(2, 1, 0), dims=(ny, nx, N_TX))
    res_mx = rt.gpu(res.permute(2, 1, 0), dims=(ny, nx, N_TX))
    rows = []
    for rep in range(repeats + 1):
        t0 = time.perf_counter()
        pf = o.pml_fields(p.x_m, p.y_m, c, np.zeros(p.shape), FREQ, -1, 10.0, p.pml_m)
        b, d, e = o.stencil_opt_params(1400.0, 1700.0, FREQ, pf.h, pf.g)
        coefs = o.nine_point_coefficients(pf.A, pf.B, pf.C, pf.k, b, d, e, pf.h, pf.g, nx, ny)
        blocks = [colmajor(coefs[n]) for n in names]
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        inv, info = rt.call(ker["decompBlockLU"], 2, *blocks)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        lu = [blocks[i] for i in (0, 1, 2, 6, 7, 8)]
        (u,) = rt.call(ker["applyBlockLU"], 1, src_mx, *lu, inv, rt.logical(False))
        t3 = time.perf_counter()
        del u
        (lam,) = rt.call(ker["applyBlockLU"], 1, res_mx, *lu, inv, rt.logical(True))
        t4 = time.perf_counter()
        del lam, inv
        if rep:
            rows.append(dict(assembly_ms=1e3 * (t1 - t0), factor_ms=1e3 * (t2 - t1),
                             factor_gpu_ms=info.field("total_gpu_ms").scalar(), forward_ms=1e3 * (t3 - t2),
                             adjoint_ms=1e3 * (t4 - t3)))
    med = {k: float(np.median([r[k] for r in rows])) for k in rows[0]}
    core = med["factor_ms"] + med["forward_ms"] + med["adjoint_ms"]
    return dict(kind="the reference's MEX kernels compiled unchanged from Runtime/solver/decompBlockLU.cu and "
                     "applyBlockLU.cu (cuSOLVER getrf/getrs per Schur page, cuBLAS Cgemm3m sweeps), called through "
                     "the MEX runtime stand-in on the same GPU; blocks assembled on the host in FP64",
                repeats=repeats, **med, kernels_ms=core, gradients_per_second_kernels=1e3 / core,
                gradients_per_second_with_assembly=1e3 / (core + med["assembly_ms"]))


def generate_observations(p, solver_cls, torch):
    """Observed pressure from the refined GPU solver on the true model."""
    from waveforminversionust_b200.objective import Observations
    ny, nx = p.shape
    s = solver_cls(p.x_m, p.y_m, p.c_true, None, FREQ, -1, 10.0, p.pml_m,
                   dict(backend="gpu", stencil_bounds=(1400, 1700)), precision="c64-refined", max_sources=N_TX)
    src = torch.zeros((N_TX, nx, ny), dtype=torch.complex64, device="cuda")
    lin = torch.as_tensor(p.tx_index - 1, device="cuda")
    src.view(N_TX, -1)[torch.arange(N_TX, device="cuda"), lin] = 1
    u = s.solve(src.permute(2, 1, 0))
    uf = u.permute(2, 1, 0).reshape(N_TX, -1)
    rx = torch.as_tensor(p.rx_index - 1, device="cuda")
    Y = uf[:, rx].cpu().numpy()[:, :, None]
    s.close()
    del src, u, uf
    mask = np.ones((N_TX, p.rx_index.size, 1), bool)
    return Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, [FREQ], Y, mask)


def run_precision(args, torch):
    """The precision study (config 3) as a report: config 1's geometry and
    phantom (224^2, 32 TX, 128 RX) at twelve frequencies from 0.3 to 1.2 MHz
    (3.1 points per wavelength at 1.2 MHz), observations from the FP64 oracle
    on the true model.  Per profile and frequency, at the initial model: the
    refinement's correction solves and the relative errors of the pressure
    fields, the misfit and the gradient against the FP64 oracle; then a
    continuation of three NCG updates per frequency and the RMS of the final
    sound speed against the plain c64 run and against the true model.  One
    JSON line per profile."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200.objective import POOL, Observations, default_config, wust_oracle
    from waveforminversionust_b200.reconstruct import wust_reconstruct
    from waveforminversionust_b200.solver import HelmholtzSolver
    freqs = np.linspace(0.3e6, 1.2e6, 12)
    p = synthetic.config1(seed=0, freqs=freqs)
    ny, nx = p.shape
    n_tx, n_rx, nf = p.tx_index.size, p.rx_index.size, freqs.size
    ocfg = o.OracleConfig(pml_m=p.pml_m, pml_strength=10, stencil_bounds=(1400, 1700), source_batch_size=n_tx)
    ones = np.ones((n_tx, n_rx, nf), bool)
    dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, freqs, np.zeros((n_tx, n_rx, nf)), ones)
    src = o.point_sources(p.tx_index, range(n_tx), ny, nx)
    Y = np.zeros((n_tx, n_rx, nf), complex)
    for fi in range(nf):
        u = o.make_solver(p.c_true, dummy, fi, ocfg).solve(src)
        Y[:, :, fi] = u.reshape(-1, n_tx, order="F")[p.rx_index - 1, :].T
    obs_o = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, freqs, Y, ones)
    obs = Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, freqs, Y, ones)
    ref = []
    for fi in range(nf):
        sv = o.make_solver(p.c_init, obs_o, fi, ocfg)
        loss, g, _ = o.wust_oracle(p.c_init, obs_o, fi, ocfg, need_gradient=True, solver=sv)
        ref.append((sv.solve(src), loss, g))

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    profiles = [("c64", "default"), ("c64-refined", "default"), ("tf32-refined", "default"), ("tf32-refined", "same"),
                ("bf16-refined", "default")]
    finals = {}
    for prec, corr in profiles:
        rows = []
        for fi, f in enumerate(freqs):
            s = HelmholtzSolver(p.x_m, p.y_m, p.c_init, None, f, -1, 10.0, p.pml_m,
                                dict(backend="gpu", stencil_bounds=(1400, 1700)), precision=prec, max_sources=n_tx,
                                correction_precision=corr)
            u = s.solve(src.astype(np.complex64)).cpu().numpy()
            st = s.stats()
            s.close()
            cfg = default_config(pml_m=p.pml_m, precision=prec, source_batch_size=n_tx, correction_precision=corr)
            loss, g = wust_oracle(p.c_init, obs, fi, cfg, nargout=2)
            u_ref, loss_ref, g_ref = ref[fi]
            rows.append(dict(f_mhz=round(f / 1e6, 4), corrections=st["refine_iters"],
                             pressure_err=rel(u[1:-1, 1:-1], u_ref[1:-1, 1:-1]),
                             misfit_err=abs(loss - loss_ref) / loss_ref, gradient_err=rel(g, g_ref)))
        POOL.clear()
        rcfg = dict(backend="gpu", bounds_mps=(1300.0, 1800.0), max_update_mps=12.0, step_damping=1.0,
                    source_batch_size=n_tx, pml_strength=10.0, pml_m=p.pml_m, stencil_bounds=(1400.0, 1700.0),
                    wavenumber="continuum", filter_cutoff=0.0, filter_order=4, update_mask=p.update_mask.astype(float),
                    frequency_schedule_hz=[f for f in freqs for _ in range(3)], precision=prec,
                    correction_precision=corr)
        t0 = time.perf_counter()
        out = wust_reconstruct(obs, p.c_init, rcfg)
        t_rec = time.perf_counter() - t0
        POOL.clear()
        name = prec if corr == "default" else f"{prec} (TF32 corrections)"
        finals[name] = out["c_mps"]
        print(json.dumps(dict(mode="precision", profile=name, workload="config1 geometry (224^2, 32 TX, 128 RX ring) "
                              "at 12 frequencies 0.3-1.2 MHz, FP64-oracle observations", per_frequency=rows,
                              max_pressure_err=max(r["pressure_err"] for r in rows),
                              max_misfit_err=max(r["misfit_err"] for r in rows),
                              max_gradient_err=max(r["gradient_err"] for r in rows),
                              corrections=[r["corrections"] for r in rows],
                              continuation=dict(updates=len(rcfg["frequency_schedule_hz"]), seconds=round(t_rec, 2),
                                                rms_vs_c64_mps=float(np.sqrt(np.mean((out["c_mps"] - finals["c64"]) ** 2))),
                                                rms_vs_true_mps=float(np.sqrt(np.mean((out["c_mps"] - p.c_true) ** 2))),
                                                rms_initial_vs_true_mps=float(np.sqrt(np.mean((p.c_init - p.c_true) ** 2)))))),
              flush=True)


def run_autograd(args, torch):
    """The differentiation check (config 4) as a report: 256^2 interior + 16-cell
    PML (288^2), dx 0.3 mm, 128-element ring, 64 transmitters, 0.4 and 0.8 MHz,
    observations from the FP64 oracle on the true model.  The slowness is
    float32, 1/1500 s/m with a 2 % smooth random perturbation.  Per profile and
    frequency, through ``torch.autograd`` over Phi_f(s) (backward = the adjoint
    solve and slowness gradient of the same call): the misfit and gradient
    against the FP64 oracle, the directional derivative along a smooth random
    direction against central differences at relative steps 1e-3 .. 1e-6 (the
    perturbed slowness formed in FP64), and the Gauss-Newton directional
    curvature against the oracle's.  Refinement target 1e-10 so the central
    differences resolve their step."""
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    from waveforminversionust_b200.autograd import curvature, misfit, misfit_and_state
    from waveforminversionust_b200.objective import POOL, Observations, default_config
    p = synthetic.config4(seed=0)
    ny, nx = p.shape
    freqs = p.frequencies_hz
    n_tx, n_rx, nf = p.tx_index.size, p.rx_index.size, freqs.size
    ocfg = o.OracleConfig(pml_m=p.pml_m, pml_strength=10, stencil_bounds=(1400, 1700), source_batch_size=n_tx)
    ones = np.ones((n_tx, n_rx, nf), bool)
    dummy = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, freqs, np.zeros((n_tx, n_rx, nf)), ones)
    src = o.point_sources(p.tx_index, range(n_tx), ny, nx)
    Y = np.zeros((n_tx, n_rx, nf), complex)
    for fi in range(nf):
        u = o.make_solver(p.c_true, dummy, fi, ocfg).solve(src)
        Y[:, :, fi] = u.reshape(-1, n_tx, order="F")[p.rx_index - 1, :].T
    obs_o = o.Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, freqs, Y, ones)
    obs = Observations(p.x_m, p.y_m, p.tx_index, p.rx_index, freqs, Y, ones)
    rng = np.random.default_rng(1)
    s32 = ((1.0 + 0.02 * synthetic._smooth_noise(rng, (ny, nx), 6.0)) / 1500.0).astype(np.float32)
    s64 = s32.astype(np.float64)
    direction = synthetic._smooth_noise(rng, (ny, nx), 10.0) * p.update_mask * 1e-2 * float(np.abs(s64).max())
    ref = []
    for fi in range(nf):
        loss, g, state = o.wust_oracle(1.0 / s64, obs_o, fi, ocfg, need_gradient=True, retain_state=True)
        ref.append((loss, g, o.directional_curvature(state, direction, obs_o.rx_index, obs_o.mask[:, :, fi])))

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    d_dev = torch.as_tensor(direction, device="cuda")
    for prec in ("c64-refined", "tf32-refined"):
        cfg = default_config(pml_m=p.pml_m, precision=prec, source_batch_size=n_tx, refine_tol=1e-10)
        rows = []
        for fi in range(nf):
            s0 = torch.tensor(s32, device="cuda", requires_grad=True)
            loss = misfit(s0, obs, fi, cfg)
            loss.backward()
            g = s0.grad.to(torch.float64)
            adj = float((g * d_dev).sum())
            fds = {}
            for rel_step in (1e-3, 1e-4, 1e-5, 1e-6):
                h = rel_step * float(np.abs(s64).max()) / float(np.abs(direction).max())
                with torch.no_grad():
                    base = torch.as_tensor(s64, device="cuda")
                    lp = float(misfit(base + h * d_dev, obs, fi, cfg))
                    lm = float(misfit(base - h * d_dev, obs, fi, cfg))
                fds[f"{rel_step:.0e}"] = abs((lp - lm) / (2 * h) - adj) / abs(adj)
            _, _, state = misfit_and_state(torch.as_tensor(s64, device="cuda"), obs, fi, cfg)
            kappa = curvature(state, direction)
            loss_ref, g_ref, kappa_ref = ref[fi]
            rows.append(dict(f_mhz=float(freqs[fi]) / 1e6, misfit_err=abs(loss.item() - loss_ref) / loss_ref,
                             gradient_err=rel(g.cpu().numpy(), g_ref), directional_fd_rel_err=fds,
                             curvature_err=abs(kappa - kappa_ref) / kappa_ref))
            POOL.clear()
        print(json.dumps(dict(mode="autograd", profile=prec, workload="config4: 256^2 + 16-cell PML, dx 0.3 mm, "
                              "128-element ring, 64 TX, 0.4/0.8 MHz, float32 slowness with a 2 % smooth perturbation",
                              refine_tol=1e-10, per_frequency=rows)), flush=True)


def batch_problems(seed: int = 0, count: int = 24):
    """Config 5's mix of independent inversions: interior grids from
    {128, 192, 256, 384, 512}^2, PML 16-20 cells, dx 0.25-0.4 mm, ring arrays of
    64-256 elements, 16-256 transmitters, each problem at its own frequency in
    0.3-1.2 MHz, a seeded smooth phantom; the homogeneous 1500 m/s start."""
    from waveforminversionust_b200 import synthetic
    rng = np.random.default_rng(seed)
    probs = []
    for k in range(count):
        interior = int(rng.choice([128, 192, 256, 384, 512]))
        pml = int(rng.integers(16, 21))
        dx = float(rng.uniform(0.25e-3, 0.4e-3))
        radius = 0.42 * interior * dx
        n_elem = int(min(rng.choice([64, 128, 256]), 2 ** int(np.log2(2 * np.pi * radius / (1.5 * dx)))))
        n_tx = int(min(rng.choice([16, 32, 64, 128, 256]), n_elem))
        f = float(rng.uniform(0.3e6, 1.2e6))
        amp, sig = float(rng.uniform(10, 40)), float(rng.uniform(0.1, 0.3)) * interior * dx
        probs.append(synthetic._problem(f"batch{k}", interior, pml, dx, n_elem, radius, n_tx, [f],
                                        lambda X, Y, a=amp, w=sig: 1500 + a * np.exp(-(X ** 2 + Y ** 2) / (2 * w * w)),
                                        0.9 * radius))
    return probs


def run_batch(args, torch):
    """Config 5: 24 independent inversions of uneven size, one gradient each
    (tf32-refined).  First every problem alone on the whole GPU, one after
    another (the reference's way: one problem at a time); then the
    autotuner's plan: problems that gain from sharing run concurrently on
    SM partitions (one stream and host thread per partition, cooperative
    kernels capped to the partition), the others alone first.  Both makespans
    are device time (events) over all 24 gradients after a warm-up gradient
    of every problem; solvers are built outside the timed regions.  The
    autotuner's measurements are timed separately."""
    from waveforminversionust_b200.batch import Autotuner, BatchProblem, Plan, run_batch as run_plan
    probs = batch_problems()
    problems = []
    for k, p in enumerate(probs):
        rng = np.random.default_rng(1000 + k)
        n_tx, n_rx = p.tx_index.size, p.rx_index.size
        Y = (rng.standard_normal((n_tx, n_rx)) + 1j * rng.standard_normal((n_tx, n_rx))) * 1e-3
        problems.append(BatchProblem(p.x_m, p.y_m, p.c_init, float(p.frequencies_hz[0]), p.pml_m, p.tx_index,
                                     p.rx_index, Y, np.ones((n_tx, n_rx), bool), precision=args.precision,
                                     name=p.name))
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    seq_plan = Plan(parts=1, cap=n_sm, exclusive=list(range(len(problems))), groups=[[]])
    seq = run_plan(problems, seq_plan)
    t0 = time.perf_counter()
    tuner = Autotuner(parts=(2, 3, 4), repeats=2)
    pl = tuner.tune(problems, n_sm=n_sm)
    tune_s = time.perf_counter() - t0
    par = run_plan(problems, pl)
    rows = []
    for i, p in enumerate(problems):
        rows.append(dict(grid=p.shape[0], n_tx=int(p.tx_index.size), n_rx=int(p.rx_index.size),
                         f_mhz=round(p.frequency_hz / 1e6, 3), alone_ms=round(seq["per_problem_ms"][i], 3),
                         planned_ms=round(par["per_problem_ms"][i], 3),
                         setting="whole GPU" if i in pl.exclusive else f"partition of {pl.cap} SMs",
                         chunks=pl.chunks.get(i, 0)))
    print(json.dumps(dict(mode="batch", precision=args.precision, problems=len(problems),
                          workload="config5: 24 independent inversions, interiors {128..512}^2 + 16-20 PML, "
                                   "dx 0.25-0.4 mm, 16-256 TX, one frequency each in 0.3-1.2 MHz",
                          unit="gradients/s", sequential=dict(value=seq["gradients_per_second"],
                                                              makespan_ms=seq["makespan_s"] * 1e3),
                          planned=dict(value=par["gradients_per_second"], makespan_ms=par["makespan_s"] * 1e3,
                                       exclusive_ms=par["exclusive_s"] * 1e3, concurrent_ms=par["concurrent_s"] * 1e3,
                                       predicted_ms=pl.predicted_s * 1e3),
                          speedup=seq["makespan_s"] / par["makespan_s"],
                          plan=dict(parts=pl.parts, cap=pl.cap, exclusive=pl.exclusive, groups=pl.groups),
                          autotuner=dict(seconds=round(tune_s, 1), measurements=tuner.measured),
                          per_problem=rows)), flush=True)


def run_simulate(args, torch):
    """RF simulation (wust_simulate): the config-2 array on its 512^2 model
    grid (dx 0.25 mm, 20-cell PML outside, 552^2 with it), 256 transmitters x
    256 receivers on the 55 mm ring, Dirichlet 1 MHz tone burst, dt 40 ns, 400
    time samples per step of the bench (the full 80 us record is 2000), all
    transmitters batched.  value: transmitter-time-steps per second with the
    model resident; e2e: the same through the Python call, RF read back to the
    host.  The FP64 oracle on one transmitter and 20 time samples is the CPU
    baseline."""
    from waveforminversionust_b200 import _lib, synthetic
    from waveforminversionust_b200.simulate import wust_simulate
    p = synthetic.config2(seed=0, freqs=[1.2e6])
    hpml = 20                                  # the Helmholtz grid's PML, cropped off
    c = p.c_true[hpml:-hpml, hpml:-hpml]
    x, y = p.x_m[hpml:-hpml], p.y_m[hpml:-hpml]
    # the k-space PML outside the 512^2 model (552^2 with it; measured: a
    # 32-cell PML, 576^2 = 2^6 3^2, ran 35 % slower through cuFFT)
    pml = 20
    ny, nx = c.shape
    # the ring's grid points, moved into the cropped model grid
    iy, ix = (p.tx_index - 1) % p.shape[0] - hpml, (p.tx_index - 1) // p.shape[0] - hpml
    tx = (iy + ny * ix + 1).astype(np.int32)
    ry, rx_ = (p.rx_index - 1) % p.shape[0] - hpml, (p.rx_index - 1) // p.shape[0] - hpml
    rx = (ry + ny * rx_ + 1).astype(np.int32)
    n_time, dt = 400, 40e-9
    c_ref = float(max(1600.0, np.ceil(c.max())))
    t = np.arange(n_time) * dt
    src = np.sin(2 * np.pi * 1e6 * t) * np.exp(-((t - 2e-6) / 0.7e-6) ** 2)
    lib = _lib.load()
    cm = np.ascontiguousarray(c.T)
    rf = torch.empty((tx.size, rx.size, n_time), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()

    def call():
        _lib.check(lib.wust_simulate(cm.ctypes.data_as(C.c_void_p), ny, nx, float(y[1] - y[0]), float(x[1] - x[0]), dt,
                                     n_time, src.ctypes.data_as(C.c_void_p), tx.ctypes.data_as(C.c_void_p), tx.size,
                                     rx.ctypes.data_as(C.c_void_p), rx.size, pml, c_ref, 1000.0, 1, 0,
                                     C.c_void_p(rf.data_ptr()), C.c_void_p(st.cuda_stream)))

    for _ in range(max(1, min(args.warmup, 2))):
        call()
    steps = max(1, min(args.steps, 3))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(steps):
        call()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    units = tx.size * n_time
    model = dict(c_mps=c, x_m=x, y_m=y, tx_index=tx, rx_index=rx, dt_s=dt, source_pressure=src)
    cfg = dict(backend="native-batch", pml_size=pml, density_kg_m3=1000, sound_speed_ref_mps=c_ref,
               downsample_factor=1, time_offset_s=0.0, work_dir=tempfile.mkdtemp(prefix="wust-sim-"))
    t0 = time.perf_counter()
    rec = wust_simulate(model, cfg)
    e2e_s = time.perf_counter() - t0
    from oracle import kwave_fp64 as o
    t0 = time.perf_counter()
    o.simulate(c, float(y[1] - y[0]), float(x[1] - x[0]), dt, src[:20], tx[:1], rx, pml, c_ref, 1000.0)
    cpu_s = time.perf_counter() - t0
    Ny, Nx = ny + 2 * pml, nx + 2 * pml
    # per transmitter and time step: 7 FFT passes (R2C of p, C2R and R2C of
    # the two velocities, C2R of the two divergences) read and write at
    # least one real plane each, the three pointwise kernels 11 planes
    plane = Ny * Nx * 4
    alg_bytes = (7 * 2 + 11) * plane
    achieved = alg_bytes * units / (ms * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    print(json.dumps(dict(
        metric="simulated transmitter-time-steps per second", value=units / (ms * 1e-3), unit="tx*steps/s", n_gpus=1,
        steps=steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f32", data="synthetic",
        config=dict(workload=f"RF simulation: {ny}x{nx} model + {pml}-cell PML ({Ny}x{Nx}), {tx.size} TX x {rx.size} RX, "
                             f"{n_time} samples of dt {dt * 1e9:.0f} ns, all transmitters batched",
                    l2=f"fields {7 * tx.size * plane / 1e9:.1f} GB, larger than L2"),
        e2e=dict(value=units / e2e_s, unit="tx*steps/s", h2d_bytes_per_step=int(cm.nbytes + src.nbytes),
                 d2h_bytes_per_step=int(rec["pressure"].nbytes)),
        roofline=dict(kernel="time step (cuFFT R2C/C2R + 3 fused pointwise kernels) over all transmitters", bound="hbm",
                      achieved=achieved, peak=hbm, unit="GB/s", frac=achieved / hbm,
                      peak_source="MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s", traffic=None,
                      algorithmic_bytes_per_tx_step=alg_bytes),
        cpu_baseline=dict(value=20 / cpu_s, unit="tx*steps/s", cores=1, kind="port",
                          sample="FP64 NumPy oracle, one transmitter, 20 time samples on the same grid"))), flush=True)


def run_dtft(args, torch):
    """The DTFT of the RF preparation (wust_dtft): 2048-sample float32 RF of
    256 x 256 transmitter/receiver pairs at 16 frequencies, RF resident in
    HBM (value) and copied from pinned host memory with Y read back (e2e);
    the oracle's FP64 NumPy DTFT on 8 transmitters as the CPU baseline."""
    from waveforminversionust_b200._lib import check, load
    n_time, n_rx, n_tx, n_f = 2048, 256, 256, 16
    t = np.arange(n_time) * 5e-8
    f = np.linspace(3e5, 1.8e6, n_f)
    rng = np.random.default_rng(0)
    host = torch.as_tensor(rng.standard_normal((n_tx, n_rx, n_time), dtype=np.float32)).pin_memory()
    rf = host.cuda()                                   # memory [time, rx, tx], time fastest
    act = torch.ones((n_rx, n_tx), dtype=torch.uint8, device="cuda")
    Y = torch.empty((n_f, n_rx, n_tx), dtype=torch.complex64, device="cuda")
    Yh = torch.empty_like(Y, device="cpu").pin_memory()
    lib = load()
    st = torch.cuda.current_stream()
    tp, fp = t.ctypes.data_as(C.c_void_p), f.ctypes.data_as(C.c_void_p)

    def call(src):
        check(lib.wust_dtft(tp, n_time, fp, n_f, C.c_void_p(src.data_ptr()), 0, n_rx, n_tx, C.c_void_p(act.data_ptr()),
                            C.c_void_p(Y.data_ptr()), C.c_void_p(st.cuda_stream)))

    for _ in range(args.warmup):
        call(rf)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(args.steps):
        call(rf)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    stage = torch.empty_like(rf)
    torch.cuda.synchronize()
    ev0.record()
    for _ in range(args.steps):
        stage.copy_(host, non_blocking=True)
        call(stage)
        Yh.copy_(Y, non_blocking=True)
    ev1.record()
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1) / args.steps
    from oracle import prepare_fp64 as o
    sample = 8
    p_np = host[:sample].numpy().transpose(2, 1, 0)
    t0 = time.perf_counter()
    o.dtft(t, f, p_np, np.ones((sample, n_rx), bool))
    cpu_s = (time.perf_counter() - t0) * n_tx / sample
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    rf_bytes = n_time * n_rx * n_tx * 4
    achieved = (rf_bytes + n_f * n_rx * n_tx * 8) / (ms * 1e-3) / 1e9
    print(json.dumps(dict(
        metric="rf_preparations_per_second", value=1e3 / ms, unit="preparations/s", n_gpus=1, steps=args.steps,
        warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
        data="synthetic",
        config=dict(workload=f"RF DTFT: {n_time} float32 samples x {n_rx} RX x {n_tx} TX, {n_f} frequencies",
                    l2="RF 512 MB, larger than L2"),
        e2e=dict(value=1e3 / e2e_ms, unit="preparations/s", h2d_bytes_per_step=rf_bytes,
                 d2h_bytes_per_step=n_f * n_rx * n_tx * 8),
        roofline=dict(kernel="dtft_kernel (FP64 CUDA-core GEMM, RF streamed once)", bound="hbm", achieved=achieved,
                      peak=hbm, unit="GB/s", frac=achieved / hbm,
                      peak_source="MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s", traffic=None),
        cpu_baseline=dict(value=1.0 / cpu_s, unit="preparations/s", cores=1, kind="port",
                          sample=f"oracle FP64 NumPy DTFT of {sample} transmitters, scaled to {n_tx}"))))


def run_ncg(args, p, obs, torch):
    """NCG updates of wust_reconstruct (oracle + ROI/filter + direction +
    curvature + step + projection) at the workload's frequency, with the
    update rules on the device (the library's wust_ncg_* entry points) and on
    the host (NumPy, as the reference runs them in MATLAB)."""
    from waveforminversionust_b200.objective import POOL
    from waveforminversionust_b200.reconstruct import wust_reconstruct
    ny, nx = p.shape
    mask = np.zeros((ny, nx))
    mask[20:-20, 20:-20] = 1.0
    n = args.warmup + args.steps
    cfg = dict(backend="gpu", bounds_mps=(1300.0, 1800.0), max_update_mps=10.0, step_damping=1.0,
               source_batch_size=N_TX, pml_strength=10.0, pml_m=p.pml_m, stencil_bounds=(1400.0, 1700.0),
               wavenumber="continuum", filter_cutoff=0.75, filter_order=4, update_mask=mask,
               frequency_schedule_hz=[FREQ] * n, precision=args.precision)
    res = {}
    for dev in (True, False):
        POOL.clear()
        torch.cuda.synchronize()
        out = wust_reconstruct(obs, p.c_init, dict(cfg, ncg_device=dev))
        recs = out["records"][args.warmup:]
        res[dev] = dict(ms_per_update=1e3 * float(np.mean([r["wall_seconds"] for r in recs])),
                        curvature_ms=1e3 * float(np.mean([r["linearized_seconds"] for r in recs])),
                        loss_first=out["records"][0]["loss_before_update"],
                        loss_last=out["records"][-1]["loss_before_update"])
    POOL.clear()
    dev, host = res[True], res[False]
    print(json.dumps(dict(
        metric="ncg_updates_per_second", value=1e3 / dev["ms_per_update"], unit="updates/s", n_gpus=1,
        steps=args.steps, warmup=args.warmup, ms_per_step=dev["ms_per_update"], higher_is_better=True,
        scaling="weak", vs_baseline=None, dtype="tf32+c128-refine" if args.precision == "tf32-refined" else args.precision,
        data="synthetic",
        config=dict(workload=WORKLOADS[WORKLOAD]["text"], loop="wust_reconstruct NCG update, one frequency",
                    filter_cutoff=0.75, precision=args.precision, timing="host wall clock per update"),
        host_rules=dict(value=1e3 / host["ms_per_update"], ms_per_update=host["ms_per_update"]),
        detail=dict(device=dev, host=host))))


def run_solves(args, p, solver_cls, torch):
    """Factor once, then time forward solves of all transmitters (one line of JSON)."""
    ny, nx = p.shape
    s = solver_cls(p.x_m, p.y_m, p.c_init, None, FREQ, -1, 10.0, p.pml_m,
                   dict(backend="gpu", stencil_bounds=(1400, 1700)), precision=args.precision, max_sources=N_TX)
    src = torch.zeros((N_TX, nx, ny), dtype=torch.complex64, device="cuda")
    lin = torch.as_tensor(p.tx_index - 1, device="cuda")
    src.view(N_TX, -1)[torch.arange(N_TX, device="cuda"), lin] = 1
    srcv = src.permute(2, 1, 0)
    for _ in range(min(args.warmup, 1)):
        s.solve(srcv)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        s.solve(srcv)
    ev1.record()
    torch.cuda.synchronize()
    st = s.stats()
    print(json.dumps(dict(mode="solve", precision=args.precision, workload=WORKLOADS[WORKLOAD]["text"],
                          ms_per_solve=ev0.elapsed_time(ev1) / args.steps, factor_ms=s.factor_seconds * 1e3,
                          refine_iters=st["refine_iters"], error_estimate=st["error_estimate"],
                          final_residual=st["final_residual"], kernel_launches=st["kernel_launches"],
                          factor_stats=s.factor_stats())), flush=True)
    s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="tf32-refined")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", default="c64,c64-refined,bf16-refined",
                    help="extra precision profiles timed beside the headline")
    ap.add_argument("--workload", default="config2", choices=sorted(WORKLOADS))
    ap.add_argument("--mode", default="gradient", choices=["gradient", "solve", "ncg", "dtft", "precision", "autograd", "batch", "simulate"],
                    help="solve: factor once, then time forward solves of all transmitters (kernel profiling); "
                         "ncg: time NCG updates of the reconstruction loop, update rules on the device and on the host; "
                         "dtft: time the RF preparation's DTFT")
    args = ap.parse_args()
    global WORKLOAD, N_TX, FREQ
    WORKLOAD = args.workload
    N_TX = WORKLOADS[WORKLOAD]["n_tx"]
    FREQ = WORKLOADS[WORKLOAD]["freq"]
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    from waveforminversionust_b200 import _lib
    from waveforminversionust_b200.objective import default_config
    from waveforminversionust_b200.solver import HelmholtzSolver
    lib = _lib.load()

    if args.mode == "dtft":
        run_dtft(args, torch)
        return
    if args.mode == "simulate":
        run_simulate(args, torch)
        return
    if args.mode == "precision":
        run_precision(args, torch)
        return
    if args.mode == "autograd":
        run_autograd(args, torch)
        return
    if args.mode == "batch":
        run_batch(args, torch)
        return
    p = make_problem(seed=rank)
    ny, nx = p.shape
    if args.mode == "solve":
        run_solves(args, p, HelmholtzSolver, torch)
        return
    obs = generate_observations(p, HelmholtzSolver, torch)
    if args.mode == "ncg":
        run_ncg(args, p, obs, torch)
        return
    fl = flops_per_gradient(ny, nx, N_TX)
    stream = torch.cuda.current_stream()
    M = media(p)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def measure(precision: str, c_model, with_e2e: bool, parity: bool = False):
        solver = HelmholtzSolver(p.x_m, p.y_m, c_model, None, FREQ, -1, 10.0, p.pml_m,
                                 dict(backend="gpu", stencil_bounds=(1400, 1700)), precision=precision,
                                 max_sources=N_TX, stream=stream)
        h = C.c_void_p(solver.handle)
        c_dev = torch.as_tensor(np.asfortranarray(c_model).T.copy(), device="cuda")   # (nx, ny) == col-major
        tx_dev = torch.as_tensor(obs.tx_index.astype(np.int32), device="cuda")
        rx_dev = torch.as_tensor(obs.rx_index.astype(np.int32), device="cuda")
        Y_dev = torch.as_tensor(np.asfortranarray(obs.Y[:, :, 0]).T.astype(np.complex64).copy(), device="cuda")
        m_dev = torch.as_tensor(np.asfortranarray(obs.mask[:, :, 0]).T.astype(np.uint8).copy(), device="cuda")
        g_dev = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
        loss = C.c_double()

        def step_device():
            _lib.check(lib.wust_solver_refactor(h, C.c_void_p(c_dev.data_ptr()), None, C.c_double(FREQ)))
            _lib.check(lib.wust_solver_oracle(h, C.c_void_p(tx_dev.data_ptr()), N_TX, C.c_void_p(rx_dev.data_ptr()),
                                              obs.n_rx, C.c_void_p(Y_dev.data_ptr()), C.c_void_p(m_dev.data_ptr()),
                                              N_TX, _lib.NEED_GRADIENT, C.byref(loss), C.c_void_p(g_dev.data_ptr())))

        # host buffers for e2e (pinned, as a caller would keep them)
        c_h = torch.as_tensor(np.asfortranarray(c_model).T.copy()).pin_memory()
        tx_h = np.ascontiguousarray(obs.tx_index.astype(np.int32))
        rx_h = np.ascontiguousarray(obs.rx_index.astype(np.int32))
        Y_h = torch.as_tensor(np.asfortranarray(obs.Y[:, :, 0]).T.astype(np.complex64).copy()).pin_memory()
        m_h = torch.as_tensor(np.asfortranarray(obs.mask[:, :, 0]).T.astype(np.uint8).copy()).pin_memory()
        g_h = torch.empty((nx, ny), dtype=torch.float64).pin_memory()

        def step_host():
            _lib.check(lib.wust_solver_refactor(h, C.c_void_p(c_h.data_ptr()), None, C.c_double(FREQ)))
            _lib.check(lib.wust_solver_oracle(h, tx_h.ctypes.data_as(C.c_void_p), N_TX,
                                              rx_h.ctypes.data_as(C.c_void_p), obs.n_rx,
                                              C.c_void_p(Y_h.data_ptr()), C.c_void_p(m_h.data_ptr()), N_TX,
                                              _lib.NEED_GRADIENT, C.byref(loss), C.c_void_p(g_h.data_ptr())))

        for _ in range(args.warmup):
            step_device()
        barrier()
        fac_ms, launches = [], 0
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sw_ms0, sw_n0 = solver.sweep_times()
        with ClockSampler(local) as clk:
            barrier()
            ev0.record(stream)
            for _ in range(args.steps):
                step_device()
                fac_ms.append(solver.factor_seconds * 1e3)
                launches += solver.stats()["kernel_launches"] + 1
            ev1.record(stream)
            barrier()
        dev_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
        sw_ms1, sw_n1 = solver.sweep_times()
        stats = solver.stats()
        res = dict(ms_per_step=dev_ms / args.steps, value=aggregate_rate(world, args.steps, dev_ms),
                   factor_ms=float(np.mean(fac_ms)), launches_per_step=launches / args.steps,
                   refine_iters=stats["refine_iters"], final_residual=stats["final_residual"],
                   loss=loss.value, clocks=clk.summary(),
                   sweep_ms_per_launch=(sw_ms1 - sw_ms0) / max(sw_n1 - sw_n0, 1),
                   sweeps_per_step=(sw_n1 - sw_n0) / args.steps, factor_stats=solver.factor_stats())
        if parity:
            # the timed call's outputs, and the forward fields of 8 transmitters
            # from a 256-source solve of the same solver (outside the timed region)
            res["gradient"] = g_dev.cpu().numpy().T.copy()
            src = torch.zeros((N_TX, nx, ny), dtype=torch.complex64, device="cuda")
            src.view(N_TX, -1)[torch.arange(N_TX, device="cuda"), torch.as_tensor(p.tx_index - 1, device="cuda")] = 1
            u = solver.solve(src.permute(2, 1, 0))
            res["fields"] = u[:, :, PARITY_TX].cpu().numpy().astype(np.complex128)
            del src, u
        if with_e2e:
            for _ in range(2):
                step_host()
            barrier()
            ev0.record(stream)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                step_host()
            ev1.record(stream)
            barrier()
            e2e_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
            N = ny * nx
            h2d = N * 8 + 4 * (obs.n_tx + obs.n_rx) + obs.n_tx * obs.n_rx * (8 + 1) + N * 4
            d2h = N * 8 + obs.n_tx * 8
            res["e2e"] = dict(value=aggregate_rate(world, args.steps, e2e_ms), unit="gradients/s",
                              h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h,
                              wall_ms_per_step=(time.perf_counter() - t0) * 1e3 / args.steps)
        solver.close()
        return res

    want_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    head = measure(args.precision, M[HEADLINE_MEDIUM], with_e2e=True, parity=want_cpu)
    other_media = {}
    for name in M:
        if name != HEADLINE_MEDIUM:
            r = measure(args.precision, M[name], with_e2e=False)
            other_media[name] = dict(ms_per_step=r["ms_per_step"], value=r["value"], factor_ms=r["factor_ms"],
                                     refine_iters=r["refine_iters"], factor_stats=r["factor_stats"])
    variants = {}
    for v in [x for x in args.variants.split(",") if x and x != args.precision]:
        variants[v] = measure(v, M[HEADLINE_MEDIUM], with_e2e=False)
        variants[v].pop("clocks", None)

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak_tf = float(peaks.get("bf16_tflops", 1590.0))
    peak_src = ("MEASURED_PEAKS.json bf16_tflops (burst; the TF32 tensor rate of this part is half of it)"
                if peaks else "fallback 1590 TFLOP/s")
    # dominant kernel of the headline step: the sweep kernel (one launch = a
    # forward + backward sweep pair over all sources) or the factorization
    sweep_ms_step = head["sweep_ms_per_launch"] * head["sweeps_per_step"]
    if sweep_ms_step >= head["factor_ms"]:
        flop = fl["apply"]
        achieved = flop / (head["sweep_ms_per_launch"] * 1e-3) / 1e12
        kname = ("tc_chunk_kernel (column-chunked tcgen05 block-LU sweep pairs, 256 sources, 3 launches per "
                 "substitution; mean over the step's pairs: 2 TF32 solves + BF16 correction solves)"
                 if args.precision == "tf32-refined" else "sweep kernels (CUDA-core block-LU sweep pair)")
    else:
        flop = fl["factor"]
        achieved = flop / (head["factor_ms"] * 1e-3) / 1e12
        kname = ("ns_factor_kernel + factor_kernel (Newton-Schulz Schur inverses, Gauss-Jordan pages)"
                 if args.precision == "tf32-refined" else "factor_kernel (Schur recursion + Gauss-Jordan inverses)")
    # DRAM bytes of one sweep pair of the dominant kernel (its six launches),
    # measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum, one
    # pass) at 552^2 with 256 sources: TF32 pair 12.48 GB read + 1.19 GB
    # written, BF16 correction pair 8.27 + 1.16 GB; weighted by the step's
    # 2 TF32 pairs and (pairs - 2) BF16 pairs
    traffic = None
    if flop == fl["apply"] and args.precision == "tf32-refined" and WORKLOAD == "config2":
        n_pairs = max(head["sweeps_per_step"], 2.0)
        traffic = (2 * 13.67e9 + (n_pairs - 2) * 9.42e9) / n_pairs
    roofline = dict(kernel=kname, bound="tensor", achieved=achieved, peak=peak_tf, unit="TFLOP/s",
                    frac=achieved / peak_tf, peak_source=peak_src, traffic=traffic,
                    traffic_unit="bytes per launch (ncu)", hbm_gbs_achieved=(
                        traffic / (head["sweep_ms_per_launch"] * 1e-3) / 1e9 if traffic else None),
                    algorithmic_flop_per_launch=flop,
                    launch_ms=head["sweep_ms_per_launch"] if flop == fl["apply"] else head["factor_ms"])
    # the step by phase: factorization (assembly, Schur inverses, and for the
    # TF32 profile the page packs and chunk propagators), the sweep pairs, and
    # the rest (FP64 refinement launches, fit, gradient, host synchronisation);
    # algorithmic flops against the tensor peak of the arithmetic used (TF32 is
    # half the bf16 figure; the CUDA-core c64 path is shown against it as well)
    tc_peak = peak_tf / 2 if args.precision == "tf32-refined" else peak_tf
    rest_ms = head["ms_per_step"] - head["factor_ms"] - sweep_ms_step
    phases = dict(
        factorization=dict(ms=head["factor_ms"], algorithmic_tflops=fl["factor"] / (head["factor_ms"] * 1e-3) / 1e12,
                           frac_of_tensor_peak=fl["factor"] / (head["factor_ms"] * 1e-3) / 1e12 / tc_peak),
        sweep_pairs=dict(ms=sweep_ms_step, pairs=head["sweeps_per_step"],
                         algorithmic_tflops=fl["apply"] / (head["sweep_ms_per_launch"] * 1e-3) / 1e12,
                         frac_of_tensor_peak=fl["apply"] / (head["sweep_ms_per_launch"] * 1e-3) / 1e12 / tc_peak),
        rest=dict(ms=rest_ms), tensor_peak_tflops=tc_peak)
    cpu = parity = None
    if want_cpu:
        from oracle.parallel_fp64 import ParallelOracle, host_cores
        with ParallelOracle() as pool:
            out = cpu_gradient(pool, p, M[HEADLINE_MEDIUM], obs.Y[:, :, 0], obs.mask[:, :, 0], keep=PARITY_TX)
        cpu = dict(value=1.0 / out["seconds"], unit="gradients/s", cores=out["workers"], kind="port",
                   sample=cpu_sample_text(out),
                   host=dict(cpu_count=os.cpu_count(), affinity_cores=host_cores(), thread_env=thread_env()))
        want_u = np.stack([out["fields"][k] for k in PARITY_TX], axis=2)

        def rel(a, b):
            return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
        parity = dict(
            reference="FP64 sparse LU (SciPy SuperLU, complex128) on the same medium and observations",
            medium=HEADLINE_MEDIUM,
            misfit_rel_err=abs(head["loss"] - out["loss"]) / out["loss"],
            gradient_rel_err=rel(head["gradient"], out["gradient"]),
            pressure_rel_err=rel(head["fields"], want_u),
            pressure_rel_err_per_tx=[rel(head["fields"][:, :, k], want_u[:, :, k]) for k in range(len(PARITY_TX))],
            pressure_tx=PARITY_TX,
            targets=dict(pressure=1e-5, gradient=1e-4))
    line = dict(metric="gradients_per_second", value=head["value"], unit="gradients/s", n_gpus=world,
                steps=args.steps, warmup=args.warmup, ms_per_step=head["ms_per_step"], higher_is_better=True,
                scaling="weak", vs_baseline=None,
                dtype={"c64": "c64", "c64-refined": "c64+c128-refine",
                       "bf16-refined": "bf16+tf32-factor+c128-refine"}.get(args.precision, "tf32+c128-refine"),
                data="synthetic",
                config=dict(workload=WORKLOADS[WORKLOAD]["text"], medium=HEADLINE_MEDIUM,
                            global_batch=N_TX * world, precision=args.precision, parallelism=f"replicas{world}",
                            l2="inputs larger than L2 (invT 1.35 GB, fields 0.62 GB)"),
                e2e=head["e2e"], gpu_launches=int(round(head["launches_per_step"] * args.steps)),
                roofline=roofline, clocks=head["clocks"],
                detail=dict(factor_ms=head["factor_ms"], refine_iters=head["refine_iters"],
                            sweep_ms_per_launch=head["sweep_ms_per_launch"], sweeps_per_step=head["sweeps_per_step"],
                            factor_stats=head["factor_stats"],
                            final_relative_residual=head["final_residual"], flops=fl, phases=phases,
                            media=dict({HEADLINE_MEDIUM: dict(ms_per_step=head["ms_per_step"], value=head["value"],
                                                              factor_ms=head["factor_ms"],
                                                              refine_iters=head["refine_iters"],
                                                              factor_stats=head["factor_stats"])}, **other_media),
                            variants=variants, parity=parity))
    if cpu:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
