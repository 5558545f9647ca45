"""FP64 wust_oracle gradient spread over the host's cores.

TEST AND MEASUREMENT INFRASTRUCTURE ONLY, like the rest of ``oracle/``: it is
imported by ``bench.py``'s CPU legs (the ``cpu_baseline`` object and
``--impl reference``) and by ``tests/``, never by the shipped package.

It runs the reference's CPU path (``HelmholtzSolver`` with backend 'cpu':
sparse LU of the nine-point operator, Runtime/solver/HelmholtzSolver.m:114-143,
then the per-batch forward solve, source fit, misfit, adjoint solve and
gradient of Runtime/matlab/wust_oracle.m:28-72) through the FP64 restatement
in ``oracle.helmholtz_fp64``, on every transmitter of the workload, measured
in full (nothing is extrapolated):

* the transmitters are cut into contiguous groups, one per worker process;
* each worker assembles the operator and factors it with SuperLU itself (a
  SuperLU factorization cannot be shared between processes), then runs
  ``wust_oracle`` on its group as one source batch (one block solve forward,
  one adjoint);
* the parent adds the workers' misfits and gradients in group order.

wust_oracle is invariant to the source batching (Runtime/tests/test_runtime.m:57-61),
so the split changes the result only by rounding.  Workers are started with
``spawn``, never ``fork``: the parent may already hold a CUDA context.  Each
worker runs one BLAS thread (set through its environment at start-up; several
BLAS threads per worker oversubscribe the cores, and changing the count of a
loaded OpenBLAS at run time made SuperLU solves a hundred times slower here),
so the process count is the core count used.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time
from concurrent.futures import ProcessPoolExecutor

import numpy as np


def host_cores() -> int:
    """Cores this process may run on (the affinity mask, not the machine's count)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


_ONE_THREAD = {"OPENBLAS_NUM_THREADS": "1", "OMP_NUM_THREADS": "1", "MKL_NUM_THREADS": "1"}


def _hold(seconds):
    time.sleep(seconds)
    return os.getpid()


def _group_gradient(args):
    """One worker: FP64 assembly + SuperLU + wust_oracle on a group of transmitters."""
    from oracle import helmholtz_fp64 as o
    (x_m, y_m, c, freq, pml_m, pml_strength, bounds, tx_index, rx_index, Y, mask, keep) = args
    t0 = time.perf_counter()
    ny, nx = c.shape
    obs = o.Observations(x_m, y_m, tx_index, rx_index, np.array([freq]), Y[:, :, None], mask[:, :, None])
    cfg = o.OracleConfig(pml_m=pml_m, pml_strength=pml_strength, stencil_bounds=bounds,
                         source_batch_size=max(tx_index.size, 1))
    solver = o.make_solver(c, obs, 0, cfg)
    t1 = time.perf_counter()
    loss, grad, cache = o.wust_oracle(c, obs, 0, cfg, solver=solver, retain_state=bool(keep))
    fields = {}
    if keep:
        u = cache["fields"][0]
        for local, tx_id in keep:
            fields[tx_id] = u[:, :, local].copy()
    t2 = time.perf_counter()
    return loss, grad, fields, (t1 - t0, t2 - t1)


def _group_observe(args):
    """One worker: the receiver pressure of a group of transmitters (FP64 forward solves)."""
    from oracle import helmholtz_fp64 as o
    (x_m, y_m, c, freq, pml_m, pml_strength, bounds, tx_index, rx_index) = args
    ny, nx = c.shape
    s = o.HelmholtzSolverFP64(x_m, y_m, c, np.zeros((ny, nx)), freq, -1, pml_strength, pml_m,
                              dict(backend="cpu", stencil_bounds=bounds))
    u = s.solve(o.point_sources(tx_index, range(tx_index.size), ny, nx))
    return u.reshape(ny * nx, tx_index.size, order="F")[rx_index - 1, :].T


class ParallelOracle:
    """A pool of spawned workers that evaluates FP64 gradients of wust_oracle."""

    def __init__(self, workers: int | None = None, max_workers: int = 32):
        self.workers = max(1, min(workers or host_cores(), max_workers))
        # BLAS reads its thread count when it loads, so the workers get one
        # thread through their environment at start-up: every worker is
        # started here (one held task each) with the variables set, then the
        # parent's environment is put back.
        saved = {k: os.environ.get(k) for k in _ONE_THREAD}
        os.environ.update(_ONE_THREAD)
        try:
            self.pool = ProcessPoolExecutor(self.workers, mp_context=mp.get_context("spawn"))
            pids = list(self.pool.map(_hold, [0.5] * self.workers))
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        self.started = len(set(pids))

    def gradient(self, x_m, y_m, c, freq, pml_m, tx_index, rx_index, Y, mask, keep_fields=(),
                 pml_strength=10.0, stencil_bounds=(1400.0, 1700.0)) -> dict:
        """Misfit and FP64 gradient over all transmitters, plus the forward
        fields of the transmitters listed in ``keep_fields`` (0-based ids).

        Y, mask: (n_tx, n_rx) complex observations and receiver mask of the
        frequency.  Returns dict(loss, gradient, fields, seconds, workers,
        factor_seconds, solve_seconds)."""
        c = np.asarray(c, np.float64)
        tx_index = np.asarray(tx_index)
        n_tx = tx_index.size
        groups = np.array_split(np.arange(n_tx), min(self.workers, n_tx))
        keep = set(int(k) for k in keep_fields)
        jobs = []
        for g in groups:
            kg = [(i, int(t)) for i, t in enumerate(g) if int(t) in keep]
            jobs.append((np.asarray(x_m), np.asarray(y_m), c, float(freq), float(pml_m), float(pml_strength),
                         tuple(stencil_bounds), tx_index[g], np.asarray(rx_index), np.asarray(Y)[g],
                         np.asarray(mask)[g], kg))
        t0 = time.perf_counter()
        results = list(self.pool.map(_group_gradient, jobs))
        seconds = time.perf_counter() - t0
        loss = 0.0
        grad = np.zeros(c.shape)
        fields = {}
        for lo, gr, fl, _ in results:
            loss += lo
            grad += gr
            fields.update(fl)
        return dict(loss=loss, gradient=grad, fields=fields, seconds=seconds, workers=len(groups),
                    factor_seconds=max(r[3][0] for r in results), solve_seconds=max(r[3][1] for r in results))

    def observe(self, x_m, y_m, c, freq, pml_m, tx_index, rx_index, pml_strength=10.0,
                stencil_bounds=(1400.0, 1700.0)) -> np.ndarray:
        """Observations (n_tx, n_rx) complex128: FP64 receiver pressure of every
        transmitter on medium ``c`` (the pattern of Runtime/tests/wust_test_measurements.m:21-35)."""
        c = np.asarray(c, np.float64)
        tx_index = np.asarray(tx_index)
        groups = np.array_split(np.arange(tx_index.size), min(self.workers, tx_index.size))
        jobs = [(np.asarray(x_m), np.asarray(y_m), c, float(freq), float(pml_m), float(pml_strength),
                 tuple(stencil_bounds), tx_index[g], np.asarray(rx_index)) for g in groups]
        return np.concatenate(list(self.pool.map(_group_observe, jobs)), axis=0)

    def close(self):
        self.pool.shutdown(wait=True, cancel_futures=True)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
