"""Many independent inversions of uneven size on one GPU at once, and the
autotuner that decides how to share the GPU between them.

The reference runs one problem at a time (its only parallelism is the
transmitter batch of wust_oracle.m:28-30).  Small problems cannot fill a
B200: their Schur recursion is a chain of ~150-550 dependent pages and their
sweeps a chain of columns, so a whole-GPU launch leaves most SMs idle.  Here
each problem gets its own solver on its own CUDA stream, confined to a
partition of the SMs by capping the CTAs of its cooperative kernels
(``max_ctas``); the caps of the partitions that run together sum to at most
the SM count, and every cooperative CTA needs a whole SM (its shared memory),
so all CTAs of every running cooperative kernel can be resident at once,
whatever the other partitions do, and their grid barriers always complete.
One host thread per partition runs that partition's problems in turn (the
library's calls release the GIL and synchronise only their own stream).

The autotuner measures (CUDA events on the problem's stream, after a warm-up)
each problem's gradient on the whole GPU and under the cap of K equal
partitions, K in ``parts``, and for the chosen setting the column-chunk count
of the chunked sweeps (the source tile is the problem's whole transmitter set,
up to 256, in every case).  ``plan`` then picks, deterministically from those
times, K, the problems that run alone on the whole GPU first (those that gain
nothing from sharing: large grids whose Newton-Schulz factorization needs
more CTAs than a partition holds), and a longest-first assignment of the
others to the K partitions.  Measurements are cached by problem signature
(grid, transmitters, receivers, frequency, profile, cap, chunk count) in
memory and, optionally, in a JSON file.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .solver import HelmholtzSolver


@dataclass
class BatchProblem:
    """One independent gradient evaluation: grid, medium, frequency, array and data."""
    x_m: np.ndarray
    y_m: np.ndarray
    c: np.ndarray                  # [ny, nx] sound speed of the current model
    frequency_hz: float
    pml_m: float
    tx_index: np.ndarray           # 1-based linear indices
    rx_index: np.ndarray
    Y: np.ndarray                  # [n_tx, n_rx] complex observations
    mask: np.ndarray               # [n_tx, n_rx] bool
    precision: str = "tf32-refined"
    name: str = ""

    @property
    def shape(self):
        return (self.y_m.size, self.x_m.size)

    def signature(self) -> tuple:
        ny, nx = self.shape
        return (ny, nx, int(self.tx_index.size), int(self.rx_index.size), round(float(self.frequency_hz), -3),
                self.precision)


class GradientJob:
    """A problem's solver (on a given stream, capped) with its inputs resident in HBM."""

    def __init__(self, prob: BatchProblem, stream: torch.cuda.Stream, max_ctas: int = 0, chunk_count: int = 0):
        self.lib = _lib.load()
        ny, nx = prob.shape
        self.prob = prob
        self.stream = stream
        self.n_tx, self.n_rx = int(prob.tx_index.size), int(prob.rx_index.size)
        self.solver = HelmholtzSolver(prob.x_m, prob.y_m, prob.c, None, prob.frequency_hz, -1, 10.0, prob.pml_m,
                                      dict(backend="gpu", stencil_bounds=(1400, 1700)), precision=prob.precision,
                                      max_sources=min(self.n_tx, 256), stream=stream, max_ctas=max_ctas,
                                      chunk_count=chunk_count)
        with torch.cuda.stream(stream):
            self.c = torch.as_tensor(np.asfortranarray(prob.c).T.copy(), device="cuda")
            self.tx = torch.as_tensor(prob.tx_index.astype(np.int32), device="cuda")
            self.rx = torch.as_tensor(prob.rx_index.astype(np.int32), device="cuda")
            self.Y = torch.as_tensor(np.asfortranarray(prob.Y).T.astype(np.complex64).copy(), device="cuda")
            self.m = torch.as_tensor(np.asfortranarray(prob.mask).T.astype(np.uint8).copy(), device="cuda")
            self.g = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
        stream.synchronize()
        self.loss = C.c_double()

    def run(self) -> float:
        """One gradient: refactor for the model, then wust_oracle with the gradient."""
        h = C.c_void_p(self.solver.handle)
        _lib.check(self.lib.wust_solver_refactor(h, C.c_void_p(self.c.data_ptr()), None,
                                                 C.c_double(self.prob.frequency_hz)))
        _lib.check(self.lib.wust_solver_oracle(h, C.c_void_p(self.tx.data_ptr()), self.n_tx,
                                               C.c_void_p(self.rx.data_ptr()), self.n_rx,
                                               C.c_void_p(self.Y.data_ptr()), C.c_void_p(self.m.data_ptr()),
                                               min(self.n_tx, 256), _lib.NEED_GRADIENT, C.byref(self.loss),
                                               C.c_void_p(self.g.data_ptr())))
        return self.loss.value

    def gradient(self) -> np.ndarray:
        return self.g.cpu().numpy().T.copy()

    def close(self):
        self.solver.close()


def lpt(times, k: int):
    """Longest-processing-time-first assignment of jobs to k machines: job
    indices per machine and the makespan.  Ties go to the lowest job index and
    the lowest machine, so the result depends on the times only."""
    order = sorted(range(len(times)), key=lambda i: (-times[i], i))
    loads = [0.0] * k
    groups = [[] for _ in range(k)]
    for i in order:
        m = min(range(k), key=lambda q: (loads[q], q))
        groups[m].append(i)
        loads[m] += times[i]
    return groups, (max(loads) if times else 0.0)


@dataclass
class Plan:
    parts: int                                     # concurrent partitions K
    cap: int                                       # CTAs per partition
    exclusive: list = field(default_factory=list)  # problems run alone on the whole GPU, in order
    groups: list = field(default_factory=list)     # per partition: problem indices, in order
    chunks: dict = field(default_factory=dict)     # problem index -> chunk count (0: automatic)
    predicted_s: float = 0.0
    table: dict = field(default_factory=dict)      # the measured times the plan came from


def plan(t_full, t_part: dict, n_sm: int) -> Plan:
    """The schedule with the smallest predicted makespan.

    t_full[p]: seconds of problem p alone on the whole GPU; t_part[K][p]:
    seconds under the cap of K equal partitions (None where the problem does
    not fit one).  A problem runs in the concurrent phase when its
    partition time, shared K ways, beats its whole-GPU time.  Candidates
    are ordered by K, and the first of equal makespans wins."""
    n = len(t_full)
    best = Plan(parts=1, cap=n_sm, exclusive=list(range(n)), groups=[[]], predicted_s=float(sum(t_full)))
    for K in sorted(t_part):
        tk = t_part[K]
        shared = [p for p in range(n) if tk[p] is not None and tk[p] / K < t_full[p]]
        alone = [p for p in range(n) if p not in shared]
        groups, span = lpt([tk[p] for p in shared], K)
        total = float(sum(t_full[p] for p in alone)) + span
        if total < best.predicted_s - 1e-12:
            best = Plan(parts=K, cap=n_sm // K, exclusive=alone, groups=[[shared[i] for i in g] for g in groups],
                        predicted_s=total)
    best.table = dict(full=list(t_full), parts={int(k): list(v) for k, v in t_part.items()})
    return best


class Autotuner:
    """Measures gradient times per (problem signature, cap, chunk count) and plans a batch."""

    def __init__(self, cache_path: str | None = None, parts=(2, 3, 4), repeats: int = 2):
        self.cache_path = cache_path
        self.parts = tuple(parts)
        self.repeats = repeats
        self.cache: dict = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = {k: v for k, v in json.load(f).items()}
        self.measured = 0

    @staticmethod
    def _key(prob: BatchProblem, cap: int, chunks: int) -> str:
        return json.dumps([*prob.signature(), int(cap), int(chunks)])

    def measure(self, prob: BatchProblem, cap: int, chunks: int = 0):
        """Seconds of one gradient under the cap (None if the solver cannot be built there)."""
        key = self._key(prob, cap, chunks)
        if key in self.cache:
            return self.cache[key]
        stream = torch.cuda.Stream()
        try:
            job = GradientJob(prob, stream, max_ctas=cap, chunk_count=chunks)
        except _lib.WustError:
            self.cache[key] = None
            return None
        try:
            job.run()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ts = []
            for _ in range(self.repeats):
                e0.record(stream)
                job.run()
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1) * 1e-3)
        finally:
            job.close()
        self.measured += 1
        self.cache[key] = float(np.median(ts))
        return self.cache[key]

    def tune(self, problems, n_sm: int | None = None, chunk_factors=(0.5, 2.0)) -> Plan:
        n_sm = n_sm or torch.cuda.get_device_properties(0).multi_processor_count
        t_full = [self.measure(p, 0) for p in problems]
        t_part = {K: [self.measure(p, n_sm // K) for p in problems] for K in self.parts}
        pl = plan(t_full, t_part, n_sm)
        # the column-chunk count of each problem at its setting (0 = the default rule)
        for idx in [*pl.exclusive, *[i for g in pl.groups for i in g]]:
            prob = problems[idx]
            cap = 0 if idx in pl.exclusive else pl.cap
            steps = prob.shape[1] - 1
            base = int(round(np.sqrt(2.0 * steps)))
            best_c, best_t = 0, (t_full[idx] if cap == 0 else t_part[pl.parts][idx])
            for f in chunk_factors:
                c = max(2, int(round(base * f)))
                t = self.measure(prob, cap, c)
                if t is not None and t < best_t * 0.98:
                    best_c, best_t = c, t
            pl.chunks[idx] = best_c
        if self.cache_path:
            os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
            with open(self.cache_path, "w") as f:
                json.dump(self.cache, f)
        return pl


def run_batch(problems, pl: Plan, repeats: int = 1, keep_gradients: bool = False) -> dict:
    """Run every problem's gradient ``repeats`` times by the plan: the
    exclusive problems one after another on the whole GPU, then the
    partitions concurrently, one host thread and one stream each.  Solvers
    are built (and warmed up) before the timed region.  The makespan is
    device time: from an event before the first gradient to the last
    stream's final event.  Returns it with per-problem device times, losses
    and, on request, the gradients."""
    streams = [torch.cuda.Stream() for _ in range(max(pl.parts, 1))]
    jobs = {}
    for idx in pl.exclusive:
        jobs[idx] = GradientJob(problems[idx], streams[0], 0, pl.chunks.get(idx, 0))
    for q, g in enumerate(pl.groups):
        for idx in g:
            jobs[idx] = GradientJob(problems[idx], streams[q], pl.cap, pl.chunks.get(idx, 0))
    for j in jobs.values():
        j.run()                                   # warm-up
    torch.cuda.synchronize()
    lat = {}
    errors = []

    def timed(idx, stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(repeats):
            jobs[idx].run()
        e1.record(stream)
        e1.synchronize()
        lat[idx] = e0.elapsed_time(e1) / repeats

    def worker(q):
        try:
            for idx in pl.groups[q]:
                timed(idx, streams[q])
        except Exception as e:           # reported after the join
            errors.append(e)

    start = torch.cuda.Event(enable_timing=True)
    mid = torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event(enable_timing=True) for _ in streams]
    start.record(streams[0])
    for idx in pl.exclusive:
        timed(idx, streams[0])
    mid.record(streams[0])
    for st in streams:
        st.wait_event(mid)
    threads = [threading.Thread(target=worker, args=(q,)) for q in range(len(pl.groups)) if pl.groups[q]]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for st, ev in zip(streams, ends):
        ev.record(st)
    torch.cuda.synchronize()
    makespan = max(start.elapsed_time(ev) for ev in ends) * 1e-3
    exclusive = start.elapsed_time(mid) * 1e-3
    out = dict(makespan_s=makespan, exclusive_s=exclusive, concurrent_s=makespan - exclusive, per_problem_ms=lat,
               losses={idx: j.loss.value for idx, j in jobs.items()},
               gradients_per_second=len(problems) * repeats / makespan)
    if keep_gradients:
        out["gradients"] = {idx: j.gradient() for idx, j in jobs.items()}
    for j in jobs.values():
        j.close()
    if errors:
        raise errors[0]
    return out
