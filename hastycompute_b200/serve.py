"""Served reconstruction loop: continuous admission of CG jobs by HBM footprint.

Jobs arrive at any time (``submit``).  A scheduler thread admits waiting jobs in arrival
order as soon as their device-memory footprint fits the budget and a slot is free;
every admitted job runs its batched CG (all its frame x encoding systems, one launch
sequence, each iteration replayed as a CUDA graph) on its own CUDA stream, so the
kernels of concurrent jobs overlap on the GPU.  When a job finishes, its memory and slot
are released and the next waiting jobs are admitted.  Coil maps and Toeplitz diagonals
are inputs that stay resident (the caller owns them); the server allocates only each
job's solution vectors and CG workspace, and counts them against the budget.

Kernels are deterministic and a job's arithmetic never depends on other jobs, so a
job's result is bitwise the same alone and in any mix (tested).

This replaces the reference's host-side fan-out of outer batches over a thread pool
with per-stream device contexts (``lib/mri/batch_sense.cpp:349-381``,
``lib/op/opalgs.ixx:93-121``) by device-resident state and stream-level overlap.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import torch

from .toeplitz import System, ToeplitzPlan


@dataclass
class ReconJob:
    """One reconstruction: systems s = 0..nsys-1 share the coil maps; system s uses
    diagonal ``frame_of_system[s]`` of ``packed_diags`` and right-hand side ``b[s]``."""
    shape: tuple
    smaps: torch.Tensor                 # [C, nz, ny, nx] complex64, resident
    packed_diags: torch.Tensor          # [nframes, packed] float32, resident
    frame_of_system: list
    b: torch.Tensor                     # [nsys, nz, ny, nx] complex64, resident
    iters: int = 15
    lam: float = 1e-3
    tol: float = 0.0
    coils: list | None = None
    job_id: int = -1


@dataclass
class ReconResult:
    job_id: int
    x: torch.Tensor
    status: list
    iterations: list
    t_submit: float
    t_admit: float
    t_done: float

    @property
    def latency(self):
        return self.t_done - self.t_submit

    @property
    def queue_wait(self):
        return self.t_admit - self.t_submit


def job_footprint(job: ReconJob, plan: ToeplitzPlan) -> int:
    """Device bytes the server allocates for a job: its solution vectors and its CG
    workspace (all systems in one launch sequence)."""
    nsys = len(job.frame_of_system)
    ncoil = len(job.coils) if job.coils is not None else job.smaps.shape[0]
    nv = 1
    for n in job.shape:
        nv *= int(n)
    ws = plan.lib.hb_systems_workspace_bytes(plan._h, nsys, nsys * ncoil, int(job.iters))
    return int(ws) + nsys * nv * 8


class AdmissionQueue:
    """Arrival-ordered admission by memory footprint and concurrency slots (no GPU).

    ``push`` queues an item with its footprint; ``admit`` pops every item at the head
    that fits the remaining budget and a free slot; ``release`` returns an item's
    footprint and slot.  The head blocks later items (no overtaking), so admission
    follows arrival order."""

    def __init__(self, budget, max_active):
        self.budget = int(budget)
        self.max_active = int(max_active)
        self.used = 0
        self.active = 0
        self._q = collections.deque()

    def push(self, item, footprint):
        if footprint > self.budget:
            raise ValueError(f"footprint {footprint} exceeds the budget {self.budget}")
        self._q.append((item, int(footprint)))

    def admit(self):
        out = []
        while self._q and self.active < self.max_active and self.used + self._q[0][1] <= self.budget:
            item, fp = self._q.popleft()
            self.used += fp
            self.active += 1
            out.append((item, fp))
        return out

    def release(self, footprint):
        self.used -= int(footprint)
        self.active -= 1

    def __len__(self):
        return len(self._q)


class ReconServer:
    def __init__(self, device=None, hbm_budget_bytes=None, max_active=4, graph=True, precision="fp32"):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget_bytes = int(free * 0.8)
        self.budget = int(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.graph = graph
        # "bf16x3": jobs with ny = nx = 128 run the forward x pass on the tensor cores
        # (ToeplitzPlan.set_precision); other sizes stay FP32
        self.precision = precision
        self._cv = threading.Condition()
        self._queue = AdmissionQueue(self.budget, self.max_active)
        self._closed = False
        self._next_id = 0
        self._plans = {}
        self._results = []
        self._threads = []
        self._errors = []
        self._sched = threading.Thread(target=self._schedule, daemon=True)
        self._sched.start()

    # ------------------------------------------------------------------ public ----
    def submit(self, job: ReconJob) -> Future:
        fut = Future()
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            job.job_id = self._next_id if job.job_id < 0 else job.job_id
            self._next_id += 1
            fp = job_footprint(job, self._plan(job.shape))
            try:
                self._queue.push((job, fut, time.perf_counter()), fp)
            except ValueError as e:
                raise RuntimeError(f"job {job.job_id}: {e}") from None
            self._cv.notify_all()
        return fut

    def close(self, wait=True):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            self._sched.join()
            for t in list(self._threads):
                t.join()
        if self._errors:
            raise self._errors[0]

    @property
    def results(self):
        return list(self._results)

    def stats(self):
        lat = sorted(r.latency for r in self._results)
        if not lat:
            return {}
        def pct(p):
            return lat[min(len(lat) - 1, int(round(p / 100.0 * (len(lat) - 1))))]
        return {"jobs": len(lat), "p50_s": pct(50), "p99_s": pct(99), "mean_s": sum(lat) / len(lat),
                "max_queue_wait_s": max(r.queue_wait for r in self._results)}

    # --------------------------------------------------------------- internals ----
    def _plan(self, shape):
        shape = tuple(int(n) for n in shape)
        if shape not in self._plans:
            self._plans[shape] = ToeplitzPlan(shape, self.device)
        return self._plans[shape]

    def _schedule(self):
        while True:
            with self._cv:
                while True:
                    admitted = self._queue.admit()
                    if admitted or (self._closed and len(self._queue) == 0):
                        break
                    self._cv.wait()
            if not admitted:
                return
            for (job, fut, t0), fp in admitted:
                t = threading.Thread(target=self._run, args=(job, fut, t0, fp), daemon=True)
                self._threads.append(t)
                t.start()

    def _run(self, job, fut, t_submit, fp):
        t_admit = time.perf_counter()
        try:
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(self.device)
            # a plan per running job: plans keep a workspace cache, jobs must not share it
            plan = ToeplitzPlan(job.shape, self.device)
            if self.precision != "fp32" and tuple(job.shape)[1:] == (128, 128):
                plan.set_precision(self.precision)
            with torch.cuda.stream(stream):
                nsys = len(job.frame_of_system)
                x = torch.zeros((nsys,) + tuple(job.shape), dtype=torch.complex64, device=self.device)
                systems = [System(x[s], job.smaps, job.packed_diags[job.frame_of_system[s]], b=job.b[s],
                                  coils=job.coils, lam=job.lam) for s in range(nsys)]
                status, iters = plan.cg_systems(systems, iters=job.iters, tol=job.tol, graph=self.graph,
                                                raise_not_pd=False)
                stream.synchronize()
            res = ReconResult(job.job_id, x, status, iters, t_submit, t_admit, time.perf_counter())
            with self._cv:
                self._results.append(res)
            fut.set_result(res)
        except Exception as e:  # reported through the future and close()
            with self._cv:
                self._errors.append(e)
            fut.set_exception(e)
        finally:
            with self._cv:
                self._queue.release(fp)
                self._cv.notify_all()
