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
    """Served reconstruction loop.

    mode "batching" (default): continuous batching.  Each image size has one running batch
    of CG solves on the device (``CgBatch``) with a fixed share of the HBM budget; every
    frame x encoding system of an arriving job waits in that size's queue and joins the
    batch at the next iteration boundary at which its memory fits (admission by HBM
    footprint), so the systems of all jobs in flight advance together, one launch sequence
    per iteration, and leave as they finish.  A job is done when its last system leaves.
    mode "streams": each admitted job solves its systems alone on its own CUDA stream
    (kernels of concurrent jobs overlap only as the GPU's scheduler allows)."""

    def __init__(self, device=None, hbm_budget_bytes=None, max_active=4, graph=True, precision="fp32",
                 mode="batching", sizes=None):
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
        if mode not in ("batching", "streams"):
            raise ValueError(f"mode must be 'batching' or 'streams', got {mode!r}")
        self.mode = mode
        self._workers = {}
        self._sizes = [tuple(int(n) for n in sz) for sz in (sizes or [])]
        if mode == "batching":
            self._sched = None
            for sz in self._sizes:  # workers for the sizes known up front (more on first use)
                self._worker(sz)
        else:
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
            if self.mode == "batching":
                self._worker(tuple(int(n) for n in job.shape)).enqueue(job, fut, time.perf_counter())
                self._cv.notify_all()
                return fut
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
            if self._sched is not None:
                self._sched.join()
            for t in list(self._threads):
                t.join()
            for w in list(self._workers.values()):
                w.thread.join()
                w.batch = None  # the running batch's workspace goes back to the allocator
            self._workers.clear()
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

    def _worker(self, shape):
        """The running batch of one image size (created under self._cv or at start-up)."""
        w = self._workers.get(shape)
        if w is None:
            w = _SizeWorker(self, shape)
            self._workers[shape] = w
            w.thread.start()
        return w

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


class _JobState:
    def __init__(self, job, fut, t_submit, device):
        self.job, self.fut, self.t_submit = job, fut, t_submit
        nsys = len(job.frame_of_system)
        self.x = torch.zeros((nsys,) + tuple(job.shape), dtype=torch.complex64, device=device)
        self.status = [0] * nsys
        self.iters = [0] * nsys
        self.remaining = nsys
        self.t_admit = None


class _SizeWorker:
    """One image size of the batching server: a CgBatch fed from a FIFO of systems."""

    def __init__(self, server, shape):
        self.server = server
        self.shape = shape
        dev = server.device
        self.plan = ToeplitzPlan(shape, dev)
        if server.precision != "fp32" and shape[1:] == (128, 128):
            self.plan.set_precision(server.precision)
        # capacity: an equal share of the budget for each size named at start-up, half of
        # what is left for a size that was not (at least one 32-coil system); per
        # (system, coil) slot the spill of 2 images, per system r, p, Ap
        nv = 1
        for n in shape:
            nv *= int(n)
        if shape in server._sizes:
            share = server.budget // len(server._sizes)
        else:
            server._unlisted_left = getattr(server, "_unlisted_left", server.budget)
            share = server._unlisted_left // 2
            server._unlisted_left -= share
        per_slot = 16 * nv
        max_slots = int(max(32, min(65535, share // (per_slot + 3 * 8 * nv // 8))))
        max_sys = int(max(1, min(4096, max_slots // 4)))
        while max_slots > 32:
            nb = int(self.plan.lib.hb_cg_batch_workspace_bytes(self.plan._h, max_sys, max_slots))
            if nb <= share:
                break
            max_slots = int(max_slots * 0.9)
            max_sys = int(max(1, min(max_sys, max_slots // 4)))
        self.batch = self.plan.cg_batch(max_sys, max_slots)
        self.queue = collections.deque()   # (job state, system index), arrival order
        self.owner = {}                    # handle -> (job state, system index)
        self.thread = threading.Thread(target=self._loop, daemon=True)

    def enqueue(self, job, fut, t_submit):
        js = _JobState(job, fut, t_submit, self.server.device)
        for s in range(len(job.frame_of_system)):
            self.queue.append((js, s))

    def _admit(self):
        """Adds queued systems in arrival order while the batch has room (no overtaking)."""
        from . import capi

        while True:
            with self.server._cv:
                if not self.queue:
                    return
                js, s = self.queue[0]
            job = js.job
            q = System(js.x[s], job.smaps, job.packed_diags[job.frame_of_system[s]], b=job.b[s], coils=job.coils,
                       lam=job.lam)
            try:
                h = self.batch.add(q, job.iters, job.tol)
            except capi.HastyError as e:
                if e.code == capi.HB_ERR_WORKSPACE:
                    return  # full: retry at the next iteration boundary
                raise
            with self.server._cv:
                self.queue.popleft()
            self.owner[h] = (js, s)
            if js.t_admit is None:
                js.t_admit = time.perf_counter()

    def _loop(self):
        srv = self.server
        try:
            torch.cuda.set_device(srv.device)
            stream = torch.cuda.Stream(srv.device)
            with torch.cuda.stream(stream):
                while True:
                    with srv._cv:
                        while not self.queue and not self.owner and not srv._closed:
                            srv._cv.wait()
                        if srv._closed and not self.queue and not self.owner:
                            return
                    self._admit()
                    self.batch.step(stream)
                    for h, st, it in self.batch.retire():
                        js, s = self.owner.pop(h)
                        js.status[s], js.iters[s] = st, it
                        js.remaining -= 1
                        if js.remaining == 0:
                            res = ReconResult(js.job.job_id, js.x, js.status, js.iters, js.t_submit, js.t_admit,
                                              time.perf_counter())
                            with srv._cv:
                                srv._results.append(res)
                            js.fut.set_result(res)
        except Exception as e:  # reported through the futures and close()
            with srv._cv:
                srv._errors.append(e)
                pending = [js for js, _ in self.owner.values()] + [js for js, _ in self.queue]
            for js in pending:
                if not js.fut.done():
                    js.fut.set_exception(e)
