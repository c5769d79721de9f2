"""Benchmark: normal-op applies/s of the batched Toeplitz SENSE CG (4D-flow batch).

Workload (default): 20 cardiac frames x 5 velocity encodings = 100 systems, 128^3
complex64 images, 16 coils, one Toeplitz diagonal (2x grid 256^3, built in FP64 on the
GPU from a per-frame interleaved golden-angle kooshball of 2000 spokes x 256 samples),
15 CG iterations with lambda = 1e-3 on every system.  One step = one batched CG solve
of all 100 systems = 100 x (1 + 15) normal-op applies.  Synthetic, seeded inputs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

By default both plans run on the same inputs: the plain FP32 plan (the headline `value`)
and the reduced-precision plan (forward x pass as BF16 hi+lo contractions on the tensor
cores) as `reduced`.  `precision_check` reports, per sampled frame, each plan's relative
L2 error against the FP64 oracle (the checker, never timed) and the reduced plan's against
the FP32 plan; `served` is a short served run of both plans (Poisson arrivals, p50/p99).

One process per GPU (torchrun for N > 1); each rank solves its own copy of the batch
(weak scaling, no collective on the data path).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "Normal-op applies/s (128^3, 16 coils)"
UNIT = "applies/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--coils", type=int, default=16)
    ap.add_argument("--frames", type=int, default=20)
    ap.add_argument("--encodings", type=int, default=5)
    ap.add_argument("--iters", type=int, default=15)
    ap.add_argument("--spokes", type=int, default=2000)
    ap.add_argument("--samples", type=int, default=256)
    ap.add_argument("--lam", type=float, default=1e-3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mode", default="batch", choices=["batch", "uneven", "serve"],
                    help="batch: the 4D-flow batch (default); uneven: heterogeneous jobs; serve: Poisson arrivals")
    ap.add_argument("--jobs", type=int, default=64, help="uneven/serve: jobs in the mix (serve: pool size)")
    ap.add_argument("--max-frames", type=int, default=20)
    ap.add_argument("--rates", default="1,2,4", help="serve: arrival rates (jobs/s)")
    ap.add_argument("--engine", default="batch", choices=["batch", "groups"],
                    help="uneven/serve: running batches with iteration-boundary admission (batch), or fixed "
                         "groups / per-job streams (groups)")
    ap.add_argument("--duration", type=float, default=30.0, help="serve: seconds of arrivals per rate")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "bf16x3"],
                    help="fp32 everywhere, or the forward x pass as a BF16 hi+lo tensor-core contraction (the "
                         "reduced-precision plan; in the uneven and serve mixes for the 128^3 jobs); both: the "
                         "FP32 plan is the headline and the reduced plan is timed beside it on the same inputs")
    ap.add_argument("--no-check", action="store_true", help="skip the accuracy report against the FP64 oracle")
    ap.add_argument("--check-frames", default="0,7,13,19", help="frames sampled by the accuracy report")
    ap.add_argument("--serve-seconds", type=float, default=12.0,
                    help="batch mode: seconds of Poisson arrivals per plan in the short served leg (0 = off)")
    ap.add_argument("--serve-rate", type=float, default=2.0, help="batch mode: served leg arrival rate (jobs/s)")
    ap.add_argument("--serve-jobs", type=int, default=8, help="batch mode: served leg job pool size")
    ap.add_argument("--serve-max-frames", type=int, default=8, help="batch mode: served leg frames per job (max)")
    ap.add_argument("--diag", default="nufft", choices=["nufft", "exact"],
                    help="Toeplitz diagonal construction: the reference's NUFFT route (tol 1e-6) or FP64-exact")
    return ap.parse_args()


def workload_config(a):
    return {
        "workload": f"4D-flow batch: {a.frames} frames x {a.encodings} encodings, {a.n}^3 complex64, "
                    f"{a.coils} coils, {a.iters}-iteration CG (lambda={a.lam}), per-frame kooshball "
                    f"{a.spokes}x{a.samples}",
        "image": [a.n] * 3, "coils": a.coils, "systems": a.frames * a.encodings, "frames": a.frames,
        "encodings": a.encodings, "cg_iters": a.iters, "lambda": a.lam,
        "applies_per_step": a.frames * a.encodings * (a.iters + 1),
        "l2": "inputs larger than L2 (per-step working set ~60 GB)",
        "parallelism": f"replicas x{a.gpus}",
    }


# ------------------------------------------------------------------ clocks -------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        busy = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- CPU baseline ------
def cpu_reference_rate(a, repeats=1, iters=2):
    """The reference's LibTorch-CPU path (oracle/torch_ref.py) on 1 system x `iters`
    CG iterations x all coils, with all host threads.  Returns (applies/s, sample, cores)."""
    from hastycompute_b200 import synth
    from oracle import torch_ref

    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    shape = (a.n,) * 3
    M = tuple(2 * n for n in shape)
    rng = np.random.default_rng(0)
    # the diagonal's values do not change the CPU path's timing; a seeded stand-in of the
    # right shape and dtype (complex64 on the 2x grid) is used
    T = torch.from_numpy((1.0 + 0.1 * rng.standard_normal(M)).astype(np.complex64))
    sm = torch.from_numpy(synth.coil_maps(a.coils, shape, seed=1))
    b = torch.from_numpy(synth.gaussian_image(shape, seed=2)).reshape((1,) + shape)
    A = torch_ref.ToeplitzSenseNormalCPU(T, sm, lam=a.lam)
    times = []
    napply = 0
    for _ in range(repeats):
        x = torch.zeros_like(b)
        t0 = time.perf_counter()
        napply = torch_ref.conjugate_gradient(A, b, x, iters=iters)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    sample = (f"1 system x {iters} CG iterations ({napply} normal-op applies x {a.coils} coils) at {a.n}^3, "
              f"median of {repeats}; applies/s extrapolates linearly to the full batch")
    return napply / t, sample, cores


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = workload_config(a)
    cfg["parallelism"] = "cpu"
    for _ in range(a.warmup):
        cpu_reference_rate(a, repeats=1, iters=1)
    rates = []
    sample = ""
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    for _ in range(a.steps):
        r, sample, cores = cpu_reference_rate(a, repeats=1, iters=1)
        rates.append(r)
    wall = time.perf_counter() - t0
    v = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1000.0 * wall / max(1, a.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32)", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------- heterogeneous job mixes ------
MIX_SHAPES = [(96, 96, 96), (128, 128, 128), (160, 160, 128)]
MIX_COILS = [8, 12, 16, 32]


def make_job_mix(a, dev, njobs, plans):
    """Seeded job mix: image size from MIX_SHAPES, coils from MIX_COILS, 1..max_frames
    frames (one system per frame), a golden-angle kooshball of 1000-4000 spokes x 256.
    The job's diagonal is built from its trajectory (``--diag``; the NUFFT route falls back
    to the exact build for 96^3 and 160^2 images) and shared by its frames
    (solve timing does not depend on the diagonal's values); b is a seeded random image."""
    from hastycompute_b200 import capi, synth
    from hastycompute_b200.toeplitz import ToeplitzPlan

    rng = np.random.default_rng(a.seed)
    g = torch.Generator(device=dev).manual_seed(a.seed)
    jobs = []
    for j in range(njobs):
        shape = MIX_SHAPES[int(rng.integers(len(MIX_SHAPES)))]
        ncoil = MIX_COILS[int(rng.integers(len(MIX_COILS)))]
        nframes = int(rng.integers(1, a.max_frames + 1))
        spokes = int(rng.integers(1000, 4001))
        if shape not in plans:
            plans[shape] = ToeplitzPlan(shape, dev)
            if a.precision != "fp32" and shape[1:] == (128, 128):  # tensor-core x pass: ny = nx = 128
                plans[shape].set_precision(a.precision)
        plan = plans[shape]
        coords = torch.from_numpy(synth.kooshball(spokes, a.samples, frame=j % 7, nframes=7))
        try:
            packed = plan.build_diagonal(coords, method=a.diag).unsqueeze(0)
        except capi.HastyError as e:  # the NUFFT route needs 4N among its grid lengths (not 96, 160)
            if e.code != capi.HB_ERR_UNSUPPORTED:
                raise
            packed = plan.build_diagonal(coords, method="exact").unsqueeze(0)
        sm = synth.coil_maps_torch(ncoil, shape, seed=1000 + j, device=dev)
        b = torch.randn((nframes,) + shape, dtype=torch.complex64, device=dev, generator=g)
        jobs.append({"shape": shape, "smaps": sm, "packed": packed, "b": b, "frames": nframes, "coils": ncoil,
                     "spokes": spokes})
    return jobs


def run_uneven(a, dev):
    precs = ["fp32", "bf16x3"] if a.precision == "both" else [a.precision]
    out = {}
    for p in precs:
        sa = argparse.Namespace(**vars(a))
        sa.precision = p
        out[p] = uneven_once(sa, dev)
        torch.cuda.empty_cache()
    line = dict(out[precs[0]])
    if len(precs) == 2:
        line["reduced"] = {k: out["bf16x3"][k] for k in ("value", "applies_per_s", "ms_per_step", "dtype", "clocks")}
        line["reduced"]["reduced_over_plain"] = out["bf16x3"]["value"] / out["fp32"]["value"]
    print(json.dumps(line), flush=True)


def uneven_once(a, dev):
    import threading

    from hastycompute_b200 import capi
    from hastycompute_b200.toeplitz import System

    plans = {}
    t0 = time.perf_counter()
    jobs = make_job_mix(a, dev, a.jobs, plans)
    tuned = {str(k): plans[k].autotune(nslots=32) for k in plans}
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    classes = {k: [j for j in jobs if j["shape"] == k] for k in plans}
    xs = {k: [torch.zeros_like(j["b"]) for j in classes[k]] for k in classes}
    ws_cap = int(min(24e9, torch.cuda.mem_get_info(dev)[0] * 0.5 / max(1, len(classes))))

    def systems_of(k):
        out = []
        for j, x in zip(classes[k], xs[k]):
            for f in range(j["frames"]):
                out.append(System(x[f], j["smaps"], j["packed"][0], b=j["b"][f], lam=a.lam))
        return out

    sysl = {k: systems_of(k) for k in classes}
    streams = {k: torch.cuda.Stream(dev) for k in classes}

    batches = {}
    if a.engine == "batch":
        # one running batch per size class, capacity from the same workspace share
        for k in classes:
            nv = k[0] * k[1] * k[2]
            slots = max(32, int(ws_cap // (16 * nv + 24 * nv // 8 + 1)))
            nsysk = max(1, slots // 4)
            while slots > 32 and plans[k].lib.hb_cg_batch_workspace_bytes(plans[k]._h, nsysk, slots) > ws_cap:
                slots = int(slots * 0.9)
                nsysk = max(1, slots // 4)
            batches[k] = plans[k].cg_batch(nsysk, slots)

    def run_batch(k):
        """Every system of size class k through its running batch: systems join as members
        leave (at iteration boundaries), one launch sequence per iteration."""
        bt = batches[k]
        queue = list(sysl[k])
        pos, left = 0, len(queue)
        while left:
            while pos < len(queue):
                try:
                    bt.add(queue[pos], a.iters)
                except capi.HastyError as e:
                    if e.code != capi.HB_ERR_WORKSPACE:
                        raise
                    break
                pos += 1
            bt.step(streams[k])
            left -= len(bt.retire())

    def solve(k, errs):
        try:
            with torch.cuda.stream(streams[k]):
                if a.engine == "batch":
                    run_batch(k)
                else:
                    plans[k].cg_systems(sysl[k], iters=a.iters, graph=True, workspace_bytes=ws_cap)
        except Exception as e:  # noqa: BLE001
            errs.append(e)

    def one_round():
        errs = []
        th = [threading.Thread(target=solve, args=(k, errs)) for k in classes]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errs:
            raise errs[0]

    one_round()  # warm-up (graphs, opt-ins)
    torch.cuda.synchronize()
    clocks = ClockSampler(int(dev.index or 0))
    clocks.start()
    launches0 = capi.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for s_ in streams.values():
        s_.wait_event(e0)
    for _ in range(a.steps):
        one_round()
    for s_ in streams.values():
        torch.cuda.current_stream(dev).wait_stream(s_)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    nsys = sum(len(v) for v in sysl.values())
    applies = nsys * (a.iters + 1) * a.steps
    line = {
        "metric": "CG solves/s (uneven batch)", "value": nsys * a.steps / (ms / 1000.0), "unit": "solves/s",
        "applies_per_s": applies / (ms / 1000.0), "n_gpus": 1, "steps": a.steps, "warmup": 1,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "data": "synthetic (seeded)", "precision": a.precision,
        "dtype": "c64 (fp32)" if a.precision == "fp32" else "c64 (fp32; 128^3 jobs: forward x pass bf16 hi+lo x3)",
        "config": {"workload": f"{a.jobs} jobs, sizes {MIX_SHAPES}, coils {MIX_COILS}, 1-{a.max_frames} frames, "
                               f"1000-4000 spokes x {a.samples}, {a.iters}-iteration CG, "
                               + ("one running batch per size class (systems join at iteration boundaries as "
                                  "members finish; one launch sequence per iteration), each on its own stream"
                                  if a.engine == "batch" else
                                  "one launch sequence per size class on its own stream, groups of systems that "
                                  "fit the workspace, iterations replayed as CUDA graphs"),
                   "engine": a.engine,
                   "systems": nsys, "jobs_per_size": {str(k): len(v) for k, v in classes.items()},
                   "autotuned_plane_schedule": tuned},
        "gpu_launches": capi.launch_count() - launches0, "clocks": clk, "setup_s": setup,
    }
    return line


def run_serve(a, dev):
    precs = ["fp32", "bf16x3"] if a.precision == "both" else [a.precision]
    per = {}
    for p in precs:
        sa = argparse.Namespace(**vars(a))
        sa.precision = p
        per[p] = serve_rates(sa, dev)
        torch.cuda.empty_cache()
    head = per[precs[0]]
    line = {"metric": "p99 recon latency (served)", "value": max(r["p99_s"] for r in head), "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "data": "synthetic (seeded)", "precision": precs[0],
            "dtype": "c64 (fp32)" if precs[0] == "fp32" else
                     "c64 (fp32; 128^3 jobs: forward x pass bf16 hi+lo x3)",
            "config": {"workload": f"Poisson arrivals, job pool of {a.jobs} as in the uneven mix with 1-{a.max_frames} "
                                   f"frames, {a.duration:.0f} s per rate, {a.iters}-iteration CG, admission by HBM "
                                   f"footprint, "
                                   + ("continuous batching: one running batch per image size, systems join at "
                                      "iteration boundaries" if a.engine == "batch" else
                                      "per-job streams (up to 4 concurrent)")},
            "per_rate": head}
    if len(precs) == 2:
        line["reduced"] = {"precision": "bf16x3", "value": max(r["p99_s"] for r in per["bf16x3"]),
                           "per_rate": per["bf16x3"]}
    print(json.dumps(line), flush=True)


def serve_rates(a, dev):
    """Poisson arrivals at each rate of a.rates for a.duration seconds from a pool of a.jobs
    jobs; returns per-rate latency statistics of the served loop."""
    from hastycompute_b200.serve import ReconJob, ReconServer

    plans = {}
    pool = make_job_mix(a, dev, a.jobs, plans)
    for k in plans:
        plans[k].autotune(nslots=32)
    torch.cuda.synchronize()
    rng = np.random.default_rng(a.seed + 1)
    results = []
    for rate in [float(r) for r in a.rates.split(",")]:
        server = ReconServer(dev, hbm_budget_bytes=int(torch.cuda.mem_get_info(dev)[0] * 0.6), max_active=4,
                             precision=a.precision, mode="batching" if a.engine == "batch" else "streams",
                             sizes=sorted({j["shape"] for j in pool}))
        # warm one job through the path
        j0 = pool[0]
        server.submit(ReconJob(j0["shape"], j0["smaps"], j0["packed"], [0] * j0["frames"], j0["b"],
                               iters=a.iters, lam=a.lam)).result()
        server._results.clear()
        t_start = time.perf_counter()
        t_next = t_start
        futs = []
        nsys = 0
        while t_next - t_start < a.duration:
            now = time.perf_counter()
            if now < t_next:
                time.sleep(t_next - now)
            j = pool[int(rng.integers(len(pool)))]
            futs.append(server.submit(ReconJob(j["shape"], j["smaps"], j["packed"], [0] * j["frames"], j["b"],
                                               iters=a.iters, lam=a.lam)))
            nsys += j["frames"]
            t_next += float(rng.exponential(1.0 / rate))
        for f in futs:
            f.result()
        t_end = time.perf_counter()
        server.close()
        st = server.stats()
        results.append({"rate_jobs_per_s": rate, "jobs": st["jobs"], "p50_s": st["p50_s"], "p99_s": st["p99_s"],
                        "mean_s": st["mean_s"], "max_queue_wait_s": st["max_queue_wait_s"],
                        "solves_per_s": nsys / (t_end - t_start), "wall_s": t_end - t_start,
                        "precision": a.precision})
    return results


# ---------------------------------------------------------------- GPU arm --------
def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.mode != "batch":
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
        (run_uneven if a.mode == "uneven" else run_serve)(a, dev)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        pg = dist

    from hastycompute_b200 import capi, synth
    from hastycompute_b200.replicas import job_rate, max_over_ranks, replica_seed
    from hastycompute_b200.toeplitz import ToeplitzPlan

    shape = (a.n,) * 3
    nsys = a.frames * a.encodings
    plan = ToeplitzPlan(shape, dev)
    t_setup = time.perf_counter()
    sm = torch.from_numpy(synth.coil_maps(a.coils, shape, seed=1)).to(dev)
    packed = torch.empty((a.frames, plan.packed_numel()), dtype=torch.float32, device=dev)
    for f in range(a.frames):
        coords = torch.from_numpy(synth.kooshball(a.spokes, a.samples, frame=f, nframes=a.frames))
        packed[f] = plan.build_diagonal(coords, method=a.diag)
    torch.cuda.synchronize()
    t_diag = time.perf_counter() - t_setup
    diag_index = [s // a.encodings for s in range(nsys)]
    xtrue = torch.empty((nsys,) + shape, dtype=torch.complex64, device=dev)
    for f in range(a.frames):
        xtrue[f * a.encodings:(f + 1) * a.encodings] = torch.from_numpy(
            synth.flow_phantom(shape, a.encodings, seed=replica_seed(100 + f, rank))).to(dev)
    b = torch.empty_like(xtrue)
    plan.sense_normal(xtrue, b, sm, packed, diag_index=diag_index, lam=a.lam)
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    applies_per_step = nsys * (a.iters + 1)
    plans_to_time = ["fp32", "bf16x3"] if a.precision == "both" else [a.precision]
    head = plans_to_time[0]

    def step():
        x.zero_()
        plan.cg(x, b, sm, packed, iters=a.iters, lam=a.lam, diag_index=diag_index)

    def timed(prec):
        """W warm-up steps, then K steps between CUDA events (max over ranks); the plan's
        per-kernel CUDA-event profile and launch count over the timed steps."""
        plan.set_precision(prec)
        for _ in range(max(3, a.warmup)):
            step()
        if prec != "fp32":
            plan.wait_status()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        clocks = ClockSampler(local)
        clocks.start()
        launches0 = capi.launch_count()
        capi.profile_start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(a.steps):
            step()
        ev1.record()
        torch.cuda.synchronize()
        prof = capi.profile_stop()
        launches = capi.launch_count() - launches0
        if pg:
            pg.barrier()
        clk = clocks.stop()
        if prec != "fp32":
            plan.wait_status()
        ms = max_over_ranks(ev0.elapsed_time(ev1), pg, dev)
        return {"ms": ms, "value": job_rate(world, applies_per_step * a.steps, ms), "prof": prof,
                "launches": launches, "clocks": clk, "x": x.clone() if a.precision == "both" else None}

    res = {p: timed(p) for p in plans_to_time}
    plan.set_precision(head)
    ms = res[head]["ms"]
    prof = res[head]["prof"]
    value = res[head]["value"]
    clk = res[head]["clocks"]
    launches = res[head]["launches"]

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not a.no_e2e:
        xh = torch.zeros((nsys,) + shape, dtype=torch.complex64).pin_memory()
        bh = b.cpu().pin_memory()
        outh = torch.empty_like(xh).pin_memory()

        def e2e_step():
            # initial guess and right-hand side from pinned host memory, solution back to it;
            # cg_host overlaps the copies of one group of systems with the solve of another
            plan.cg_host(xh, bh, sm, packed, iters=a.iters, lam=a.lam, diag_index=diag_index, chunks=4,
                         out_host=outh)

        e2e_step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1), pg, dev)
        e2e = {"value": job_rate(world, applies_per_step * a.steps, ems), "unit": UNIT,
               "h2d_bytes_per_step": int(xh.numel() * 8 + bh.numel() * 8), "d2h_bytes_per_step": int(outh.numel() * 8),
               "plan": head}
        del xh, bh, outh

    # ---- roofline of the dominant kernel ----
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    U = 8.0 * a.n ** 3
    C = a.coils
    per_kernel = {k: {"ms_total": v[0], "launches": v[1]} for k, v in prof.items() if v[1]}
    # algorithmic bytes per launch of each pass (one CG normal op over all systems):
    #  expand_fwd_x : read S_c (U) + write spill (2U) per slot, read x (U) per system
    #  plane_yz     : read + write the spill (4U) per slot, read Re(T) (4U) per frame
    #  inv_x_combine: read spill (2U) + S_c (U) per slot, read x (U) + write out (U) per system
    alg = {"expand_fwd_x": (3 * C + 1) * U * nsys, "plane_yz": 4 * U * C * nsys + 4 * U * a.frames,
           "inv_x_combine": (3 * C + 2) * U * nsys}
    dom = max(("expand_fwd_x", "plane_yz", "inv_x_combine"), key=lambda k: prof[k][0])
    dms = prof[dom][0] / max(1, prof[dom][1])
    achieved = alg[dom] / (dms / 1000.0) / 1e9
    # DRAM bytes (read + write) per (system, coil) slot of each pass, measured by ncu on one
    # 16-coil system at 128^3 (the passes' ncu summary under profiles/); a launch's traffic grows
    # in proportion to its slots, so a full launch is that figure x slots
    traffic_per_slot = {"expand_fwd_x": 766.4e6 / 16, "plane_yz": 1084.0e6 / 16, "inv_x_combine": 839.6e6 / 16}
    traffic = traffic_per_slot[dom] * C * nsys if a.n == 128 else None
    sched = plan.plane_schedule()
    kernel_name = {"expand_fwd_x": f"expand_fwd_x_kernel<{a.n},16>",
                   "inv_x_combine": f"inv_x_combine_kernel<{a.n},16>",
                   "plane_yz": (f"plane_mod_kernel ({sched})" if sched.startswith("mod")
                                else f"plane_yz_kernel ({sched})")}[dom]
    roofline = {"bound": "hbm", "kernel": kernel_name, "profile_kind": dom, "achieved": achieved,
                "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_src, "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read+write of one 16-slot launch, scaled by slots"
                if traffic is not None else None,
                "alg_bytes_per_launch": alg[dom], "ms_per_launch": dms}
    # reduced-precision plan: tensor-pipe roofline of the tensor-core x pass.  Per (slot, z) it
    # issues 8 chunks x 12 contractions of 128 x 256 x 16 (BF16 in, FP32 accumulate); a third
    # of them carry the hi*hi products, the rest the hi*lo / lo*hi corrections
    tensor_roofline = None
    if "bf16x3" in res and a.n == 128 and res["bf16x3"]["prof"]["expand_fwd_x"][1]:
        pr = res["bf16x3"]["prof"]["expand_fwd_x"]
        ms_tc = pr[0] / pr[1]
        flops = C * nsys * a.n * 8 * 12 * 2.0 * 128 * 256 * 16
        peak_t = float(peaks.get("bf16_tflops_sustained", 1400.0))
        tensor_roofline = {"bound": "tensor", "kernel": "expand_fwd_x_tc", "achieved": flops / (ms_tc / 1000.0) / 1e12,
                           "peak": peak_t, "unit": "TFLOP/s", "frac": flops / (ms_tc / 1000.0) / 1e12 / peak_t,
                           "peak_source": "measured (sustained bf16)" if "bf16_tflops_sustained" in peaks
                           else "fallback", "flops_per_launch": flops, "ms_per_launch": ms_tc}
    # whole-apply yardstick: (18C + 10) * U bytes per normal-op apply
    b_alg = (18 * C + 10) * U
    apply_rate_dev = applies_per_step * a.steps / (ms / 1000.0)
    yard = {"bytes_per_apply": b_alg, "achieved_gbs": b_alg * apply_rate_dev / 1e9,
            "frac_of_hbm": b_alg * apply_rate_dev / 1e9 / hbm}

    reduced = None
    if a.precision == "both":
        r = res["bf16x3"]
        reduced = {"precision": "bf16x3", "value": r["value"], "unit": UNIT, "ms_per_step": r["ms"] / a.steps,
                   "reduced_over_plain": r["value"] / value, "gpu_launches": r["launches"], "clocks": r["clocks"],
                   "kernels": {k: {"ms_total": v[0], "launches": v[1]} for k, v in r["prof"].items() if v[1]},
                   "dtype": "c64 (fp32; forward x pass bf16 hi+lo x3 on tensor cores, fp32 accumulation)"}

    # ---- accuracy of both plans against the FP64 oracle (the checker; never timed) ----
    precision_check = None
    if rank == 0 and not a.no_check:
        precision_check = accuracy_report(a, plan, res, sm, packed, xtrue, b, diag_index, dev)
        plan.set_precision(head)

    # ---- a short served run of both plans (Poisson arrivals, continuous admission) ----
    served = None
    if rank == 0 and world == 1 and a.serve_seconds > 0:
        del res
        x.zero_()
        plan._ws = None
        torch.cuda.empty_cache()
        served = {}
        for prec in plans_to_time:
            sa = argparse.Namespace(**vars(a))
            sa.jobs, sa.max_frames, sa.rates, sa.duration = a.serve_jobs, a.serve_max_frames, str(a.serve_rate), \
                a.serve_seconds
            sa.precision = prec
            served[prec] = serve_rates(sa, dev)[0]
        served["config"] = (f"Poisson arrivals at {a.serve_rate} jobs/s for {a.serve_seconds:.0f} s per plan, pool of "
                            f"{a.serve_jobs} jobs drawn as in the uneven mix with 1-{a.serve_max_frames} frames, "
                            f"{a.iters}-iteration CG, admission by HBM footprint, "
                            + ("continuous batching (one running batch per image size)" if a.engine == "batch"
                               else "up to 4 concurrent jobs on their own streams"))

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        r_, sample, cores = cpu_reference_rate(a)
        cpu = {"value": r_, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": max(3, a.warmup), "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic (seeded)", "config": workload_config(a),
            "dtype": "c64 (fp32)" if head == "fp32" else
                     "c64 (fp32; forward x pass bf16 hi+lo x3 on tensor cores, fp32 accumulation)",
            "precision": head, "reduced": reduced, "precision_check": precision_check,
            "tensor_roofline": tensor_roofline, "served": served,
            "cg_solves_per_s": value / (a.iters + 1), "e2e": e2e, "gpu_launches": launches,
            "roofline": roofline, "apply_yardstick": yard, "kernels": per_kernel, "cpu_baseline": cpu,
            "clocks": clk, "setup_s": {"diagonals": t_diag, "diagonal_method": a.diag},
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def accuracy_report(a, plan, res, sm, packed, xtrue, b, diag_index, dev):
    """Relative L2 errors of the plans on the benchmark's own inputs, per sampled frame.

    * one normal-op apply of the frame's first system: each plan against the FP64 oracle
      (the oracle's complex128 restatement of nufft.cpp:1163-1197 / sense.ixx:500-578, with
      the plans' own diagonal), and the reduced plan against the FP32 plan;
    * the timed CG solutions: reduced plan against the FP32 plan, every system (max) and per
      sampled frame;
    * a 5-iteration CG of the frame's first system, each plan against the oracle's FP64 CG
      (after 5 iterations FP32-vector CG has not yet drifted from exact arithmetic on this
      system; after 15 it has, for the reference's own FP32 CG as well).
    The oracle is the checker here: nothing it computes is timed or returned as a result."""
    from oracle import oracle as O

    frames = sorted({int(f) for f in a.check_frames.split(",") if f.strip() != "" and int(f) < a.frames})
    T_ref = unpack_diagonal(plan, packed)  # [frames] of FP64 Re(T) on the 2x grid, reference layout
    sm64 = sm.to(torch.complex128)
    plans = ["fp32", "bf16x3"] if a.precision == "both" else [a.precision]
    per_frame = []
    for f in frames:
        s = f * a.encodings
        T = T_ref(f)
        A = O.regularized(lambda v: O.sense_normal_toeplitz_t(v, sm64, T), a.lam)
        xs = xtrue[s:s + 1]
        ref = A(xs[0])
        row = {"frame": f, "system": s}
        outs = {}
        for p in plans:
            plan.set_precision(p)
            o = torch.empty_like(xs)
            plan.sense_normal(xs, o, sm, packed, diag_index=diag_index[s:s + 1], lam=a.lam)
            if p != "fp32":
                plan.wait_status()
            outs[p] = o[0]
            row[f"apply_{p}_vs_fp64"] = O.rel_l2(o[0], ref)
        if len(plans) == 2:
            row["apply_bf16x3_vs_fp32"] = O.rel_l2(outs["bf16x3"], outs["fp32"])
        xo5, _ = O.conjugate_gradient(A, b[s], iters=5)
        for p in plans:
            plan.set_precision(p)
            x5 = torch.zeros_like(b[s:s + 1])
            plan.cg(x5, b[s:s + 1], sm, packed, iters=5, lam=a.lam, diag_index=diag_index[s:s + 1])
            if p != "fp32":
                plan.wait_status()
            row[f"cg5_{p}_vs_fp64_cg"] = O.rel_l2(x5[0], xo5)
        if len(plans) == 2:
            xf, xr = res["fp32"]["x"], res["bf16x3"]["x"]
            row["cg15_bf16x3_vs_fp32"] = max(O.rel_l2(xr[s + e], xf[s + e]) for e in range(a.encodings))
        per_frame.append(row)
        del T, A, ref
    out = {"frames": per_frame, "tolerance": {"fp32": 1e-5, "bf16x3": 1e-4}}
    if len(plans) == 2:
        xf, xr = res["fp32"]["x"], res["bf16x3"]["x"]
        out["cg15_bf16x3_vs_fp32_max_all_systems"] = max(O.rel_l2(xr[i], xf[i]) for i in range(xf.shape[0]))
        out["apply_bf16x3_vs_fp64_max"] = max(r["apply_bf16x3_vs_fp64"] for r in per_frame)
    out["apply_fp32_vs_fp64_max"] = max(r[f"apply_{plans[0]}_vs_fp64"] for r in per_frame) if per_frame else None
    return out


TEAM_SHAPE = {8: (4, 2), 16: (4, 4), 32: (8, 4), 64: (8, 8), 128: (16, 8), 256: (16, 16), 96: (24, 4),
              160: (40, 4), 192: (24, 8), 320: (40, 8), 512: (32, 16)}


def column_kz(m0):
    """kz held at each position p of a packed z column: lane t's register r = 4j + c sits at
    p = (j*S + t)*4 + c and holds the z transform's output index (t + S*(r//S)) + E*(r%S)
    (E, S: the team shape of m0)."""
    E, S = TEAM_SHAPE[m0]
    p = np.arange(m0)
    c, q = p % 4, p // 4
    t, r = q % S, 4 * (q // S) + c
    return (t + S * (r // S)) + E * (r % S)


def unpack_diagonal(plan, packed):
    """Reference-layout Re(T) (complex128, [2nz, 2ny, 2nx]) of frame f from the packed
    diagonals the plans read: packed[f] holds Re(T)/prod(2N) as [kx][h][ky'][p] with
    ky = 2ky' + h and each z column in lane order (position p holds kz = column_kz(p);
    the layout hb_diag_pack writes).  Im(T) never reaches the cropped output, so Re(T)
    gives the reference operator exactly."""
    n0, n1, n2 = plan.shape
    m0, m1, m2 = 2 * n0, 2 * n1, 2 * n2
    kz_of = torch.from_numpy(column_kz(m0))

    def get(f):
        p = packed[f].to(torch.float64).reshape(m2, 2, n1, m0) * float(m0 * m1 * m2)
        col = torch.empty_like(p)
        col[..., kz_of.to(p.device)] = p  # back to natural kz order
        t = col.permute(3, 2, 1, 0).reshape(m0, m1, m2)  # [kz][ky' * 2 + h][kx]
        return t.to(torch.complex128)
    return get


if __name__ == "__main__":
    main()
