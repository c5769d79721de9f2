"""Served loop: admission policy on CPU; on the GPU, jobs arriving while others run,
with a budget that forces queueing, give the same bits as each job solved alone."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import synth
from hastycompute_b200.serve import AdmissionQueue


def test_admission_by_footprint_and_slots():
    q = AdmissionQueue(budget=100, max_active=2)
    for name, fp in [("a", 60), ("b", 30), ("c", 50), ("d", 10)]:
        q.push(name, fp)
    got = [i for i, _ in q.admit()]
    assert got == ["a", "b"]            # 90 used, slots full
    assert q.admit() == []
    q.release(60)                       # a done: 30 used, 1 slot
    assert [i for i, _ in q.admit()] == ["c"]   # 80 used, slots full
    q.release(30)
    assert [i for i, _ in q.admit()] == ["d"]   # arrival order kept
    with pytest.raises(ValueError):
        q.push("huge", 101)


def test_admission_head_blocks_later_items():
    q = AdmissionQueue(budget=100, max_active=4)
    q.push("big", 90)
    q.push("small", 5)
    q.push("next", 50)
    assert [i for i, _ in q.admit()] == ["big", "small"]
    assert q.admit() == []              # "next" waits for memory, nothing overtakes it
    q.release(90)
    assert [i for i, _ in q.admit()] == ["next"]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["batching", "streams"])
def test_served_jobs_match_alone(cuda, mode):
    from hastycompute_b200.serve import ReconJob, ReconServer, job_footprint
    from hastycompute_b200.toeplitz import System, ToeplitzPlan

    rng = np.random.default_rng(0)
    specs = [((16, 16, 16), 4, 2), ((32, 32, 32), 6, 1), ((16, 16, 16), 3, 3), ((32, 32, 32), 2, 2)]
    jobs = []
    for i, (shape, nc, nf) in enumerate(specs):
        plan = ToeplitzPlan(shape, cuda)
        packed = torch.stack([plan.build_diagonal(torch.from_numpy(synth.kooshball(64 + 32 * f, 2 * shape[0], f, nf)))
                              for f in range(nf)])
        sm = torch.from_numpy(synth.coil_maps(nc, shape, seed=i)).to(cuda)
        nsys = 2 * nf
        b = torch.from_numpy(np.stack([synth.gaussian_image(shape, seed=10 * i + s) for s in range(nsys)])).to(cuda)
        jobs.append(ReconJob(shape=shape, smaps=sm, packed_diags=packed, frame_of_system=[s // 2 for s in range(nsys)],
                             b=b, iters=5, lam=1e-3))
    # budget: the largest job fits, two large ones do not -> queueing happens
    fps = [job_footprint(j, ToeplitzPlan(j.shape, cuda)) for j in jobs]
    # batching: each size's running batch gets half of that budget, so systems queue for it
    server = ReconServer(cuda, hbm_budget_bytes=max(fps) + min(fps), max_active=3, mode=mode,
                         sizes=[(16, 16, 16), (32, 32, 32)])
    futs = [server.submit(j) for j in jobs]
    results = [f.result(timeout=300) for f in futs]
    server.close()
    st = server.stats()
    assert st["jobs"] == len(jobs) and st["p99_s"] >= st["p50_s"] > 0
    for j, r in zip(jobs, results):
        plan = ToeplitzPlan(j.shape, cuda)
        x = torch.zeros_like(r.x)
        plan.cg_systems([System(x[s], j.smaps, j.packed_diags[j.frame_of_system[s]], b=j.b[s], lam=j.lam)
                         for s in range(x.shape[0])], iters=j.iters, graph=False)
        assert torch.equal(x, r.x)
        assert r.iterations == [j.iters] * x.shape[0]
