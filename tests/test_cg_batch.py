"""The running batch of CG solves (continuous batching, hb_cg_batch_*) against the batched
CG of the same systems: bitwise the same iterates whatever joins or leaves the batch
around them, and the reference's stopping rules (iteration budget, tolerance, breakdown).
Also checked against the FP64 oracle's CG (relative L2 <= 1e-4, as the plain CG tests)."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.toeplitz import System, ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _jobs(plan, cuda, n, lam=1e-3):
    shape = plan.shape
    jobs = []
    for j in range(n):
        rng = np.random.default_rng(50 + j)
        T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 600)), shape)
        nc = 2 + j % 3
        sm = synth.coil_maps(nc + 1, shape, seed=60 + j)
        coils = list(range(nc + 1))[j % 2:][:nc]
        xt = synth.gaussian_image(shape, seed=70 + j)
        b = O.sense_normal_toeplitz(xt, sm, T, coils) + lam * xt
        jobs.append(dict(T=T, sm=sm, smt=_c64(sm, cuda), coils=coils, b=b, bt=_c64(b, cuda), lam=lam,
                         packed=plan.pack_diagonal(_c64(T, cuda))))
    return jobs


def _solo(plan, cuda, j, iters):
    x = torch.zeros(plan.shape, dtype=torch.complex64, device=cuda)
    st, it = plan.cg_systems([System(x, j["smt"], j["packed"], b=j["bt"], coils=j["coils"], lam=j["lam"])],
                             iters=iters, graph=False)
    return x, st[0], it[0]


def test_staggered_arrivals_bitwise_equal_to_batched_cg(cuda):
    shape = (16, 16, 32)
    plan = ToeplitzPlan(shape, cuda)
    jobs = _jobs(plan, cuda, 4)
    budgets = [6, 4, 7, 3]
    arrive = [0, 2, 2, 5]  # step at which each system joins
    batch = plan.cg_batch(max_systems=3, max_coil_slots=12)
    xs = [torch.zeros(shape, dtype=torch.complex64, device=cuda) for _ in jobs]
    handle_of, result, waiting = {}, {}, list(range(len(jobs)))
    step = 0
    while len(result) < len(jobs):
        for i in list(waiting):
            if arrive[i] <= step:
                j = jobs[i]
                try:
                    h = batch.add(System(xs[i], j["smt"], j["packed"], b=j["bt"], coils=j["coils"], lam=j["lam"]),
                                  budgets[i])
                except capi.HastyError as e:  # full: wait for a system to leave
                    assert e.code == capi.HB_ERR_WORKSPACE
                    continue
                handle_of[h] = i
                waiting.remove(i)
        batch.step()
        for h, st, it in batch.retire():
            result[handle_of[h]] = (st, it)
        step += 1
        assert step < 100
    for i, j in enumerate(jobs):
        x_solo, st_solo, it_solo = _solo(plan, cuda, j, budgets[i])
        assert result[i] == (st_solo, it_solo) == (capi.HB_CG_RUNNING, budgets[i])
        assert torch.equal(xs[i], x_solo), i
        A = O.regularized(lambda v, j=j: O.sense_normal_toeplitz(v, j["sm"], j["T"], j["coils"]), j["lam"])
        xo, _ = O.conjugate_gradient(A, j["b"], iters=budgets[i])
        assert O.rel_l2(xs[i].cpu().numpy().astype(np.complex128), xo) < 1e-4


def test_tolerance_breakdown_and_capacity(cuda):
    shape = (16, 16, 16)
    plan = ToeplitzPlan(shape, cuda)
    sm = _c64(synth.coil_maps(2, shape, seed=1), cuda)
    ident = plan.pack_diagonal(_c64(np.ones(plan.grid), cuda))  # normal op = identity
    neg = plan.pack_diagonal(_c64(-np.ones(plan.grid), cuda))   # negative definite
    b = _c64(synth.gaussian_image(shape, seed=2), cuda)
    batch = plan.cg_batch(max_systems=2, max_coil_slots=4)
    x1, x2, x3 = (torch.zeros_like(b) for _ in range(3))
    h1 = batch.add(System(x1, sm, ident, b=b), 20, tol=1e-3)
    h2 = batch.add(System(x2, sm, neg, b=b), 20)
    with pytest.raises(capi.HastyError):  # no free system slot
        batch.add(System(x3, sm, ident, b=b), 5)
    done = {}
    for _ in range(25):
        batch.step()
        done.update({h: (st, it) for h, st, it in batch.retire()})
        if len(done) == 2:
            break
    assert done[h2] == (capi.HB_CG_NOT_PD, 0)
    st1, it1 = done[h1]
    assert st1 == capi.HB_CG_CONVERGED and it1 <= 2
    assert (torch.linalg.vector_norm(x1 - b) / torch.linalg.vector_norm(b)).item() < 1e-5
    h3 = batch.add(System(x3, sm, ident, b=b), 5)  # capacity is free again
    while batch.step():
        pass
    assert [r[0] for r in batch.retire()] == [h3]
