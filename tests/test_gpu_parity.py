"""GPU parity of the sm_100a path (through the C ABI) against the FP64 oracle.

Tolerance: relative L2 <= 1e-5 for the FP32 path (FP32 FFT arithmetic vs FP64)."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _case(shape, ncoil, K, seed):
    rng = np.random.default_rng(seed)
    coords = rng.uniform(-np.pi, np.pi, (3, K)).astype(np.float32)
    x = synth.gaussian_image(shape, seed=seed + 1)
    sm = synth.coil_maps(ncoil, shape, seed=seed + 2)
    T = O.toeplitz_diagonal(coords.astype(np.float64), shape)
    return coords, x, sm, T


SHAPES = [(8, 8, 8), (8, 16, 32), (32, 8, 16), (16, 16, 16), (32, 32, 32), (64, 32, 16),
          (8, 8, 96), (16, 16, 160), (96, 96, 16), (160, 160, 8)]


@pytest.mark.parametrize("shape", SHAPES)
def test_toeplitz_apply_modes(cuda, shape):
    coords, x, sm, T = _case(shape, 1, 300, 11)
    plan = ToeplitzPlan(shape, cuda)
    packed = plan.pack_diagonal(_c64(T, cuda))
    xt = _c64(x, cuda)
    ref = O.toeplitz_apply(x, T)
    # apply: view into storage2
    s2 = torch.zeros((1,) + plan.grid, dtype=torch.complex64, device=cuda)
    y = plan.apply(xt, packed, s2)
    assert O.rel_l2(_np(y[0]), ref) < TOL
    # apply_add
    add_to = _c64(sm[0], cuda)
    plan.apply_add(xt, add_to, packed)
    assert O.rel_l2(_np(add_to), sm[0] + ref) < TOL
    # apply_addcmul
    mul = np.conj(sm[0])
    add_to = _c64(sm[0], cuda)
    plan.apply_addcmul(xt, add_to, _c64(mul, cuda), packed)
    assert O.rel_l2(_np(add_to), sm[0] + ref * mul) < TOL
    # apply_inplace
    xi = xt.clone()
    plan.apply_inplace(xi, packed)
    assert O.rel_l2(_np(xi), ref) < TOL


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 8, 32), (16, 16, 16)])
def test_diagonal_build_fp64(cuda, shape):
    coords, x, sm, T = _case(shape, 1, 1000, 12)
    plan = ToeplitzPlan(shape, cuda)
    packed, Tg = plan.build_diagonal(torch.from_numpy(coords), want_complex=True)
    assert O.rel_l2(_np(Tg), T) < 1e-6
    packed_ref = plan.pack_diagonal(_c64(T, cuda))
    assert O.rel_l2(packed.cpu().numpy(), packed_ref.cpu().numpy()) < 1e-6
    packed_real_only = plan.build_diagonal(torch.from_numpy(coords))  # Re(T) accumulation only
    assert O.rel_l2(packed_real_only.cpu().numpy(), packed_ref.cpu().numpy()) < 1e-6


def test_diagonal_build_on_grid_samples(cuda):
    """Samples exactly on grid frequencies (the Dirichlet kernel's removable singularity)."""
    shape = (8, 8, 8)
    c = np.zeros((3, 64), np.float32)
    c[:, 1:] = (np.random.default_rng(3).integers(-8, 8, (3, 63)) * (2 * np.pi / 16)).astype(np.float32)
    T = O.toeplitz_diagonal(c.astype(np.float64), shape)
    plan = ToeplitzPlan(shape, cuda)
    _, Tg = plan.build_diagonal(torch.from_numpy(c), want_complex=True)
    assert O.rel_l2(_np(Tg), T) < 1e-6


@pytest.mark.parametrize("shape,ncoil", [((16, 16, 16), 4), ((8, 16, 32), 3), ((32, 32, 32), 8)])
def test_sense_normal_batched(cuda, shape, ncoil):
    rng = np.random.default_rng(13)
    plan = ToeplitzPlan(shape, cuda)
    sm = synth.coil_maps(ncoil, shape, seed=5)
    Ts = [O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 400)), shape) for _ in range(2)]
    packed = torch.cat([plan.pack_diagonal(_c64(T, cuda)) for T in Ts])
    nsys = 3
    xs = np.stack([synth.gaussian_image(shape, seed=20 + s) for s in range(nsys)])
    diag_index = [1, 0, 1]
    coils = [ncoil - 1] + list(range(ncoil - 1))[::2]  # a permuted subset
    lam = 1e-3
    out = torch.empty((nsys,) + shape, dtype=torch.complex64, device=cuda)
    plan.sense_normal(_c64(xs, cuda), out, _c64(sm, cuda), packed, coils=coils, diag_index=diag_index, lam=lam)
    for s in range(nsys):
        ref = O.sense_normal_toeplitz(xs[s], sm, Ts[diag_index[s]], coils) + lam * xs[s]
        assert O.rel_l2(_np(out[s]), ref) < TOL


def test_sense_normal_workspace_groups(cuda):
    """A workspace too small for all systems at once: processed in groups, same result."""
    shape = (16, 16, 16)
    plan = ToeplitzPlan(shape, cuda)
    sm = _c64(synth.coil_maps(4, shape, seed=6), cuda)
    T = O.toeplitz_diagonal(np.random.default_rng(1).uniform(-np.pi, np.pi, (3, 300)), shape)
    packed = plan.pack_diagonal(_c64(T, cuda))
    xs = _c64(np.stack([synth.gaussian_image(shape, seed=s) for s in range(5)]), cuda)
    full = torch.empty_like(xs)
    plan.sense_normal(xs, full, sm, packed)
    part = torch.empty_like(xs)
    nb = capi.load().hb_normal_workspace_bytes(plan._h, 2, 4)
    plan._ws = None
    plan.sense_normal(xs, part, sm, packed, workspace_bytes=nb)
    assert torch.equal(full, part)


def test_config1_size_normal_op(cuda):
    """64^3, 8 coils (the CPU-runnable configuration's size) against the FP64 oracle."""
    shape = (64, 64, 64)
    rng = np.random.default_rng(14)
    plan = ToeplitzPlan(shape, cuda)
    coords = synth.kooshball(256, 128)
    packed, Tg = plan.build_diagonal(torch.from_numpy(coords), want_complex=True)
    T = _np(Tg)  # reference-layout diagonal from the GPU FP64 builder (checked separately)
    sm = synth.coil_maps(8, shape, seed=7)
    x = synth.gaussian_image(shape, seed=8)
    out = torch.empty(shape, dtype=torch.complex64, device=cuda)
    plan.sense_normal(_c64(x, cuda), out, _c64(sm, cuda), packed)
    ref = O.sense_normal_toeplitz(x, sm, T)
    assert O.rel_l2(_np(out), ref) < TOL


def test_config1_cg_matches_oracle(cuda):
    """The CPU-runnable configuration end to end: 64^3, 8 coils, the 4096 x 128 kooshball,
    b = A x_true + lambda x_true with lambda = 1e-3, 10-iteration CG; against the oracle's
    FP64 CG on the same diagonal, and against the reference's own FP32 LibTorch CG
    (opalgs.cpp:50-96 restated call for call).  CG amplifies rounding on this system: the
    reference's FP32 CG lands 2.2e-3 from the FP64 one, this path's (FP64 scalars) 2.7e-4."""
    shape = (64, 64, 64)
    plan = ToeplitzPlan(shape, cuda)
    coords = synth.kooshball(4096, 128)
    packed, Tg = plan.build_diagonal(torch.from_numpy(coords), want_complex=True)
    T = _np(Tg)
    sm = synth.coil_maps(8, shape, seed=21)
    xt = synth.gaussian_image(shape, seed=22).astype(np.complex128)
    lam = 1e-3
    b = O.sense_normal_toeplitz(xt, sm, T) + lam * xt
    x = torch.zeros(shape, dtype=torch.complex64, device=cuda)
    status, done = plan.cg(x, _c64(b, cuda), _c64(sm, cuda), packed, iters=10, lam=lam)
    assert done == [10]
    A = O.regularized(lambda v: O.sense_normal_toeplitz(v, sm, T), lam)
    xo, _ = O.conjugate_gradient(A, b, iters=10)
    from oracle import torch_ref as R

    Ar = R.ToeplitzSenseNormalCPU(torch.from_numpy(T.astype(np.complex64)), torch.from_numpy(sm), lam=lam)
    xr = torch.zeros((1,) + shape, dtype=torch.complex64)
    R.conjugate_gradient(Ar, torch.from_numpy(b.astype(np.complex64)).reshape((1,) + shape), xr, iters=10)
    e_gpu = O.rel_l2(_np(x), xo)
    e_ref = O.rel_l2(xr.numpy()[0].astype(np.complex128), xo)
    assert e_gpu < 1e-3 and e_gpu < e_ref


def test_large_size_properties(cuda):
    """128^3 x 16 coils: Hermitian (<Ax,y> = <x,Ay>), linearity, bitwise determinism."""
    shape = (128, 128, 128)
    plan = ToeplitzPlan(shape, cuda)
    coords = synth.kooshball(400, 256)
    packed = plan.build_diagonal(torch.from_numpy(coords))
    sm = _c64(synth.coil_maps(16, shape, seed=9), cuda)
    g = torch.Generator(device="cpu").manual_seed(0)
    xs = torch.randn((2,) + shape, dtype=torch.complex64, generator=g).to(cuda)
    out = torch.empty_like(xs)
    plan.sense_normal(xs, out, sm, packed)
    ax, ay = out[0].to(torch.complex128), out[1].to(torch.complex128)
    x, y = xs[0].to(torch.complex128), xs[1].to(torch.complex128)
    lhs = torch.vdot(ax.flatten(), y.flatten())
    rhs = torch.vdot(x.flatten(), ay.flatten())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    assert torch.vdot(x.flatten(), ax.flatten()).real > 0
    # linearity
    comb = (xs[0] * (0.5 - 0.25j) + xs[1] * 2.0).unsqueeze(0).contiguous()
    oc = torch.empty_like(comb)
    plan.sense_normal(comb, oc, sm, packed)
    lin = out[0] * (0.5 - 0.25j) + out[1] * 2.0
    assert (torch.linalg.vector_norm(oc[0] - lin) / torch.linalg.vector_norm(lin)).item() < 1e-5
    # determinism
    out2 = torch.empty_like(xs)
    plan.sense_normal(xs, out2, sm, packed)
    assert torch.equal(out, out2)


@pytest.mark.parametrize("shape,ncoil,nsys", [((16, 16, 16), 4, 3), ((32, 32, 32), 8, 2)])
def test_cg_matches_oracle(cuda, shape, ncoil, nsys):
    rng = np.random.default_rng(15)
    plan = ToeplitzPlan(shape, cuda)
    sm = synth.coil_maps(ncoil, shape, seed=10)
    Ts = [O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 2000)), shape) for _ in range(2)]
    packed = torch.cat([plan.pack_diagonal(_c64(T, cuda)) for T in Ts])
    diag_index = [s % 2 for s in range(nsys)]
    lam = 1e-3
    iters = 10
    xtrue = np.stack([synth.gaussian_image(shape, seed=30 + s) for s in range(nsys)])
    bs = np.stack([O.sense_normal_toeplitz(xtrue[s], sm, Ts[diag_index[s]]) + lam * xtrue[s] for s in range(nsys)])
    xg = torch.zeros((nsys,) + shape, dtype=torch.complex64, device=cuda)
    status, done = plan.cg(xg, _c64(bs, cuda), _c64(sm, cuda), packed, iters=iters, lam=lam, diag_index=diag_index)
    assert status == [capi.HB_CG_RUNNING] * nsys and done == [iters] * nsys
    for s in range(nsys):
        A = O.regularized(lambda v, s=s: O.sense_normal_toeplitz(v, sm, Ts[diag_index[s]]), lam)
        xo, n = O.conjugate_gradient(A, bs[s], iters=iters)
        assert O.rel_l2(_np(xg[s]), xo) < 1e-4  # FP32 vectors over 10 iterations


def test_cg_tol_stops_early(cuda):
    shape = (16, 16, 16)
    plan = ToeplitzPlan(shape, cuda)
    sm = _c64(synth.coil_maps(2, shape, seed=1), cuda)
    T = np.ones(plan.grid, np.complex128)  # identity normal op: sum_c |S_c|^2 = 1
    packed = plan.pack_diagonal(_c64(T, cuda))
    b = _c64(synth.gaussian_image(shape, seed=2), cuda)
    x = torch.zeros_like(b)
    status, done = plan.cg(x, b, sm, packed, iters=20, tol=1e-3)
    assert status == [capi.HB_CG_CONVERGED]
    assert done[0] <= 2
    assert (torch.linalg.vector_norm(x - b) / torch.linalg.vector_norm(b)).item() < 1e-5


def test_cg_not_positive_definite(cuda):
    """A host-made fault: a negated diagonal makes A negative definite; the device flags
    the system and the call raises like the reference ("A was not positive definite")."""
    shape = (16, 16, 16)
    plan = ToeplitzPlan(shape, cuda)
    sm = _c64(synth.coil_maps(2, shape, seed=1), cuda)
    T = -np.ones(plan.grid, np.complex128)
    packed = plan.pack_diagonal(_c64(T, cuda))
    b = _c64(synth.gaussian_image(shape, seed=2), cuda)
    x = torch.zeros_like(b)
    with pytest.raises(capi.NotPositiveDefinite):
        plan.cg(x, b, sm, packed, iters=5)
    status, done = plan.cg(torch.zeros_like(b), b, sm, packed, iters=5, raise_not_pd=False)
    assert status == [capi.HB_CG_NOT_PD] and done == [0]


def test_invalid_arguments_raise(cuda):
    with pytest.raises(capi.HastyError):
        ToeplitzPlan((12, 16, 16), cuda)
    plan = ToeplitzPlan((8, 8, 8), cuda)
    with pytest.raises(RuntimeError):
        plan.pack_diagonal(torch.zeros((16, 16, 16), dtype=torch.complex128, device=cuda))
    lib = capi.load()
    assert lib.hb_toeplitz_apply(plan._h, None, None, 0, 0, None, 0, None, None, 0, None) == capi.HB_ERR_INVALID
    assert b"NULL" in lib.hb_last_error()


# plane-pass schedule indices grouped by arithmetic family: the parity split (cluster
# split Q x CTA size), the mod-4 split and the mod-8 split (CTA sizes)
@pytest.mark.parametrize("shape,families", [((64, 64, 64), [[0, 1, 2, 3], [4, 5], [6]]),
                                            ((128, 128, 128), [[1, 2, 3, 4, 5], [0, 6, 7], [8, 9]]),
                                            ((96, 96, 32), [[0, 1, 2]]), ((160, 160, 16), [[0, 1]])])
def test_plane_variants_agree(cuda, shape, families, monkeypatch):
    """Every schedule of one family gives bitwise the same result; the families differ
    only by FP32 rounding, and every family matches the FP64 oracle (its complex128 torch
    restatement, on the GPU, at every size)."""
    plan = ToeplitzPlan(shape, cuda)
    coords = synth.kooshball(64, 2 * shape[0])
    packed, Tg = plan.build_diagonal(torch.from_numpy(coords), want_complex=True)
    sm = _c64(synth.coil_maps(2, shape, seed=3), cuda)
    xn = synth.gaussian_image(shape, seed=4)
    x = _c64(xn, cuda)
    outs = {}
    for fam in families:
        for v in fam:
            monkeypatch.setenv("HB_PLANE_VARIANT", str(v))
            out = torch.empty_like(x)
            plan.sense_normal(x, out, sm, packed)
            outs[v] = out
    for fam in families:
        for v in fam[1:]:
            assert torch.equal(outs[fam[0]], outs[v]), v
    first = outs[families[0][0]]
    for v, o in outs.items():
        assert O.rel_l2(_np(o), _np(first)) < 1e-6, v
    ref = O.sense_normal_toeplitz_t(x, sm.to(torch.complex128), Tg.to(torch.complex128))
    for fam in families:
        for v in fam:
            assert O.rel_l2(outs[v], ref) < TOL, (fam, v)


@pytest.mark.parametrize("shape,ncoil", [((96, 96, 96), 3), ((160, 160, 128), 2)])
def test_sense_normal_non_power_of_two(cuda, shape, ncoil):
    """The uneven-batch image sizes (radix-3 and radix-5 FFT lengths) against the FP64 oracle."""
    plan = ToeplitzPlan(shape, cuda)
    coords = synth.kooshball(128, 2 * shape[0])
    packed, Tg = plan.build_diagonal(torch.from_numpy(coords), want_complex=True)
    T = _np(Tg)
    sm = synth.coil_maps(ncoil, shape, seed=11)
    x = synth.gaussian_image(shape, seed=12)
    out = torch.empty(shape, dtype=torch.complex64, device=cuda)
    plan.sense_normal(_c64(x, cuda), out, _c64(sm, cuda), packed, lam=1e-3)
    ref = O.sense_normal_toeplitz(x, sm, T) + 1e-3 * x
    assert O.rel_l2(_np(out), ref) < TOL


def _mixed_jobs(plan, cuda, seeds, ncoils, lam=1e-3):
    from hastycompute_b200.toeplitz import System
    shape = plan.shape
    jobs = []
    for seed, nc in zip(seeds, ncoils):
        rng = np.random.default_rng(seed)
        T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 800)), shape)
        sm = synth.coil_maps(nc + 1, shape, seed=seed)
        coils = list(range(nc + 1))[1:] if nc % 2 else list(range(nc))
        xt = synth.gaussian_image(shape, seed=seed + 100)
        b = O.sense_normal_toeplitz(xt, sm, T, coils) + lam * xt
        jobs.append(dict(T=T, sm=sm, coils=coils, b=b, packed=plan.pack_diagonal(_c64(T, cuda)),
                         smt=_c64(sm, cuda), bt=_c64(b, cuda), lam=lam, x=xt))
    return jobs


def test_heterogeneous_systems_normal_and_cg(cuda):
    """Systems of different jobs (own buffers, coil maps, coil counts, diagonals) in one
    launch sequence, against the FP64 oracle; graph and plain CG agree bitwise."""
    from hastycompute_b200.toeplitz import System
    shape = (16, 16, 32)
    plan = ToeplitzPlan(shape, cuda)
    jobs = _mixed_jobs(plan, cuda, [1, 2, 3], [3, 5, 2])
    # normal op
    systems, outs = [], []
    for j in jobs:
        out = torch.empty(shape, dtype=torch.complex64, device=cuda)
        outs.append(out)
        systems.append(System(_c64(j["x"], cuda), j["smt"], j["packed"], out=out, coils=j["coils"], lam=j["lam"]))
    plan.sense_normal_systems(systems)
    for j, out in zip(jobs, outs):
        assert O.rel_l2(_np(out), j["b"]) < TOL
    # CG, plain and graph-replayed
    res = {}
    for graph in (False, True):
        xs = [torch.zeros(shape, dtype=torch.complex64, device=cuda) for _ in jobs]
        sys_cg = [System(x, j["smt"], j["packed"], b=j["bt"], coils=j["coils"], lam=j["lam"]) for x, j in zip(xs, jobs)]
        status, done = plan.cg_systems(sys_cg, iters=8, graph=graph)
        assert done == [8] * len(jobs)
        res[graph] = xs
    for a, b in zip(res[False], res[True]):
        assert torch.equal(a, b)
    for j, x in zip(jobs, res[True]):
        A = O.regularized(lambda v, j=j: O.sense_normal_toeplitz(v, j["sm"], j["T"], j["coils"]), j["lam"])
        xo, _ = O.conjugate_gradient(A, j["b"], iters=8)
        assert O.rel_l2(_np(x), xo) < 1e-4


def test_result_same_alone_and_in_the_mix(cuda):
    """A job solved alone and solved inside a mix of other jobs gives the same bits."""
    from hastycompute_b200.toeplitz import System
    shape = (32, 32, 32)
    plan = ToeplitzPlan(shape, cuda)
    jobs = _mixed_jobs(plan, cuda, [7, 8, 9, 10], [4, 8, 2, 6])
    def solve(sel, graph):
        xs = {i: torch.zeros(shape, dtype=torch.complex64, device=cuda) for i in sel}
        plan.cg_systems([System(xs[i], jobs[i]["smt"], jobs[i]["packed"], b=jobs[i]["bt"], coils=jobs[i]["coils"],
                                lam=jobs[i]["lam"]) for i in sel], iters=6, graph=graph)
        return xs
    alone = solve([1], graph=False)[1]
    mixed = solve([3, 1, 0, 2], graph=True)[1]
    assert torch.equal(alone, mixed)


def test_autotune_picks_a_schedule_and_keeps_results(cuda):
    shape = (64, 64, 64)
    plan = ToeplitzPlan(shape, cuda)
    coords = synth.kooshball(64, 128)
    packed = plan.build_diagonal(torch.from_numpy(coords))
    sm = _c64(synth.coil_maps(2, shape, seed=3), cuda)
    x = _c64(synth.gaussian_image(shape, seed=4), cuda)
    before = torch.empty_like(x)
    plan.sense_normal(x, before, sm, packed)
    chosen, ms = plan.autotune(nslots=8)
    assert 0 <= chosen < 7 and ms > 0
    after = torch.empty_like(x)
    plan.sense_normal(x, after, sm, packed)
    assert torch.equal(before, after)


def test_cg_host_buffers_match_device_cg(cuda):
    """cg_host (host buffers, copies overlapped with the solves of other groups) gives the
    device CG's result bit for bit."""
    shape = (16, 16, 16)
    coords, x, sm, T = _case(shape, 3, 600, 31)
    plan = ToeplitzPlan(shape, cuda)
    packed = plan.pack_diagonal(_c64(T, cuda))
    rng = np.random.default_rng(32)
    b = (rng.standard_normal((5,) + shape) + 1j * rng.standard_normal((5,) + shape)).astype(np.complex64)
    xd = torch.zeros((5,) + shape, dtype=torch.complex64, device=cuda)
    plan.cg(xd, torch.from_numpy(b).to(cuda), _c64(sm, cuda), packed, iters=6, lam=1e-2)
    xh = torch.zeros((5,) + shape, dtype=torch.complex64).pin_memory()
    out = torch.empty_like(xh).pin_memory()
    st, it = plan.cg_host(xh, torch.from_numpy(b).pin_memory(), _c64(sm, cuda), packed, iters=6, lam=1e-2, chunks=3,
                          out_host=out)
    torch.cuda.synchronize()
    assert it == [6] * 5
    assert torch.equal(out, xd.cpu())
    assert float(xh.abs().max()) == 0.0  # the initial guess is read, not overwritten


def test_bench_unpacks_the_packed_diagonal(cuda):
    """bench.py's accuracy report rebuilds Re(T) from the packed diagonal the plans read;
    it must equal Re(T) of the reference-layout diagonal that was packed."""
    import bench

    shape = (8, 16, 32)
    coords, x, sm, T = _case(shape, 1, 500, 41)
    plan = ToeplitzPlan(shape, cuda)
    packed = plan.pack_diagonal(_c64(T, cuda)).unsqueeze(0)
    got = bench.unpack_diagonal(plan, packed)(0)
    want = torch.from_numpy(T.real.astype(np.float32).astype(np.float64)).to(cuda)
    assert torch.allclose(got.real, want, rtol=1e-6, atol=0) and float(got.imag.abs().max()) == 0.0


def test_x_pass_wait_that_runs_out_is_reported(cuda):
    """Pass C made to wait for a spill tile that is never copied (hb_plan_inject_x_stall:
    a wait that nothing completes): each CTA gives up after about a second and returns
    without its output, the flag reaches the host through hb_wait_status and through the
    CG's own check, and later calls on the same device are correct."""
    shape = (8, 32, 32)  # 16 pass-C CTAs, all resident at once: about two seconds per launch
    rng = np.random.default_rng(61)
    T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 200)), shape)
    sm = synth.coil_maps(2, shape, seed=62)
    x = synth.gaussian_image(shape, seed=63)
    plan = ToeplitzPlan(shape, cuda)
    lib = plan.lib
    packed = plan.pack_diagonal(_c64(T, cuda))
    smt, xt = _c64(sm, cuda), _c64(x, cuda)
    assert lib.hb_plan_inject_x_stall(plan._h, -2) == capi.HB_ERR_INVALID
    capi.check(lib.hb_plan_inject_x_stall(plan._h, 1))
    out = torch.empty_like(xt)
    plan.sense_normal(xt, out, smt, packed)
    with pytest.raises(capi.HastyError) as e:
        plan.wait_status()
    assert e.value.code == capi.HB_ERR_CUDA and "gave up waiting" in str(e.value)
    plan.wait_status()  # read once, then cleared
    b = _c64(O.sense_normal_toeplitz(x, sm, T), cuda)
    with pytest.raises(capi.HastyError) as e:
        plan.cg(torch.zeros_like(b), b, smt, packed, iters=1)
    assert "gave up waiting" in str(e.value)
    capi.check(lib.hb_plan_inject_x_stall(plan._h, -1))
    plan.sense_normal(xt, out, smt, packed)
    plan.wait_status()
    assert O.rel_l2(_np(out), O.sense_normal_toeplitz(x, sm, T)) < TOL
