"""GPU tests of the reduced-precision plan (HB_PRECISION_BF16X3): the forward x pass as a
tcgen05 tensor-core contraction with BF16 hi + lo operands and FP32 accumulation.

Tolerances: <= 1e-4 relative L2 against the FP64 oracle (the bar for the reduced-precision
path); against the plan's own FP32 path <= 2e-5 (a numpy emulation of the BF16 hi+lo
three-product contraction gives 3.8e-6 for this transform alone).  The tensor-core pass
needs ny = nx = 128; nz = 16 keeps the oracle cheap."""
import numpy as np
import pytest
import torch

from hastycompute_b200 import capi, synth
from hastycompute_b200.toeplitz import ToeplitzPlan
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (16, 128, 128)
TOL_ORACLE = 1e-4
TOL_FP32 = 2e-5


def _c64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64)).to(dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.complex128)


def _rel(a, b):
    return (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(41)
    Ts = [O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 120)), SHAPE) for _ in range(2)]
    sm = synth.coil_maps(3, SHAPE, seed=42)
    xs = np.stack([synth.gaussian_image(SHAPE, seed=43 + s) for s in range(2)])
    return Ts, sm, xs


def test_precision_switch_and_unsupported_sizes(cuda):
    plan = ToeplitzPlan(SHAPE, cuda)
    assert plan.precision == "fp32"
    plan.set_precision("bf16x3")
    assert plan.precision == "bf16x3"
    plan.set_precision("fp32")
    assert plan.precision == "fp32"
    with pytest.raises(capi.HastyError) as e:
        ToeplitzPlan((16, 16, 16), cuda, precision="bf16x3")
    assert e.value.code == capi.HB_ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        plan.set_precision("fp8")


def test_toeplitz_apply_matches_oracle(cuda, case):
    Ts, _, xs = case
    plan = ToeplitzPlan(SHAPE, cuda, precision="bf16x3")
    packed = plan.pack_diagonal(_c64(Ts[0], cuda))
    xt = _c64(xs[0], cuda)
    xi = xt.clone()
    plan.apply_inplace(xi, packed)  # unit coil map: the pass's multiplier-free branch
    plan.wait_status()
    assert O.rel_l2(_np(xi), O.toeplitz_apply(xs[0], Ts[0])) < TOL_ORACLE


def test_sense_normal_matches_oracle_and_fp32(cuda, case):
    Ts, sm, xs = case
    tc = ToeplitzPlan(SHAPE, cuda, precision="bf16x3")
    fp = ToeplitzPlan(SHAPE, cuda)
    packed = torch.cat([tc.pack_diagonal(_c64(T, cuda)) for T in Ts])
    smt, xt = _c64(sm, cuda), _c64(xs, cuda)
    coils = [2, 0]
    lam = 1e-3
    out_tc = torch.empty_like(xt)
    out_fp = torch.empty_like(xt)
    tc.sense_normal(xt, out_tc, smt, packed, coils=coils, diag_index=[1, 0], lam=lam)
    fp.sense_normal(xt, out_fp, smt, packed, coils=coils, diag_index=[1, 0], lam=lam)
    tc.wait_status()
    for s, d in enumerate([1, 0]):
        ref = O.sense_normal_toeplitz(xs[s], sm, Ts[d], coils) + lam * xs[s]
        assert O.rel_l2(_np(out_tc[s]), ref) < TOL_ORACLE
        assert _rel(out_tc[s], out_fp[s]) < TOL_FP32
    # deterministic: a second call gives the same bits
    again = torch.empty_like(xt)
    tc.sense_normal(xt, again, smt, packed, coils=coils, diag_index=[1, 0], lam=lam)
    assert torch.equal(again, out_tc)


def test_cg_matches_oracle(cuda, case):
    Ts, sm, xs = case
    plan = ToeplitzPlan(SHAPE, cuda, precision="bf16x3")
    packed = torch.cat([plan.pack_diagonal(_c64(T, cuda)) for T in Ts])
    lam, iters = 1e-3, 8
    bs = np.stack([O.sense_normal_toeplitz(xs[s], sm, Ts[s]) + lam * xs[s] for s in range(2)])
    xg = torch.zeros((2,) + SHAPE, dtype=torch.complex64, device=cuda)
    status, done = plan.cg(xg, _c64(bs, cuda), _c64(sm, cuda), packed, iters=iters, lam=lam, diag_index=[0, 1])
    plan.wait_status()
    assert done == [iters, iters]
    for s in range(2):
        A = O.regularized(lambda v, s=s: O.sense_normal_toeplitz(v, sm, Ts[s]), lam)
        xo, _ = O.conjugate_gradient(A, bs[s], iters=iters)
        assert O.rel_l2(_np(xg[s]), xo) < TOL_ORACLE


def test_unaligned_image_and_maps_take_the_narrow_loads(cuda, case):
    """Images and coil maps only 8-byte aligned (complex64 views one element into a
    buffer) go through the pass's 8-byte loads and give the same bits as aligned copies."""
    Ts, sm, xs = case
    plan = ToeplitzPlan(SHAPE, cuda, precision="bf16x3")
    packed = plan.pack_diagonal(_c64(Ts[0], cuda))
    n = int(np.prod(SHAPE))
    xbuf = torch.zeros(n + 1, dtype=torch.complex64, device=cuda)
    xbuf[1:] = _c64(xs[0], cuda).reshape(-1)
    sbuf = torch.zeros(3 * n + 1, dtype=torch.complex64, device=cuda)
    sbuf[1:] = _c64(sm, cuda).reshape(-1)
    x_odd, s_odd = xbuf[1:].view(SHAPE), sbuf[1:].view((3,) + SHAPE)
    assert x_odd.data_ptr() % 16 == 8 and s_odd.data_ptr() % 16 == 8
    out_odd = torch.empty(SHAPE, dtype=torch.complex64, device=cuda)
    out = torch.empty_like(out_odd)
    plan.sense_normal(x_odd, out_odd, s_odd, packed)
    plan.sense_normal(_c64(xs[0], cuda), out, _c64(sm, cuda), packed)
    plan.wait_status()
    assert torch.equal(out_odd, out)
    assert O.rel_l2(_np(out), O.sense_normal_toeplitz(xs[0], sm, Ts[0])) < TOL_ORACLE


def test_cg_systems_that_converge_early_are_skipped(cuda, case):
    """One system converges in the first iterations (identity operator, unit-power maps)
    while the other keeps iterating: later launches skip the converged system's slots."""
    Ts, sm, xs = case
    plan = ToeplitzPlan(SHAPE, cuda, precision="bf16x3")
    T_id = np.ones(plan.grid, np.complex128)
    packed = torch.cat([plan.pack_diagonal(_c64(T_id, cuda)), plan.pack_diagonal(_c64(Ts[1], cuda))])
    # the second right-hand side is scaled so that its residual stays far above the
    # (absolute) tolerance for all 6 iterations (oracle: 6.9 against 0.51 at the last)
    bs = np.stack([xs[0], 1e5 * O.sense_normal_toeplitz(xs[1], sm, Ts[1])])
    x = torch.zeros((2,) + SHAPE, dtype=torch.complex64, device=cuda)
    status, done = plan.cg(x, _c64(bs, cuda), _c64(sm, cuda), packed, iters=6, tol=1e-3 * float(np.linalg.norm(bs[0])),
                           diag_index=[0, 1])
    plan.wait_status()
    assert status[0] == capi.HB_CG_CONVERGED and done[0] <= 2 and done[1] == 6
    assert O.rel_l2(_np(x[0]), xs[0]) < 1e-4
    A = lambda v: O.sense_normal_toeplitz(v, sm, Ts[1])
    xo, _ = O.conjugate_gradient(A, bs[1], iters=6)
    assert O.rel_l2(_np(x[1]), xo) < TOL_ORACLE


def test_a_wait_that_runs_out_is_reported_and_the_device_stays_usable(cuda):
    """A wait made to run out (the plan omits one DFT-table copy, so nothing completes that
    wait): each CTA gives up after about a second and returns without its output, the flag
    reaches the host through hb_wait_status and through the CG's own check, and later calls
    on the same device are correct."""
    shape = (8, 128, 128)  # 8 CTAs per slot: about one second per stalled launch
    rng = np.random.default_rng(51)
    T = O.toeplitz_diagonal(rng.uniform(-np.pi, np.pi, (3, 100)), shape)
    sm = synth.coil_maps(1, shape, seed=52)
    x = synth.gaussian_image(shape, seed=53)
    plan = ToeplitzPlan(shape, cuda, precision="bf16x3")
    lib = plan.lib
    packed = plan.pack_diagonal(_c64(T, cuda))
    assert lib.hb_plan_inject_tc_stall(plan._h, 8) == capi.HB_ERR_INVALID
    capi.check(lib.hb_plan_inject_tc_stall(plan._h, 3))
    xi = _c64(x, cuda)
    plan.apply_inplace(xi, packed)
    with pytest.raises(capi.HastyError) as e:
        plan.wait_status()
    assert e.value.code == capi.HB_ERR_CUDA and "gave up waiting" in str(e.value)
    plan.wait_status()  # read once, then cleared
    b = _c64(O.sense_normal_toeplitz(x, sm, T), cuda)
    with pytest.raises(capi.HastyError) as e:
        plan.cg(torch.zeros_like(b), b, _c64(sm, cuda), packed, iters=1)
    assert "gave up waiting" in str(e.value)
    capi.check(lib.hb_plan_inject_tc_stall(plan._h, -1))
    xi = _c64(x, cuda)
    plan.apply_inplace(xi, packed)
    plan.wait_status()
    assert O.rel_l2(_np(xi), O.toeplitz_apply(x, T)) < TOL_ORACLE
