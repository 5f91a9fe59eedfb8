"""GPU parity: the sm_100a kernels behind the C ABI against the CPU oracle on
identical inputs (FP64: relative error <= 1e-12 per H·psi and per boundary)."""
import numpy as np
import pytest

from dmrgb200 import engine as E
from dmrgb200 import models as M
from helpers import OracleChain, make_chain, random_psi

import oracle as O

TOL = 1e-12

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _gpu_hpsi(ctx, ch, x):
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    plan.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    return yd.cpu().numpy(), (plan, Lb, Rb, xd, yd)


@pytest.mark.parametrize("name,L,Mmax", [("heisenberg", 8, 6), ("hubbard", 6, 8), ("bose", 6, 4)])
def test_hpsi_every_site(ctx, name, L, Mmax):
    model, bonds, tensors, rng = make_chain(name, L, Mmax, seed=21)
    for i in range(L - 1):
        ch = OracleChain(model, bonds, tensors, i)
        x = random_psi(ch.p12, ch.left, ch.right, rng).data
        y, _ = _gpu_hpsi(ctx, ch, x)
        assert _rel(y, ch.hpsi(x)) <= TOL, (name, i)


@pytest.mark.parametrize("name,L,m", [("hubbard", 16, 96), ("heisenberg", 24, 64), ("bose", 12, 64)])
def test_hpsi_synthetic_bond_dimension(ctx, name, L, m):
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=7, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, L // 2 - 1)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y, _ = _gpu_hpsi(ctx, ch, x)
    assert _rel(y, ch.hpsi(x)) <= TOL


def test_hpsi_bitwise_reproducible(ctx):
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=4, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 5)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y1, keep = _gpu_hpsi(ctx, ch, x)
    plan, Lb, Rb, xd, yd = keep
    yd.zero_()
    plan.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(y1, yd.cpu().numpy())


@pytest.mark.parametrize("symmetric", [True, False])
def test_boundary_steps_match_oracle(ctx, symmetric):
    model, bonds, tensors, rng = make_chain("hubbard", 10, 0, seed=9, synthetic_m=48)
    # left chain on the device vs the oracle, step by step
    Lidx = E.edge_bindex(model.symm, bonds[0])
    Lval = Lidx.edge_values()
    Lbuf = E.to_device(Lval)
    for p in range(6):
        W = M.MPOHandle(model.mpo[p], model.symm)
        t = tensors[p]
        sch, nidx = E.schedule_left_step(model.phys, bonds[p], bonds[p + 1], W, Lidx, symmetric)
        ref = O.left_step(sch.plan, Lval, Lidx, t.data, t.left_paired(), nidx)
        nidx2, Lbuf = E.device_left_step(ctx, model.phys, bonds[p], bonds[p + 1], W, Lidx, Lbuf,
                                         E.to_device(t.data), E.to_device(t.left_paired()), symmetric)
        got = Lbuf.cpu().numpy()[:nidx.n_elems]
        assert _rel(got, ref) <= TOL, p
        Lidx, Lval = nidx2, ref
    Ridx = E.edge_bindex(model.symm, bonds[10])
    Rval = Ridx.edge_values()
    Rbuf = E.to_device(Rval)
    for p in range(9, 4, -1):
        W = M.MPOHandle(model.mpo[p], model.symm)
        t = tensors[p]
        sch, nidx = E.schedule_right_step(model.phys, bonds[p], bonds[p + 1], W, Ridx, symmetric)
        ref = O.right_step(sch.plan, Rval, Ridx, t.data, t.data, nidx)
        td = E.to_device(t.data)
        nidx2, Rbuf = E.device_right_step(ctx, model.phys, bonds[p], bonds[p + 1], W, Ridx, Rbuf, td, td, symmetric)
        got = Rbuf.cpu().numpy()[:nidx.n_elems]
        assert _rel(got, ref) <= TOL, p
        Ridx, Rval = nidx2, ref


def test_site_problem_end_to_end(ctx):
    """Boundaries and H·psi entirely on the device vs the oracle chain."""
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=13, synthetic_m=64)
    sp = E.SiteProblem(ctx, model, tensors, bonds, 5)
    ch = OracleChain(model, bonds, tensors, 5)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    sp.hpsi(xd, yd)
    torch.cuda.synchronize()
    assert _rel(yd.cpu().numpy(), ch.hpsi(x)) <= TOL


def test_stage_timing_reports(ctx):
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=1, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 5)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    _, keep = _gpu_hpsi(ctx, ch, x)
    plan, Lb, Rb, xd, yd = keep
    import ctypes as C
    from dmrgb200 import _capi as capi
    capi.check(capi.lib.dmrgb200_plan_set_timing(plan.handle, 1), "timing")
    for _ in range(3):
        plan.hpsi(xd.data_ptr(), yd.data_ptr())
    ms = (C.c_double * 3)()
    fl = (C.c_uint64 * 3)()
    calls = C.c_uint64()
    capi.check(capi.lib.dmrgb200_plan_stage_times(plan.handle, ms, fl, C.byref(calls)), "stage_times")
    assert calls.value == 3 and all(v > 0 for v in ms) and sum(fl) == plan.flops


def test_autotuned_variants_give_identical_results(ctx):
    """Every grouped-GEMM variant sums in the same order: H·psi after an explicit
    re-tune (whatever variants it picks) equals the default-variant result bitwise."""
    import ctypes as C

    from dmrgb200 import _capi as capi
    model, bonds, tensors, rng = make_chain("hubbard", 16, 0, seed=17, synthetic_m=96)
    ch = OracleChain(model, bonds, tensors, 7)
    y0, keep = _gpu_hpsi(ctx, ch, random_psi(ch.p12, ch.left, ch.right, rng).data)
    plan, Lb, Rb, xd, yd = keep
    chosen = (C.c_int32 * 2)()
    capi.check(capi.lib.dmrgb200_plan_autotune(plan.handle, xd.data_ptr(), yd.data_ptr(), None, chosen), "autotune")
    assert all(0 <= v < capi.lib.dmrgb200_gemm_variant_count() for v in chosen)
    assert capi.lib.dmrgb200_gemm_variant_name(chosen[0]).startswith(b"tile")
    yd.zero_()
    plan.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(y0, yd.cpu().numpy())


@pytest.mark.parametrize("name,L,m", [("hubbard", 16, 96), ("qc", 8, 64)])
def test_hpsi_host_buffers_bitwise_equal(ctx, name, L, m):
    """dmrgb200_hpsi_host (pinned host x and y, copies overlapped with the split
    stages) gives bitwise the device H·psi, repeatedly."""
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=8, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, L // 2 - 1)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y_dev, keep = _gpu_hpsi(ctx, ch, x)
    plan = keep[0]
    xh = torch.from_numpy(x.copy()).pin_memory()
    for _ in range(2):
        yh = torch.full((len(x),), float("nan"), dtype=torch.float64).pin_memory()
        plan.hpsi_host(xh.data_ptr(), yh.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(yh.numpy(), y_dev)
    assert _rel(y_dev, ch.hpsi(x)) <= TOL


def test_hpsi_host_pageable_buffers(ctx):
    """dmrgb200_hpsi_host also takes pageable host memory (no overlap then)."""
    model, bonds, tensors, rng = make_chain("hubbard", 12, 0, seed=9, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 5)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y_dev, keep = _gpu_hpsi(ctx, ch, x)
    xh = np.ascontiguousarray(x)
    yh = np.full(len(x), np.nan)
    keep[0].hpsi_host(xh.ctypes.data, yh.ctypes.data)
    torch.cuda.synchronize()
    assert np.array_equal(yh, y_dev)


@pytest.mark.parametrize("name,L,m", [("hubbard", 16, 96), ("qc", 8, 48)])
def test_per_block_launch_path_matches(ctx, name, L, m):
    """The reference-style launch pattern (one library GEMM per T task and per cohort,
    dmrgb200_hpsi_per_block) computes the same H·psi as the grouped kernels."""
    import ctypes as C
    from dmrgb200 import _capi as capi
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=12, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, L // 2 - 1)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y, keep = _gpu_hpsi(ctx, ch, x)
    plan, Lb, Rb, xd, yd = keep
    yp = torch.full_like(xd, float("nan"))
    n = C.c_uint64()
    capi.check(capi.lib.dmrgb200_hpsi_per_block(plan.handle, xd.data_ptr(), yp.data_ptr(), None, C.byref(n)),
               "dmrgb200_hpsi_per_block")
    torch.cuda.synchronize()
    mask = np.zeros(len(y), dtype=bool)
    for off, r, c in zip(ch.sched.plan["out_off"], ch.sched.plan["out_rows"], ch.sched.plan["out_cols"]):
        mask[int(off):int(off) + int(r) * int(c)] = True
    got = yp.cpu().numpy()
    assert _rel(got[mask], y[mask]) <= TOL
    assert n.value >= len(ch.sched.plan["t_lb"]) + 1
