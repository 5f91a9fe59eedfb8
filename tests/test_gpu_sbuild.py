"""S build in its two device forms: the per-line walk and the line groups (a
unit's lines sharing one list of source cells).  DMRGB200_SBUILD forces one
form for every unit of a plan compiled while it is set; each form is checked
against the CPU oracle (FP64, 1e-12) for H·psi and both boundary steps, and
the grouped form for bitwise reproducibility."""
import numpy as np
import pytest

import oracle as O
from dmrgb200 import engine as E
from dmrgb200 import models as M
from helpers import OracleChain, make_chain, random_psi

TOL = 1e-12

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MODES = ["lines", "groups", "auto"]


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _hpsi(ctx, ch, x, reps=1):
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    xd = E.to_device(x)
    out = []
    for _ in range(reps):
        yd = torch.zeros_like(xd)
        plan.hpsi(xd.data_ptr(), yd.data_ptr())
        torch.cuda.synchronize()
        out.append(yd.cpu().numpy())
    return out


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name,L,m,i", [("qc", 8, 64, 3), ("hubbard", 12, 64, 5), ("heisenberg", 16, 48, 7)])
def test_hpsi_each_sbuild_form(ctx, monkeypatch, mode, name, L, m, i):
    monkeypatch.setenv("DMRGB200_SBUILD", mode)
    model, bonds, tensors, rng = make_chain(name, L, 0, seed=5, synthetic_m=m)
    ch = OracleChain(model, bonds, tensors, i)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    (y,) = _hpsi(ctx, ch, x)
    assert _rel(y, ch.hpsi(x)) <= TOL


def test_grouped_sbuild_bitwise_reproducible(ctx, monkeypatch):
    monkeypatch.setenv("DMRGB200_SBUILD", "groups")
    model, bonds, tensors, rng = make_chain("qc", 8, 0, seed=6, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 3)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    y1, y2 = _hpsi(ctx, ch, x, reps=2)
    assert np.array_equal(y1, y2)


@pytest.mark.parametrize("mode", MODES)
def test_boundary_steps_each_sbuild_form(ctx, monkeypatch, mode):
    monkeypatch.setenv("DMRGB200_SBUILD", mode)
    L = 8
    model, bonds, tensors, rng = make_chain("qc", L, 0, seed=9, synthetic_m=48)
    Lidx = E.edge_bindex(model.symm, bonds[0])
    Lval = Lidx.edge_values()
    Lbuf = E.to_device(Lval)
    for p in range(4):
        W = M.MPOHandle(model.mpo[p], model.symm)
        t = tensors[p]
        sch, nidx = E.schedule_left_step(model.phys, bonds[p], bonds[p + 1], W, Lidx, True)
        ref = O.left_step(sch.plan, Lval, Lidx, t.data, t.left_paired(), nidx)
        nidx2, Lbuf = E.device_left_step(ctx, model.phys, bonds[p], bonds[p + 1], W, Lidx, Lbuf,
                                         E.to_device(t.data), E.to_device(t.left_paired()), True)
        assert _rel(Lbuf.cpu().numpy()[:nidx.n_elems], ref) <= TOL, p
        Lidx, Lval = nidx2, ref
    Ridx = E.edge_bindex(model.symm, bonds[L])
    Rval = Ridx.edge_values()
    Rbuf = E.to_device(Rval)
    for p in range(L - 1, 3, -1):
        W = M.MPOHandle(model.mpo[p], model.symm)
        t = tensors[p]
        sch, nidx = E.schedule_right_step(model.phys, bonds[p], bonds[p + 1], W, Ridx, True)
        ref = O.right_step(sch.plan, Rval, Ridx, t.data, t.data, nidx)
        td = E.to_device(t.data)
        nidx2, Rbuf = E.device_right_step(ctx, model.phys, bonds[p], bonds[p + 1], W, Ridx, Rbuf, td, td, True)
        assert _rel(Rbuf.cpu().numpy()[:nidx.n_elems], ref) <= TOL, p
        Ridx, Rval = nidx2, ref


def test_grouped_sbuild_reads_no_unwritten_scratch(ctx, monkeypatch):
    """T blocks are padded to 32 elements and stage 1 never writes the gaps; the grouped S
    build (its zero-alpha padding sources included) must not read them.  Device memory is
    filled with NaN and handed back to the driver before the plan allocates its scratch, so
    gaps that were read would turn whole lines into NaN."""
    monkeypatch.setenv("DMRGB200_SBUILD", "groups")
    model, bonds, tensors, rng = make_chain("qc", 8, 0, seed=6, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 3)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    poison = torch.full((64 * 1024 * 1024,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    del poison
    torch.cuda.empty_cache()
    y1, y2 = _hpsi(ctx, ch, x, reps=2)
    assert np.isfinite(y1).all() and _rel(y1, ch.hpsi(x)) <= TOL
    assert np.array_equal(y1, y2)
