"""The split's density matrix with the state prediction on the device
(dmrgb200_step_alpha_dm) against the oracle on identical inputs (FP64, relative
error <= 1e-12), and perturbed device sweeps against perturbed oracle sweeps and
exact diagonalisation."""
import numpy as np
import pytest

import dense
import oracle as O
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import models as M
from sweep_backend import OracleBackend
from test_alpha_dm import site_pair

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


@pytest.mark.parametrize("name", ["heisenberg", "hubbard", "su2u1"])
@pytest.mark.parametrize("left", [True, False])
def test_device_alpha_dm_matches_oracle(ctx, name, left):
    model, ch, psi, i = site_pair(name, L=10, m=48)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    t, _ = G.theta_site(psi, model.phys, model.phys, offs, left)
    be = G.DeviceBackend(ctx)
    if left:
        W = M.MPOHandle(model.mpo[i], model.symm)
        Bidx, Bval = ch.Lidx, ch.Lval
    else:
        W = M.MPOHandle(model.mpo[i + 1], model.symm)
        Bidx, Bval = ch.Ridx, ch.Rval
    got = be.alpha_dm(model.phys, W, Bidx, E.to_device(Bval), t, 0.25, left)
    want = OracleBackend().alpha_dm(model.phys, W, Bidx, Bval, t, 0.25, left)
    num = sum(float(np.linalg.norm(a - b) ** 2) for a, b in zip(got, want))
    den = sum(float(np.linalg.norm(b) ** 2) for b in want)
    assert len(got) == len(want) and den > 0 and np.sqrt(num / den) <= 1e-12, np.sqrt(num / den)


def test_perturbed_device_sweeps_match_oracle_sweeps(ctx):
    L = 10
    model = M.heisenberg(L)
    from dmrgb200 import mps as S
    A = S.random_mps(model.phys, S.allowed_sectors(model.phys, L, model.total_charge, 2), np.random.default_rng(3))
    alpha = lambda sweep: 1e-3 if sweep < 2 else 0.0
    dev = G.TwoSiteDMRG(G.DeviceBackend(ctx), model, list(A), 32, jd_tol=1e-10, jd_maxiter=16, alpha=alpha)
    cpu = G.TwoSiteDMRG(OracleBackend(), model, list(A), 32, jd_tol=1e-10, jd_maxiter=16, alpha=alpha)
    for sw in range(4):
        dev.sweep(sw)
        cpu.sweep(sw)
    ed = np.array([x[2] for x in dev.log.energies])
    ec = np.array([x[2] for x in cpu.log.energies])
    assert np.abs(ed - ec).max() <= 1e-9
    assert abs(ed[-1] - dense.ground_energy(model, L)) <= 1e-9


def test_alpha_dm_rejects_bad_arguments(ctx):
    """dmrgb200_step_alpha_dm checks its arguments before any device work: alpha < 0, an
    H·psi plan, and a dm view with a missing block are rejected with their status."""
    from dmrgb200 import _capi as capi
    model, ch, psi, i = site_pair("heisenberg", L=8, m=16)
    p12, offs = M.fuse_phys(model.phys, model.phys)
    t, _ = G.theta_site(psi, model.phys, model.phys, offs, True)
    W = M.MPOHandle(model.mpo[i], model.symm)
    sch, _ = E.schedule_left_step(model.phys, t.left, t.right, W, ch.Lidx, False)
    Lb = E.to_device(ch.Lval)
    plan = E.DevicePlan(ctx, sch.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()))
    ket, bra = E.to_device(t.data), E.to_device(t.left_paired())
    dims = [int(r) for r in sch.plan["out_rows"]]
    store = torch.zeros(sum(d * d for d in dims) + 1, dtype=torch.float64, device="cuda")
    offs_ = np.concatenate([[0], np.cumsum([d * d for d in dims])])
    addr = np.array([store.data_ptr() + 8 * int(o) for o in offs_[:-1]], dtype=np.uint64)
    with pytest.raises(capi.DmrgError) as e1:
        plan.alpha_dm(ket.data_ptr(), bra.data_ptr(), addr, -1.0)
    assert e1.value.status == capi.INVALID_ARGUMENT
    bad = addr.copy()
    bad[int(np.argmax(dims))] = 0
    with pytest.raises(capi.DmrgError) as e2:
        plan.alpha_dm(ket.data_ptr(), bra.data_ptr(), bad, 0.5)
    assert e2.value.status == capi.INVALID_ARGUMENT
    hp = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                      other_addr=ch.Ridx.cohort_addresses(E.to_device(ch.Rval).data_ptr()))
    with pytest.raises(capi.DmrgError) as e3:
        hp.alpha_dm(ket.data_ptr(), bra.data_ptr(), addr, 0.5)
    assert e3.value.status == capi.INVALID_PLAN
    plan.alpha_dm(ket.data_ptr(), bra.data_ptr(), addr, 0.5)  # the plan still works
    torch.cuda.synchronize()
