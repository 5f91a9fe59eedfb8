"""Emulated FP64 inside the eigen-solve and the sweeps: the H·psi contractions on
the INT8 tensor cores (dmrgb200_plan_set_precision), everything else of the
Jacobi-Davidson in native FP64; the slice count from an error target
(dmrgb200_plan_tune_slices); stream-ordered emulated H·psi whose device error
words are read by dmrgb200_plan_check.  Energies must stay within 1e-9 of the
FP64 path, per H·psi the emulation tolerance 1e-10."""
import numpy as np
import pytest

import dense
from dmrgb200 import _capi as capi
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import models as M
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import su2u1 as SU
from helpers import random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


def site_problem(ctx, L=16, m=96, seed=3):
    model = M.fermi_hubbard(L)
    rng = np.random.default_rng(seed)
    bonds = [S.synthetic_sectors(model.phys, L, model.total_charge, m, i) for i in range(L + 1)]
    i = L // 2 - 1
    A = G.left_canonicalize(G.right_canonicalize(S.random_mps(model.phys, bonds, rng), 0.0), i, 0.0)
    bonds = [t.left for t in A] + [A[-1].right]
    sp = E.SiteProblem(ctx, model, A, bonds, i)
    x = random_psi(sp.p12, sp.left, sp.right, rng).data
    return sp, x / np.linalg.norm(x)


def test_emulated_hpsi_stream_ordered_and_checked(ctx):
    sp, x = site_problem(ctx)
    xd = E.to_device(x)
    y64, ye = torch.zeros_like(xd), torch.zeros_like(xd)
    sp.plan.hpsi(xd.data_ptr(), y64.data_ptr())
    for _ in range(3):  # no synchronisation inside the calls
        sp.plan.hpsi(xd.data_ptr(), ye.data_ptr(), capi.PREC_FP64_EMULATED)
    sp.plan.check()
    err = float(torch.linalg.norm(ye - y64) / torch.linalg.norm(y64))
    assert err <= 1e-10, err


def test_tune_slices_meets_the_target(ctx):
    sp, x = site_problem(ctx)
    xd = E.to_device(x)
    s_tight, e_tight = sp.plan.tune_slices(xd.data_ptr(), 1e-12)
    assert e_tight <= 1e-12 and 3 <= s_tight <= 8
    s_loose, e_loose = sp.plan.tune_slices(xd.data_ptr(), 1e-6)
    assert e_loose <= 1e-6 and s_loose < s_tight
    # the kept count is the last tuned one: the emulated H·psi now has the loose error
    y64, ye = torch.zeros_like(xd), torch.zeros_like(xd)
    sp.plan.hpsi(xd.data_ptr(), y64.data_ptr())
    sp.plan.hpsi(xd.data_ptr(), ye.data_ptr(), capi.PREC_FP64_EMULATED)
    sp.plan.check()
    err = float(torch.linalg.norm(ye - y64) / torch.linalg.norm(y64))
    assert abs(err - e_loose) <= 1e-3 * e_loose + 1e-15


@pytest.mark.parametrize("mode", [capi.SOLVER_GRAPH, capi.SOLVER_STEPWISE])
def test_emulated_solve_energy_within_1e9(ctx, mode):
    sp, x = site_problem(ctx)
    xd = E.to_device(x)
    xo = torch.zeros_like(xd)
    sp.plan.set_solver(mode)
    e64, st64 = sp.plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-10, max_iter=24)
    s, err = sp.plan.tune_slices(xd.data_ptr(), 1e-10)
    sp.plan.set_precision(capi.PREC_FP64_EMULATED)
    ee, ste = sp.plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-10, max_iter=24)
    sp.plan.set_precision(capi.PREC_FP64)
    assert abs(ee - e64) <= 1e-9 * max(1.0, abs(e64)), (ee, e64, s, err)


def test_emulated_sweeps_match_fp64_sweeps(ctx):
    """Heisenberg L=12 (U1), m=32: the per-site energies of emulated and FP64 device
    sweeps within 1e-9; the final one within 1e-9 of exact diagonalisation."""
    L = 12
    model = M.heisenberg(L)
    A = S.random_mps(model.phys, S.allowed_sectors(model.phys, L, model.total_charge, 5), np.random.default_rng(1))
    runs = {}
    for name, prec in (("fp64", capi.PREC_FP64), ("emulated", capi.PREC_FP64_EMULATED)):
        be = G.DeviceBackend(ctx, precision=prec)
        dm = G.TwoSiteDMRG(be, model, list(A), 32, jd_tol=1e-10, jd_maxiter=16)
        for sw in range(3):
            dm.sweep(sw)
        runs[name] = np.array([e[2] for e in dm.log.energies])
        if name == "emulated":
            assert all(err <= 1e-10 for _, err in be.slices_used)
    assert np.abs(runs["emulated"] - runs["fp64"]).max() <= 1e-9
    assert abs(runs["emulated"][-1] - dense.ground_energy(model, L)) <= 1e-9


def test_emulated_su2u1_sweep_reaches_fci(ctx):
    L, n = 6, 6
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n, 0, h=h, eri=eri)
    A = S.random_mps(SU.PHYS, SU.allowed_sectors(L, (n, 0), 3), np.random.default_rng(2))
    dm = G.TwoSiteDMRG(G.DeviceBackend(ctx, precision=capi.PREC_FP64_EMULATED), model, list(A), 100, jd_tol=1e-10,
                       jd_maxiter=12)
    for sw in range(3):
        e = dm.sweep(sw)
    assert abs(e - dense.spin_sector_spectrum(h, eri, n, 0)[0]) <= 1e-9
