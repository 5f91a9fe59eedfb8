"""Two-site DMRG sweeps on the device path reach exact ground-state energies,
including the reference's coded Bose-Hubbard known answer
(dmrg/regression/applications/dmrg/test_coded_bh_ts.py:16-53:
L=10, Nmax=2, t=1, U=8, N=5, m=200, E = -6.881090360639349 within 1e-3)."""
import numpy as np
import pytest

import dense as D
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import models as M
from dmrgb200 import mps as S

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

E_BH_REFERENCE = -6.881090360639349


def _run(model, L, m, sweeps, seed=1, init_m=5):
    ctx = E.Context(0)
    rng = np.random.default_rng(seed)
    bonds = S.allowed_sectors(model.phys, L, model.total_charge, init_m)
    A = S.random_mps(model.phys, bonds, rng)
    opt = G.TwoSiteDMRG(G.DeviceBackend(ctx), model, A, m, cutoff=1e-16, jd_tol=1e-10, jd_maxiter=16)
    e = None
    for s in range(sweeps):
        e = opt.sweep(s)
    return e, opt


def test_bose_hubbard_known_answer():
    model = M.bose_hubbard(10, t=1.0, U=8.0, Nmax=2, N=5)
    e, opt = _run(model, 10, 200, 5)
    assert abs(e - E_BH_REFERENCE) <= 1e-3
    e_exact = D.ground_energy(model, 10)
    assert abs(e - e_exact) <= 1e-8


@pytest.mark.parametrize("name,L,m", [("heisenberg", 10, 32), ("hubbard", 6, 64)])
def test_sweeps_reach_exact_ground_state(name, L, m):
    model = M.heisenberg(L) if name == "heisenberg" else M.fermi_hubbard(L)
    e, opt = _run(model, L, m, 3)
    assert abs(e - D.ground_energy(model, L)) <= 1e-9


def test_device_sweep_matches_oracle_sweep():
    """A whole two-site sweep on the device path against the same sweep replayed
    on the CPU oracle (reference JD restatement + oracle H·psi and boundary
    steps): per-site energies within 1e-9."""
    from sweep_backend import OracleBackend
    model = M.fermi_hubbard(10)
    rng = np.random.default_rng(4)
    bonds = S.allowed_sectors(model.phys, 10, model.total_charge, 5)
    A = S.random_mps(model.phys, bonds, rng)
    dev = G.TwoSiteDMRG(G.DeviceBackend(E.Context(0)), model, [t for t in A], 32, jd_tol=1e-8, jd_maxiter=8)
    cpu = G.TwoSiteDMRG(OracleBackend(), model, [t for t in A], 32, jd_tol=1e-8, jd_maxiter=8)
    for s in range(2):
        dev.sweep(s)
        cpu.sweep(s)
    ed = np.array([e[2] for e in dev.log.energies])
    ec = np.array([e[2] for e in cpu.log.energies])
    assert np.max(np.abs(ed - ec)) <= 1e-9


def test_device_split_sweeps():
    """Sweeps whose splits run on the device (split_device): the Bose-Hubbard
    known answer with truncation to m=200, and the same energies as the sweeps
    with host SVDs within 1e-8."""
    model = M.bose_hubbard(10, t=1.0, U=8.0, Nmax=2, N=5)
    res = {}
    for dsplit in (False, True):
        rng = np.random.default_rng(1)
        bonds = S.allowed_sectors(model.phys, 10, model.total_charge, 5)
        A = S.random_mps(model.phys, bonds, rng)
        opt = G.TwoSiteDMRG(G.DeviceBackend(E.Context(0)), model, A, 200, cutoff=1e-16, jd_tol=1e-10, jd_maxiter=16,
                            device_split=dsplit)
        for s in range(5):
            e = opt.sweep(s)
        res[dsplit] = e
    assert abs(res[True] - E_BH_REFERENCE) <= 1e-3
    assert abs(res[True] - res[False]) <= 1e-8
    assert abs(res[True] - D.ground_energy(model, 10)) <= 1e-8
