"""GPU parity for the spin-adapted (SU2U1) quantum-chemistry path: the device
H·psi, boundary steps, Jacobi-Davidson solve and sweeps against the CPU oracle on
identical inputs (FP64: relative error <= 1e-12), the emulated H·psi within the
emulation tolerance, and eigenvalues / sweep energies against the FCI spectrum
of the spin sector (oracle/dense.py spin_sector_spectrum)."""
import numpy as np
import pytest

import dense
import oracle as O
from dmrgb200 import _capi as capi
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import su2u1 as SU
from helpers import OracleChain, random_psi

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def synthetic_chain(L, m, seed=11):
    model = SU.quantum_chemistry(L, L, 0)
    bonds = SU.synthetic_bonds(L, (L, 0), m)
    rng = np.random.default_rng(seed)
    A = S.random_mps(SU.PHYS, bonds, rng)
    return model, bonds, A, rng


@pytest.mark.parametrize("L,m", [(8, 48), (12, 128)])
def test_hpsi_and_boundaries_match_oracle(ctx, L, m):
    """Boundaries built by device steps (SiteProblem) and by oracle steps (OracleChain)
    from the same tensors, then H·psi on the device against the oracle's."""
    model, bonds, A, rng = synthetic_chain(L, m)
    i = L // 2 - 1
    ch = OracleChain(model, bonds, A, i)
    sp = E.SiteProblem(ctx, model, A, bonds, i)
    assert _rel(sp.Lbuf.cpu().numpy(), ch.Lval) <= TOL
    assert _rel(sp.Rbuf.cpu().numpy(), ch.Rval) <= TOL
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    sp.plan.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    assert _rel(yd.cpu().numpy(), ch.hpsi(x)) <= TOL


def test_emulated_hpsi_within_emulation_tolerance(ctx):
    model, bonds, A, rng = synthetic_chain(10, 96)
    sp = E.SiteProblem(ctx, model, A, bonds, 4)
    x = torch.tensor(rng.standard_normal(sp.size), dtype=torch.float64, device="cuda")
    y64, yem = torch.zeros_like(x), torch.zeros_like(x)
    sp.plan.hpsi(x.data_ptr(), y64.data_ptr())
    sp.plan.hpsi(x.data_ptr(), yem.data_ptr(), capi.PREC_FP64_EMULATED)
    torch.cuda.synchronize()
    err = float(torch.linalg.norm(yem - y64) / torch.linalg.norm(y64))
    assert err <= 1e-10, err


def test_device_solve_gives_fci_ground_energy(ctx):
    """Complete bond spaces, mixed-canonical environment: the device JD's lowest
    eigenvalue of H_eff is the FCI singlet ground energy."""
    L, n = 6, 6
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n, 0, h=h, eri=eri)
    A = S.random_mps(SU.PHYS, SU.allowed_sectors(L, (n, 0), 10 ** 6), np.random.default_rng(3))
    i = L // 2 - 1
    A = G.left_canonicalize(G.right_canonicalize(A), i)
    bonds = [t.left for t in A] + [A[-1].right]
    sp = E.SiteProblem(ctx, model, A, bonds, i)
    x0 = random_psi(sp.p12, sp.left, sp.right, np.random.default_rng(4)).data
    x0 /= np.linalg.norm(x0)
    xd = E.to_device(x0)
    xo = torch.zeros_like(xd)
    e, st = sp.plan.solve(xd.data_ptr(), xo.data_ptr(), xd.numel(), tol=1e-12, max_iter=32)
    e0 = dense.spin_sector_spectrum(h, eri, n, 0)[0]
    assert abs(e - e0) <= 1e-9, (e, e0, st.iterations)


def test_device_sweeps_reach_fci_and_match_oracle_sweep(ctx):
    L, n = 6, 6
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, n, 0, h=h, eri=eri)
    A = S.random_mps(SU.PHYS, SU.allowed_sectors(L, (n, 0), 3), np.random.default_rng(2))
    from sweep_backend import OracleBackend
    dev = G.TwoSiteDMRG(G.DeviceBackend(ctx), model, list(A), 100, jd_tol=1e-10, jd_maxiter=12)
    cpu = G.TwoSiteDMRG(OracleBackend(), model, list(A), 100, jd_tol=1e-10, jd_maxiter=12)
    for sw in range(2):
        dev.sweep(sw)
        cpu.sweep(sw)
    ed = np.array([x[2] for x in dev.log.energies])
    ec = np.array([x[2] for x in cpu.log.energies])
    assert np.abs(ed - ec).max() <= 1e-9
    assert abs(ed[-1] - dense.spin_sector_spectrum(h, eri, n, 0)[0]) <= 1e-9
