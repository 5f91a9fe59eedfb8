"""GPU parity at the benchmark sizes: the device H·psi against the reference's own
solver core (tasks.cpp compiled into oracle/_ref; the oracle restatement where it
is absent) on the bench workloads themselves -- config 2 (Fermi-Hubbard L=64,
TwoU1, m=1024, middle pair) and the spin-adapted quantum-chemistry Hamiltonian at
L=16, m=512 (SU2U1) -- within 1e-12 relative."""
import numpy as np
import pytest

import oracle as O
import ref as REF
from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import su2u1 as SU
from helpers import OracleChain

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


def _cpu_hpsi(ch, x):
    if REF.available():
        return REF.Hpsi(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx).run(x)
    return ch.hpsi(x)


def _device_hpsi(ctx, ch, x):
    Lb, Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
    plan = E.DevicePlan(ctx, ch.sched.plan, left_addr=ch.Lidx.cohort_addresses(Lb.data_ptr()),
                        other_addr=ch.Ridx.cohort_addresses(Rb.data_ptr()))
    xd = E.to_device(x)
    yd = torch.zeros_like(xd)
    plan.hpsi(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def test_config2_hubbard_L64_m1024():
    import bench
    ctx = E.Context(0)
    model, bonds, tensors, i, psi = bench.build_workload()
    ch = OracleChain(model, bonds, tensors, i)
    y = _device_hpsi(ctx, ch, psi.data)
    ref = _cpu_hpsi(ch, psi.data)
    assert np.linalg.norm(y - ref) <= TOL * np.linalg.norm(ref)


def test_qc_su2u1_L16_m512():
    ctx = E.Context(0)
    L, m = 16, 512
    h, eri = qc.synthetic_integrals(L)
    model = SU.quantum_chemistry(L, L, 0, h=h, eri=eri)
    bonds = SU.synthetic_bonds(L, (L, 0), m)
    rng = np.random.default_rng(2)
    i = L // 2 - 1
    tensors = G.left_canonicalize(G.right_canonicalize(S.random_mps(SU.PHYS, bonds, rng), 0.0), i, 0.0)
    bonds = [t.left for t in tensors] + [tensors[-1].right]
    ch = OracleChain(model, bonds, tensors, i)
    x = rng.standard_normal(int(ch.sched.plan["in_size"]))
    y = _device_hpsi(ctx, ch, x)
    ref = _cpu_hpsi(ch, x)
    assert np.linalg.norm(y - ref) <= TOL * np.linalg.norm(ref)
