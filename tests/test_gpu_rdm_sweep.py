"""Integral derivatives of a whole MPS by moving the centre (dmrgb200.rdm) on the
device (boundary steps, splits and dmrgb200_hpsi_adjoint), against the same sweep on
the CPU oracle and against dense RDM elements."""
import numpy as np
import pytest

from dmrgb200 import dmrg as G
from dmrgb200 import engine as E
from dmrgb200 import mps as S
from dmrgb200 import qc
from dmrgb200 import rdm
from sweep_backend import OracleBackend
from test_rdm_sweep import INTEGRALS, dense_derivatives

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_device_integral_derivatives_over_the_chain():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    ctx = E.Context(0)
    L = 5
    model = qc.quantum_chemistry(L, 2, 2)
    tensors = S.random_mps(model.phys, S.allowed_sectors(model.phys, L, model.total_charge, 16),
                           np.random.default_rng(7))
    dev = rdm.integral_derivatives(G.DeviceBackend(ctx), model, tensors, INTEGRALS)
    cpu = rdm.integral_derivatives(OracleBackend(), model, tensors, INTEGRALS)
    want = dense_derivatives(model, tensors, L)
    for key in INTEGRALS:
        assert abs(dev[key] - cpu[key]) <= 1e-12 * max(1.0, abs(cpu[key])), (key, dev[key], cpu[key])
        assert abs(dev[key] - want[key]) <= 1e-11 * max(1.0, abs(want[key])), (key, dev[key], want[key])
