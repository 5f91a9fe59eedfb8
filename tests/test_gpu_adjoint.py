"""GPU adjoint of H·psi (dmrgb200_hpsi_adjoint) against the CPU oracle, and the
derivative of E = <psi|H|psi>/<psi|psi> through a torch.autograd.Function that
wraps the C ABI (test harness only), checked by central finite differences and
by the local RDM elements of the dense Hamiltonian."""
import dataclasses

import numpy as np
import pytest

from dmrgb200 import engine as E
from helpers import OracleChain, hubbard_center_terms, hubbard_derivative_ops, make_chain, random_psi, unit_mask

import dense as D
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return E.Context(0)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


class DeviceChain:
    """Oracle boundaries uploaded once; device plans per set of term alphas."""

    def __init__(self, ctx, ch):
        self.ctx, self.ch = ctx, ch
        self.Lb, self.Rb = E.to_device(ch.Lval), E.to_device(ch.Rval)
        self._plans = {}

    def plan(self, alpha=None):
        key = None if alpha is None else np.asarray(alpha, dtype=np.float64).tobytes()
        if key not in self._plans:
            p = dict(self.ch.sched.plan)
            if alpha is not None:
                p["term_alpha"] = np.array(alpha, dtype=np.float64)
            self._plans[key] = E.DevicePlan(self.ctx, p, left_addr=self.ch.Lidx.cohort_addresses(self.Lb.data_ptr()),
                                            other_addr=self.ch.Ridx.cohort_addresses(self.Rb.data_ptr()))
        return self._plans[key]

    def adjoint(self, w, x, want_gx=True, want_ga=True, plan=None):
        plan = plan or self.plan()
        wd, xd = E.to_device(w), E.to_device(x)
        gx = torch.full_like(xd, float("nan")) if want_gx else None
        ga = torch.full((len(plan.plan["term_alpha"]),), float("nan"), dtype=torch.float64,
                        device="cuda") if want_ga else None
        plan.adjoint(wd.data_ptr(), xd.data_ptr(), gx.data_ptr() if want_gx else 0, ga.data_ptr() if want_ga else 0)
        torch.cuda.synchronize()
        return (gx.cpu().numpy() if want_gx else None), (ga.cpu().numpy() if want_ga else None)


class Hpsi(torch.autograd.Function):
    """y = H(alpha) x on the device; backward through dmrgb200_hpsi_adjoint."""

    @staticmethod
    def forward(fctx, x, alpha, chain):
        plan = chain.plan(alpha.detach().cpu().numpy())
        y = torch.zeros_like(x)
        plan.hpsi(x.data_ptr(), y.data_ptr())
        fctx.save_for_backward(x, alpha)
        fctx.chain = chain
        return y

    @staticmethod
    def backward(fctx, gy):
        x, alpha = fctx.saved_tensors
        plan = fctx.chain.plan(alpha.detach().cpu().numpy())
        gy = gy.contiguous()
        gx, ga = torch.empty_like(x), torch.empty_like(alpha)
        plan.adjoint(gy.data_ptr(), x.data_ptr(), gx.data_ptr(), ga.data_ptr())
        return gx, ga, None


def _energy(chain, x, alpha):
    y = Hpsi.apply(x, alpha, chain)
    return (x @ y) / (x @ x)


@pytest.mark.parametrize("name,L,m,i", [("hubbard", 8, 0, 3), ("heisenberg", 10, 0, 4), ("bose", 6, 0, 2),
                                        ("hubbard", 16, 128, 7), ("heisenberg", 24, 96, 11)])
def test_adjoint_matches_oracle(ctx, name, L, m, i):
    model, bonds, tensors, rng = make_chain(name, L, 8, seed=31, synthetic_m=m or None)
    ch = OracleChain(model, bonds, tensors, i)
    dc = DeviceChain(ctx, ch)
    w = random_psi(ch.p12, ch.left, ch.right, rng).data
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    gx, ga = dc.adjoint(w, x)
    gx_o, ga_o = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, w, x)
    assert _rel(gx, gx_o) <= TOL
    assert _rel(ga, ga_o) <= TOL
    # the two outputs alone, and a second call: bitwise identical
    gx2, _ = dc.adjoint(w, x, want_ga=False)
    _, ga2 = dc.adjoint(w, x, want_gx=False)
    assert np.array_equal(gx, gx2) and np.array_equal(ga, ga2)


@pytest.mark.parametrize("mode", ["lines", "groups", "auto"])
def test_adjoint_qc_each_sbuild_form(ctx, monkeypatch, mode):
    """Quantum chemistry: galpha from the line groups' Gram blocks (grouped units) and
    term by term (the others) against the oracle, and bitwise repeatable."""
    monkeypatch.setenv("DMRGB200_SBUILD", mode)
    model, bonds, tensors, rng = make_chain("qc", 8, 0, seed=33, synthetic_m=64)
    ch = OracleChain(model, bonds, tensors, 3)
    dc = DeviceChain(ctx, ch)
    w = random_psi(ch.p12, ch.left, ch.right, rng).data
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    gx, ga = dc.adjoint(w, x)
    gx_o, ga_o = O.hpsi_adjoint(ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, w, x)
    assert _rel(gx, gx_o) <= TOL
    assert _rel(ga, ga_o) <= TOL
    assert np.max(np.abs(ga - ga_o)) <= 1e-12 * np.max(np.abs(ga_o))
    _, ga2 = dc.adjoint(w, x, want_gx=False)
    assert np.array_equal(ga, ga2)


def test_adjoint_identities_at_size(ctx):
    """Hubbard L=16, centre sites (7, 8), synthetic m=512: transpose and
    term-linearity identities on the device (no oracle at this size)."""
    model, bonds, tensors, rng = make_chain("hubbard", 16, 0, seed=5, synthetic_m=512)
    sp = E.SiteProblem(ctx, model, tensors, bonds, 7)
    plan = sp.plan
    mask = unit_mask(random_psi(sp.p12, sp.left, sp.right, rng))
    w = torch.zeros(sp.size, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(w)
    w[torch.from_numpy(mask).cuda()] = torch.randn(int(mask.sum()), dtype=torch.float64, device="cuda")
    x[torch.from_numpy(mask).cuda()] = torch.randn(int(mask.sum()), dtype=torch.float64, device="cuda")
    hx, hw = torch.zeros_like(x), torch.zeros_like(x)
    plan.hpsi(x.data_ptr(), hx.data_ptr())
    plan.hpsi(w.data_ptr(), hw.data_ptr())
    gx = torch.empty_like(x)
    ga = torch.empty(len(plan.plan["term_alpha"]), dtype=torch.float64, device="cuda")
    plan.adjoint(w.data_ptr(), x.data_ptr(), gx.data_ptr(), ga.data_ptr())
    torch.cuda.synchronize()
    ref = float(w @ hx)
    scale = float(w.norm() * hx.norm())
    alpha = torch.from_numpy(plan.plan["term_alpha"]).cuda()
    assert abs(float(gx @ x) - ref) <= 1e-12 * scale
    assert abs(float(alpha @ ga) - ref) <= 1e-12 * scale
    assert float((gx - hw).norm()) <= 1e-12 * float(hw.norm())


def test_energy_gradient_autograd_vs_finite_differences(ctx):
    model, bonds, tensors, rng = make_chain("hubbard", 8, 8, seed=41)
    ch = OracleChain(model, bonds, tensors, 3)
    dc = DeviceChain(ctx, ch)
    x0 = random_psi(ch.p12, ch.left, ch.right, rng).data
    a0 = ch.sched.plan["term_alpha"].copy()
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    alpha = torch.tensor(a0, device="cuda", requires_grad=True)
    Eval = _energy(dc, x, alpha)
    Eval.backward()
    gx, ga = x.grad.cpu().numpy(), alpha.grad.cpu().numpy()
    # analytic: dE/dx = 2 (H x - E x) / <x|x>
    hx = ch.hpsi(x0)
    e0 = x0 @ hx / (x0 @ x0)
    assert abs(float(Eval) - e0) <= 1e-12 * abs(e0)
    assert _rel(gx, 2 * (hx - e0 * x0) / (x0 @ x0)) <= 1e-11
    # central differences: along a random direction in psi, and in single alphas
    mask = unit_mask(random_psi(ch.p12, ch.left, ch.right, rng))
    d = np.zeros_like(x0)
    d[mask] = rng.standard_normal(int(mask.sum()))
    h = 1e-6
    xp = torch.tensor(x0 + h * d, device="cuda")
    xm = torch.tensor(x0 - h * d, device="cuda")
    at = torch.tensor(a0, device="cuda")
    fd = (float(_energy(dc, xp, at)) - float(_energy(dc, xm, at))) / (2 * h)
    assert abs(fd - gx @ d) <= 1e-7 * max(1.0, abs(fd))
    xt = torch.tensor(x0, device="cuda")
    for k in rng.choice(len(a0), size=6, replace=False):
        ap, am = a0.copy(), a0.copy()
        ap[k] += h
        am[k] -= h
        fd = (float(_energy(dc, xt, torch.tensor(ap, device="cuda"))) -
              float(_energy(dc, xt, torch.tensor(am, device="cuda")))) / (2 * h)
        assert abs(fd - ga[k]) <= 1e-7 * max(1.0, abs(ga[k])), k


def test_coefficient_gradient_matches_dense_rdm(ctx):
    """dE/dt (centre-bond hopping) and dE/dU (centre sites) through the device
    adjoint and the schedule's term provenance equal <P psi|dH/dc|P psi>/<psi|psi>."""
    L, i = 6, 2
    model, bonds, tensors, rng = make_chain("hubbard", L, 8, seed=43)
    ch = OracleChain(model, bonds, tensors, i, merge=False)
    dc = DeviceChain(ctx, ch)
    psi = random_psi(ch.p12, ch.left, ch.right, rng).data
    x = torch.tensor(psi, device="cuda")
    alpha = torch.tensor(ch.sched.plan["term_alpha"], device="cuda", requires_grad=True)
    _energy(dc, x, alpha).backward()
    g = ch.sched.mpo_term_grad(alpha.grad.cpu().numpy(), ch.W12.n_terms)
    sel = hubbard_center_terms(ch.W12, ch.W12mpo)
    coeff = {"t": 1.0, "U1": 4.0, "U2": 4.0}
    P = D.embedding(ch.tensors[:i], ch.tensors[i + 2:], model.phys, model.phys, ch.left, ch.right, ch.p12)
    v = P @ psi
    for name, terms in hubbard_derivative_ops(model, i).items():
        grad = sum(g[j] * ch.W12.term_scale[j] / coeff[name] for j in sel[name])
        Op = D.sparse_hamiltonian(dataclasses.replace(model, dense_terms=terms), L)
        expect = (v @ (Op @ v)) / (psi @ psi)
        assert abs(grad - expect) <= 1e-11 * max(1.0, abs(expect)), (name, grad, expect)
