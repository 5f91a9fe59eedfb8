"""The site-problem dump (dmrgb200.dump): a plan, both boundaries and a psi written
to one archive and read back give identical arrays and the same H·psi."""
import numpy as np

import oracle as O
from dmrgb200 import dump
from helpers import OracleChain, make_chain, random_psi


def test_site_problem_round_trip(tmp_path):
    model, bonds, tensors, rng = make_chain("hubbard", 10, 0, seed=4, synthetic_m=40)
    ch = OracleChain(model, bonds, tensors, 4)
    x = random_psi(ch.p12, ch.left, ch.right, rng).data
    path = tmp_path / "site.npz"
    dump.save_site_problem(path, ch.sched.plan, ch.Lval, ch.Lidx, ch.Rval, ch.Ridx, psi=x,
                           meta={"workload": "hubbard_L10_m40_site4"})
    d = dump.load_site_problem(path)
    for k, v in ch.sched.plan.items():
        assert np.array_equal(np.asarray(d.plan[k]), np.asarray(v)), k
    assert np.array_equal(d.L, ch.Lval) and np.array_equal(d.R, ch.Rval) and np.array_equal(d.psi, x)
    for f in ("storage_off", "lsize", "rsize", "nblocks", "tr"):
        assert np.array_equal(getattr(d.Lidx, f), getattr(ch.Lidx, f))
        assert np.array_equal(getattr(d.Ridx, f), getattr(ch.Ridx, f))
    assert d.meta["workload"] == "hubbard_L10_m40_site4"
    y0 = ch.hpsi(x)
    y1 = O.hpsi(d.plan, d.L, d.Lidx, d.R, d.Ridx, d.psi)
    assert np.linalg.norm(y1 - y0) <= 1e-14 * np.linalg.norm(y0)
