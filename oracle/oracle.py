"""ORACLE — test infrastructure only (tests, __graft_entry__.smoke(), bench.py's
CPU baseline).  The product never imports this module.

Python front-end of liboracle.so (plan_exec.cpp): the CPU restatement of the
reference's schedule execution (create_T / create_s_r / contract and the
boundary-step kernels create_T_left / create_s / prop_l / prop_r, OpenMP over
task groups + BLAS).  Plans are the flat plan dictionaries exported by the
library's schedule builder; boundaries are numpy vectors in the library's
cohort storage layout.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "maquis-dmrg_b200"))

from dmrgb200 import _capi as capi  # noqa: E402
from dmrgb200 import engine  # noqa: E402

LIB = HERE / "liboracle.so"


def build_oracle() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < (HERE / "plan_exec.cpp").stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build_oracle()))
        PD = C.POINTER(capi.PlanDesc)
        pp = C.POINTER(C.c_void_p)
        _lib.oracle_hpsi.argtypes = [PD, pp, pp, C.c_void_p, C.c_void_p]
        _lib.oracle_left_step.argtypes = [PD, pp, C.c_void_p, C.c_void_p, pp]
        _lib.oracle_right_step.argtypes = [PD, pp, C.c_void_p, C.c_void_p, pp]
        _lib.oracle_hpsi_adjoint.argtypes = [PD, pp, pp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_alpha_dm.argtypes = [PD, pp, C.c_void_p, C.c_void_p, C.c_double, C.c_int, pp]
        _lib.oracle_set_threads.argtypes = [C.c_int]
        _lib.oracle_set_threads(int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1)))
    return _lib


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def _ptrs(storage: np.ndarray, bidx: engine.BIndex):
    base = storage.ctypes.data
    addr = bidx.cohort_addresses(base)
    arr = (C.c_void_p * max(len(addr), 1))(*[int(a) if a else None for a in addr])
    return arr


def hpsi(plan: dict, L: np.ndarray, Lidx: engine.BIndex, R: np.ndarray, Ridx: engine.BIndex,
         x: np.ndarray) -> np.ndarray:
    desc, keep = capi.numpy_to_desc(plan)
    y = np.zeros(plan["out_size"])
    la, ra = _ptrs(L, Lidx), _ptrs(R, Ridx)
    x = np.ascontiguousarray(x, dtype=np.float64)
    rc = lib().oracle_hpsi(C.byref(desc), la, ra, x.ctypes.data, y.ctypes.data)
    assert rc == 0
    del keep
    return y


def hpsi_adjoint(plan: dict, L: np.ndarray, Lidx: engine.BIndex, R: np.ndarray, Ridx: engine.BIndex,
                 w: np.ndarray, x: np.ndarray):
    """(gx, galpha): gx = H^T w, galpha[k] = <w | H_k x> (plan_exec.cpp oracle_hpsi_adjoint)."""
    desc, keep = capi.numpy_to_desc(plan)
    gx = np.zeros(plan["in_size"])
    galpha = np.zeros(len(plan["term_alpha"]))
    la, ra = _ptrs(L, Lidx), _ptrs(R, Ridx)
    w = np.ascontiguousarray(w, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    rc = lib().oracle_hpsi_adjoint(C.byref(desc), la, ra, w.ctypes.data, x.ctypes.data, gx.ctypes.data,
                                   galpha.ctypes.data)
    assert rc == 0
    del keep
    return gx, galpha


def left_step(plan: dict, L: np.ndarray, Lidx: engine.BIndex, ket_rp: np.ndarray, bra_lp: np.ndarray,
              new_idx: engine.BIndex) -> np.ndarray:
    desc, keep = capi.numpy_to_desc(plan)
    out = np.zeros(new_idx.n_elems)
    la, oa = _ptrs(L, Lidx), _ptrs(out, new_idx)
    rc = lib().oracle_left_step(C.byref(desc), la, np.ascontiguousarray(ket_rp).ctypes.data,
                                np.ascontiguousarray(bra_lp).ctypes.data, oa)
    assert rc == 0
    del keep
    return out


def right_step(plan: dict, R: np.ndarray, Ridx: engine.BIndex, ket_rp: np.ndarray, bra_rp: np.ndarray,
               new_idx: engine.BIndex) -> np.ndarray:
    desc, keep = capi.numpy_to_desc(plan)
    out = np.zeros(new_idx.n_elems)
    ra, oa = _ptrs(R, Ridx), _ptrs(out, new_idx)
    rc = lib().oracle_right_step(C.byref(desc), ra, np.ascontiguousarray(ket_rp).ctypes.data,
                                 np.ascontiguousarray(bra_rp).ctypes.data, oa)
    assert rc == 0
    del keep
    return out


def dm_storage(plan: dict):
    """Zeroed square column-major blocks of a step plan's density matrix, one per bra
    block (left step: out_rows; right step: out_cols), as views of one flat array,
    with the block pointer array for the C calls."""
    left = int(plan["kind"]) == capi.PLAN_LEFT
    dims = [int(r) if left else int(c) for r, c in zip(plan["out_rows"], plan["out_cols"])]
    offs = np.concatenate([[0], np.cumsum([d * d for d in dims])]).astype(np.int64)
    flat = np.zeros(max(int(offs[-1]), 1))
    blocks = [flat[offs[b]:offs[b + 1]].reshape(d, d, order="F") for b, d in enumerate(dims)]
    ptrs = (C.c_void_p * max(len(dims), 1))(*[flat.ctypes.data + 8 * int(offs[b]) for b in range(len(dims))])
    return blocks, flat, ptrs


def alpha_dm(plan: dict, B: np.ndarray, Bidx: engine.BIndex, ket: np.ndarray, bra: np.ndarray, alpha: float,
             with_theta: bool = True):
    """Density matrix of the split with the perturbation, per bra block (plan_exec.cpp
    oracle_alpha_dm): a list of square column-major blocks."""
    desc, keep = capi.numpy_to_desc(plan)
    blocks, flat, ptrs = dm_storage(plan)
    rc = lib().oracle_alpha_dm(C.byref(desc), _ptrs(B, Bidx), np.ascontiguousarray(ket).ctypes.data,
                               np.ascontiguousarray(bra).ctypes.data, float(alpha), int(with_theta), ptrs)
    assert rc == 0
    del keep
    return blocks
