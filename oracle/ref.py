"""ORACLE — test infrastructure only.  Python front-end of oracle/_ref/libmaquis_ref.so:
the reference's own solver core (tasks.cpp) driven with flat plans
(ref_adapter.cpp).  Available where oracle/build_ref.sh could compile the
reference sources (the reference tree and this image's compilers)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from dmrgb200 import _capi as capi

LIB = Path(__file__).resolve().parent / "_ref" / "libmaquis_ref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(LIB))
        PD = C.POINTER(capi.PlanDesc)
        u32 = C.POINTER(C.c_uint32)
        pp = C.POINTER(C.c_void_p)
        _lib.ref_hpsi.argtypes = [PD, C.c_uint32, u32, u32, u32, pp, C.c_uint32, pp, C.c_void_p, C.c_void_p]
        _lib.ref_left_step.argtypes = [PD, C.c_uint32, u32, u32, u32, pp, C.c_void_p, C.c_void_p, pp]
        _lib.ref_right_step.argtypes = [PD, C.c_uint32, u32, u32, u32, pp, C.c_void_p, C.c_void_p, pp]
        _lib.ref_hpsi_create.argtypes = [PD, C.c_uint32, u32, u32, u32, pp, C.c_uint32, pp]
        _lib.ref_hpsi_create.restype = C.c_void_p
        _lib.ref_hpsi_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.ref_hpsi_destroy.argtypes = [C.c_void_p]
        _lib.ref_alpha_dm.argtypes = [PD, C.c_uint32, u32, u32, u32, pp, C.c_void_p, C.c_double, pp]
        _lib.ref_hpsi_flatten.argtypes = [C.c_void_p]
        _lib.ref_hpsi_flatten.restype = C.POINTER(capi.PlanDesc)
    return _lib


def _ptrs(storage, bidx):
    addr = bidx.cohort_addresses(storage.ctypes.data)
    return (C.c_void_p * max(len(addr), 1))(*[int(a) if a else None for a in addr])


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def hpsi(plan, L, Lidx, R, Ridx, x):
    desc, keep = capi.numpy_to_desc(plan)
    y = np.zeros(plan["out_size"])
    ls, rs, nb = _u32(Ridx.lsize), _u32(Ridx.rsize), _u32(Ridx.nblocks)
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    rc = lib().ref_hpsi(C.byref(desc), Ridx.n_cohorts, u(ls), u(rs), u(nb), _ptrs(L, Lidx), Lidx.n_cohorts,
                        _ptrs(R, Ridx), np.ascontiguousarray(x).ctypes.data, y.ctypes.data)
    assert rc == 0
    return y


class Hpsi:
    """The reference's ScheduleNew for one H psi plan, built once (as the reference
    builds one schedule per site problem) and run on many x: `run(x)` executes
    only create_T and contract on the host cores."""

    def __init__(self, plan, L, Lidx, R, Ridx):
        self._desc, self._keep = capi.numpy_to_desc(plan)
        self._L, self._R = L, R
        self._ls, self._rs, self._nb = _u32(Ridx.lsize), _u32(Ridx.rsize), _u32(Ridx.nblocks)
        self._lp, self._rp = _ptrs(L, Lidx), _ptrs(R, Ridx)
        u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
        self.out_size = int(plan["out_size"])
        self._h = lib().ref_hpsi_create(C.byref(self._desc), Ridx.n_cohorts, u(self._ls), u(self._rs), u(self._nb),
                                        self._lp, Lidx.n_cohorts, self._rp)
        assert self._h

    def run(self, x, y=None):
        y = np.zeros(self.out_size) if y is None else y
        assert lib().ref_hpsi_run(self._h, np.ascontiguousarray(x).ctypes.data, y.ctypes.data) == 0
        return y

    def flatten(self) -> dict:
        """The reference's ScheduleNew flattened back into a plan description (ref_flatten.cpp),
        copied into numpy arrays."""
        d = lib().ref_hpsi_flatten(self._h)
        assert d
        return capi.desc_to_numpy(d.contents)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_hpsi_destroy(self._h)
            self._h = None


def left_step(plan, L, Lidx, ket_rp, bra_lp, new_idx):
    desc, keep = capi.numpy_to_desc(plan)
    out = np.zeros(new_idx.n_elems)
    ls, rs, nb = _u32(Lidx.lsize), _u32(Lidx.rsize), _u32(Lidx.nblocks)
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    rc = lib().ref_left_step(C.byref(desc), Lidx.n_cohorts, u(ls), u(rs), u(nb), _ptrs(L, Lidx),
                             np.ascontiguousarray(ket_rp).ctypes.data, np.ascontiguousarray(bra_lp).ctypes.data,
                             _ptrs(out, new_idx))
    assert rc == 0
    return out


def right_step(plan, R, Ridx, ket_rp, bra_rp, new_idx):
    desc, keep = capi.numpy_to_desc(plan)
    out = np.zeros(new_idx.n_elems)
    ls, rs, nb = _u32(Ridx.lsize), _u32(Ridx.rsize), _u32(Ridx.nblocks)
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    rc = lib().ref_right_step(C.byref(desc), Ridx.n_cohorts, u(ls), u(rs), u(nb), _ptrs(R, Ridx),
                              np.ascontiguousarray(ket_rp).ctypes.data, np.ascontiguousarray(bra_rp).ctypes.data,
                              _ptrs(out, new_idx))
    assert rc == 0
    return out


def alpha_dm(plan, B, Bidx, ket, alpha):
    """The reference's perturbation terms alpha sum S S^T (left step) or alpha sum S^T S
    (right step) per bra block, from its own Cohort::lbtm / rbtm; a list of square
    column-major blocks (see oracle.alpha_dm)."""
    import oracle as O
    desc, keep = capi.numpy_to_desc(plan)
    blocks, flat, ptrs = O.dm_storage(plan)
    ls, rs, nb = _u32(Bidx.lsize), _u32(Bidx.rsize), _u32(Bidx.nblocks)
    u = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
    rc = lib().ref_alpha_dm(C.byref(desc), Bidx.n_cohorts, u(ls), u(rs), u(nb), _ptrs(B, Bidx),
                            np.ascontiguousarray(ket).ctypes.data, float(alpha), ptrs)
    assert rc == 0
    del keep
    return blocks
