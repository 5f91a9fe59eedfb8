"""Binary dump of a site problem: the flat H·psi plan, both boundaries (values and
cohort layout) and optionally a two-site tensor, so that a site problem can be
reproduced exactly in another process (benchmarks, regression checks) without
rebuilding the MPO, the boundaries or the schedule.  The reference serialises
Boundary objects and whole MPS checkpoints through Boost binary archives
(Boundary::save_boundary, mp_tensors/boundary.h:422-429; ts_optimize snapshots,
optimize/ts_optimize.hpp:185-215).

Format: one NumPy .npz archive (zip of .npy arrays; little endian, fixed dtypes):
  format = "dmrgb200-site-problem", version = 1
  plan/<key>        every array of the flat plan (the dmrgb200_plan_desc fields),
                    plan/kind, plan/in_size, plan/out_size as 0-d uint64
  L/values, R/values  boundary storage (FP64), each cohort at its storage offset
  L/<field>, R/<field>  cohort layout: storage_off (uint64, 2^64-1 without storage),
                    lsize, rsize, nblocks (uint32), tr (uint8)
  psi               (optional) a vector in the plan's in layout
  meta/<key>        (optional) strings or numbers describing the workload
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FORMAT = "dmrgb200-site-problem"
VERSION = 1
_INDEX_FIELDS = ("storage_off", "lsize", "rsize", "nblocks", "tr")
_NO_STORAGE = np.uint64(0xFFFFFFFFFFFFFFFF)


class StoredIndex:
    """The cohort layout of a boundary read back from a dump: enough to address its
    cohorts (cohort_addresses) and to describe them to the oracle and the reference."""

    def __init__(self, storage_off, lsize, rsize, nblocks, tr):
        self.storage_off = np.asarray(storage_off, dtype=np.uint64)
        self.lsize = np.asarray(lsize, dtype=np.uint32)
        self.rsize = np.asarray(rsize, dtype=np.uint32)
        self.nblocks = np.asarray(nblocks, dtype=np.uint32)
        self.tr = np.asarray(tr, dtype=np.uint8)
        self.n_cohorts = len(self.storage_off)

    def has_storage(self, ci):
        return self.storage_off[ci] != _NO_STORAGE

    def cohort_addresses(self, base: int) -> np.ndarray:
        out = np.zeros(self.n_cohorts, dtype=np.uint64)
        for ci in range(self.n_cohorts):
            if self.has_storage(ci):
                out[ci] = np.uint64(base + 8 * int(self.storage_off[ci]))
        return out


@dataclass
class SiteProblemData:
    plan: dict
    L: np.ndarray
    Lidx: StoredIndex
    R: np.ndarray
    Ridx: StoredIndex
    psi: np.ndarray | None
    meta: dict


def save_site_problem(path, plan: dict, L: np.ndarray, Lidx, R: np.ndarray, Ridx, psi=None, meta=None) -> None:
    """Write a site problem; Lidx / Ridx are engine.BIndex (or StoredIndex) objects."""
    arrays = {"format": np.array(FORMAT), "version": np.array(VERSION, dtype=np.uint32)}
    for k, v in plan.items():
        arrays["plan/" + k] = np.asarray(v) if not np.isscalar(v) else np.array(v, dtype=np.uint64)
    for side, vals, idx in (("L", L, Lidx), ("R", R, Ridx)):
        arrays[side + "/values"] = np.ascontiguousarray(vals, dtype=np.float64)
        for f in _INDEX_FIELDS:
            arrays[f"{side}/{f}"] = np.asarray(getattr(idx, f))
    if psi is not None:
        arrays["psi"] = np.ascontiguousarray(psi, dtype=np.float64)
    for k, v in (meta or {}).items():
        arrays["meta/" + k] = np.array(v)
    with open(path, "wb") as f:
        np.savez(f, **arrays)


def load_site_problem(path) -> SiteProblemData:
    with np.load(path, allow_pickle=False) as z:
        if str(z["format"]) != FORMAT:
            raise ValueError(f"{path}: not a {FORMAT} file")
        if int(z["version"]) != VERSION:
            raise ValueError(f"{path}: version {int(z['version'])}, this reader knows {VERSION}")
        plan, meta = {}, {}
        idx = {"L": {}, "R": {}}
        vals = {}
        psi = None
        for k in z.files:
            if k.startswith("plan/"):
                a = z[k]
                plan[k[5:]] = int(a) if a.ndim == 0 else a.copy()
            elif k.startswith("meta/"):
                a = z[k]
                meta[k[5:]] = a.item() if a.ndim == 0 else a.copy()
            elif k[:2] in ("L/", "R/"):
                side, f = k.split("/", 1)
                if f == "values":
                    vals[side] = z[k].copy()
                else:
                    idx[side][f] = z[k].copy()
            elif k == "psi":
                psi = z[k].copy()
    return SiteProblemData(plan, vals["L"], StoredIndex(**idx["L"]), vals["R"], StoredIndex(**idx["R"]), psi, meta)
