"""Host-side driver of the hot path over the C ABI.

* schedule building (host, libdmrgb200's C++ builder): H·psi and left/right
  boundary-step plans, returned as flat numpy plan dictionaries;
* device execution: plans bound to device-resident boundaries (torch CUDA
  tensors used as plain device buffers) and run by the library's sm_100a
  kernels; there is no CPU execution path here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi
from .models import MPOHandle


class IndexArrays:
    """dmrgb200_index_desc over a [(charge, size)] list."""

    def __init__(self, idx):
        self.charges = np.ascontiguousarray(np.array([list(c) for c, _ in idx], dtype=np.int32).reshape(-1))
        self.sizes = np.ascontiguousarray(np.array([m for _, m in idx], dtype=np.uint32))
        self.desc = capi.IndexDesc()
        self.desc.n = len(idx)
        self.desc.charges = capi.ptr(self.charges, C.c_int32) if len(idx) else None
        self.desc.sizes = capi.ptr(self.sizes, C.c_uint32) if len(idx) else None

    @property
    def ref(self):
        return C.byref(self.desc)


class BIndex:
    """A boundary index handle plus its described storage layout."""

    def __init__(self, handle):
        self.handle = handle
        nc, aux, ne = C.c_uint32(), C.c_uint32(), C.c_uint64()
        capi.check(capi.lib.dmrgb200_bindex_info(handle, C.byref(nc), C.byref(aux), C.byref(ne)), "bindex_info")
        self.n_cohorts, self.aux, self.n_elems = nc.value, aux.value, ne.value
        n, a = self.n_cohorts, max(self.aux, 1)
        self.lb = np.zeros(n, np.uint32)
        self.rb = np.zeros(n, np.uint32)
        self.tr = np.zeros(n, np.uint8)
        self.storage_off = np.zeros(n, np.uint64)
        self.lsize = np.zeros(n, np.uint32)
        self.rsize = np.zeros(n, np.uint32)
        self.nblocks = np.zeros(n, np.uint32)
        self.offsets = np.zeros(n * a, np.int64)
        self.conj = np.zeros(n * a, np.float64)
        self.trans = np.zeros(n * a, np.uint8)
        capi.check(capi.lib.dmrgb200_bindex_describe(
            handle, capi.ptr(self.lb, C.c_uint32), capi.ptr(self.rb, C.c_uint32), capi.ptr(self.tr, C.c_uint8),
            capi.ptr(self.storage_off, C.c_uint64), capi.ptr(self.lsize, C.c_uint32),
            capi.ptr(self.rsize, C.c_uint32), capi.ptr(self.nblocks, C.c_uint32), capi.ptr(self.offsets, C.c_int64),
            capi.ptr(self.conj, C.c_double), capi.ptr(self.trans, C.c_uint8)), "bindex_describe")
        self.offsets = self.offsets.reshape(n, a)
        self.conj = self.conj.reshape(n, a)
        self.trans = self.trans.reshape(n, a)

    def signature(self) -> int:
        """Hash of the index structure (cohorts, sizes, storage layout, conjugation and
        transposition tables): equal for indices that schedules cannot tell apart."""
        if getattr(self, "_sig", None) is None:
            import hashlib
            hsh = hashlib.blake2b(digest_size=16)
            for a in (self.lb, self.rb, self.tr, self.storage_off, self.lsize, self.rsize, self.nblocks, self.offsets,
                      self.conj, self.trans):
                hsh.update(np.ascontiguousarray(a).tobytes())
            hsh.update(np.array([self.n_cohorts, self.aux, self.n_elems], dtype=np.uint64).tobytes())
            self._sig = int.from_bytes(hsh.digest(), "little")
        return self._sig

    def has_storage(self, ci):
        return self.storage_off[ci] != np.uint64(0xFFFFFFFFFFFFFFFF)

    def cohort_addresses(self, base: int) -> np.ndarray:
        """Address of each cohort's storage for a buffer at `base` (0 without storage)."""
        out = np.zeros(self.n_cohorts, dtype=np.uint64)
        for ci in range(self.n_cohorts):
            if self.has_storage(ci):
                out[ci] = np.uint64(base + 8 * int(self.storage_off[ci]))
        return out

    def edge_values(self) -> np.ndarray:
        """Storage filled with ones (an edge boundary, boundary.h:257-283)."""
        v = np.zeros(self.n_elems)
        for ci in range(self.n_cohorts):
            if self.has_storage(ci):
                o = int(self.storage_off[ci])
                v[o:o + int(self.lsize[ci]) * int(self.rsize[ci]) * int(self.nblocks[ci])] = 1.0
        return v

    def __del__(self):
        if getattr(self, "handle", None):
            capi.lib.dmrgb200_bindex_destroy(self.handle)
            self.handle = None


def edge_bindex(symm: int, index, aux: int = 1) -> BIndex:
    ia = IndexArrays(index)
    h = C.c_void_p()
    capi.check(capi.lib.dmrgb200_bindex_create_edge(symm, ia.ref, aux, C.byref(h)), "bindex_create_edge")
    return BIndex(h)


class Schedule:
    """A host-side flat plan (dmrgb200_schedule_t) and its numpy export."""

    def __init__(self, handle):
        self.handle = handle
        d = capi.PlanDesc()
        capi.check(capi.lib.dmrgb200_schedule_export(handle, C.byref(d)), "schedule_export")
        self.plan = capi.desc_to_numpy(d)
        f = C.c_uint64()
        capi.check(capi.lib.dmrgb200_schedule_flops(handle, C.byref(f)), "schedule_flops")
        self.flops = f.value

    def term_sources(self):
        """(src, dscale) per plan term: the MPO term it comes from and d alpha / d scale
        (dmrgb200_schedule_term_sources; H·psi schedules only)."""
        n = len(self.plan["term_alpha"])
        src = np.zeros(max(n, 1), dtype=np.uint32)
        dsc = np.zeros(max(n, 1), dtype=np.float64)
        capi.check(capi.lib.dmrgb200_schedule_term_sources(
            self.handle, src.ctypes.data_as(C.POINTER(C.c_uint32)), dsc.ctypes.data_as(C.POINTER(C.c_double))),
            "schedule_term_sources")
        return src[:n], dsc[:n]

    def mpo_term_grad(self, galpha: np.ndarray, n_mpo_terms: int) -> np.ndarray:
        """d<w|H x>/d (MPO term scale) from the per-term derivatives galpha."""
        src, dsc = self.term_sources()
        g = np.zeros(n_mpo_terms)
        np.add.at(g, src, dsc * np.asarray(galpha, dtype=np.float64))
        return g

    def __del__(self):
        if getattr(self, "handle", None):
            capi.lib.dmrgb200_schedule_destroy(self.handle)
            self.handle = None


def schedule_hpsi(phys, left, right, mpo: MPOHandle, L: BIndex, R: BIndex) -> Schedule:
    p, l, r = IndexArrays(phys), IndexArrays(left), IndexArrays(right)
    h = C.c_void_p()
    capi.check(capi.lib.dmrgb200_schedule_hpsi(p.ref, l.ref, r.ref, mpo.handle, L.handle, R.handle, C.byref(h)),
               "schedule_hpsi")
    return Schedule(h)


def schedule_left_step(phys, left, right, mpo: MPOHandle, L: BIndex, symmetric=True):
    p, l, r = IndexArrays(phys), IndexArrays(left), IndexArrays(right)
    h, nb = C.c_void_p(), C.c_void_p()
    capi.check(capi.lib.dmrgb200_schedule_left_step(p.ref, l.ref, r.ref, mpo.handle, L.handle, int(symmetric),
                                                    C.byref(h), C.byref(nb)), "schedule_left_step")
    return Schedule(h), BIndex(nb)


def schedule_right_step(phys, left, right, mpo: MPOHandle, R: BIndex, symmetric=True):
    p, l, r = IndexArrays(phys), IndexArrays(left), IndexArrays(right)
    h, nb = C.c_void_p(), C.c_void_p()
    capi.check(capi.lib.dmrgb200_schedule_right_step(p.ref, l.ref, r.ref, mpo.handle, R.handle, int(symmetric),
                                                     C.byref(h), C.byref(nb)), "schedule_right_step")
    return Schedule(h), BIndex(nb)


# ---- device side --------------------------------------------------------------------

def _view(addresses: np.ndarray):
    arr = (C.c_void_p * max(len(addresses), 1))(*[int(a) if a else None for a in addresses])
    v = capi.BoundaryView()
    v.n_cohorts = len(addresses)
    v.cohort_ptr = C.cast(arr, C.POINTER(C.c_void_p))
    return v, arr


class Context:
    def __init__(self, device: int = 0):
        h = C.c_void_p()
        capi.check(capi.lib.dmrgb200_context_create(device, C.byref(h)), "context_create")
        self.handle = h
        self.device = device

    def __del__(self):
        if getattr(self, "handle", None):
            capi.lib.dmrgb200_context_destroy(self.handle)
            self.handle = None


class DevicePlan:
    """A plan bound to device boundaries (dmrgb200_plan_create)."""

    def __init__(self, ctx: Context, plan: dict, left_addr=None, other_addr=None):
        desc, self._keep = capi.numpy_to_desc(plan)
        lv = ov = None
        if left_addr is not None:
            lv, la = _view(left_addr)
            self._keep.append(la)
        if other_addr is not None:
            ov, oa = _view(other_addr)
            self._keep.append(oa)
        h = C.c_void_p()
        capi.check(capi.lib.dmrgb200_plan_create(ctx.handle, C.byref(desc), C.byref(lv) if lv else None,
                                                 C.byref(ov) if ov else None, C.byref(h)), "plan_create")
        self.handle = h
        self.plan = plan
        f, s = C.c_uint64(), C.c_uint64()
        capi.check(capi.lib.dmrgb200_plan_flops(h, C.byref(f)), "plan_flops")
        capi.check(capi.lib.dmrgb200_plan_scratch_bytes(h, C.byref(s)), "plan_scratch_bytes")
        self.flops, self.scratch_bytes = f.value, s.value

    def hpsi(self, x_ptr: int, y_ptr: int, prec: int = capi.PREC_FP64, stream: int = 0) -> None:
        capi.check(capi.lib.dmrgb200_hpsi(self.handle, x_ptr, y_ptr, prec, stream or None), "dmrgb200_hpsi")

    def hpsi_host(self, x_host_ptr: int, y_host_ptr: int, stream: int = 0) -> None:
        """H·psi from and into host buffers (dmrgb200_hpsi_host: copies overlapped with the
        products; pinned buffers for the overlap; synchronise the stream before reading)."""
        capi.check(capi.lib.dmrgb200_hpsi_host(self.handle, x_host_ptr, y_host_ptr, stream or None),
                   "dmrgb200_hpsi_host")

    def adjoint(self, w_ptr: int, x_ptr: int, gx_ptr: int, galpha_ptr: int, stream: int = 0) -> None:
        """gx = H^T w and galpha[k] = <w|H_k x> (dmrgb200_hpsi_adjoint; 0 skips an output)."""
        capi.check(capi.lib.dmrgb200_hpsi_adjoint(self.handle, w_ptr, x_ptr or None, gx_ptr or None,
                                                  galpha_ptr or None, stream or None), "dmrgb200_hpsi_adjoint")

    def set_precision(self, prec: int) -> None:
        """Precision of the H·psi inside solve (dmrgb200_plan_set_precision)."""
        capi.check(capi.lib.dmrgb200_plan_set_precision(self.handle, prec), "dmrgb200_plan_set_precision")

    def set_slices(self, slices: int) -> None:
        capi.check(capi.lib.dmrgb200_plan_set_slices(self.handle, slices), "dmrgb200_plan_set_slices")

    def set_gemm_variants(self, stage1: int, stage3: int) -> None:
        """Pin the grouped-GEMM variants of stages 1 and 3 (dmrgb200_plan_set_gemm_variants)."""
        capi.check(capi.lib.dmrgb200_plan_set_gemm_variants(self.handle, stage1, stage3),
                   "dmrgb200_plan_set_gemm_variants")

    def tune_slices(self, x_ptr: int, target: float = 1e-10, stream: int = 0):
        """Smallest digit-plane count whose emulated H·psi of x is within `target` (relative)
        of the FP64 one (dmrgb200_plan_tune_slices); returns (slices, relative error)."""
        sl, err = C.c_int32(), C.c_double()
        capi.check(capi.lib.dmrgb200_plan_tune_slices(self.handle, x_ptr, target, stream or None, C.byref(sl),
                                                      C.byref(err)), "dmrgb200_plan_tune_slices")
        return sl.value, err.value

    def boundaries_changed(self) -> None:
        """The bound boundary buffers were rewritten in place (dmrgb200_plan_boundaries_changed)."""
        capi.check(capi.lib.dmrgb200_plan_boundaries_changed(self.handle), "dmrgb200_plan_boundaries_changed")

    def check(self, stream: int = 0) -> None:
        """Synchronise and raise if a kernel's bounded wait ran out (dmrgb200_plan_check)."""
        capi.check(capi.lib.dmrgb200_plan_check(self.handle, stream or None), "dmrgb200_plan_check")

    def set_solver(self, mode: int) -> None:
        """capi.SOLVER_GRAPH (default: one CUDA graph per solve) or capi.SOLVER_STEPWISE."""
        capi.check(capi.lib.dmrgb200_plan_set_solver(self.handle, mode), "dmrgb200_plan_set_solver")

    def solve(self, x0_ptr: int, x_out_ptr: int, n: int, ortho_ptrs=(), tol: float = 1e-8, max_iter: int = 8,
              stream: int = 0):
        """Jacobi-Davidson lowest eigenpair (dmrgb200_solve); returns (energy, stats)."""
        e = C.c_double()
        st = capi.SolveStats()
        arr = (C.c_void_p * max(len(ortho_ptrs), 1))(*[int(p) for p in ortho_ptrs])
        capi.check(capi.lib.dmrgb200_solve(self.handle, n, x0_ptr, C.cast(arr, C.POINTER(C.c_void_p)),
                                           len(ortho_ptrs), tol, max_iter, C.byref(e), x_out_ptr, C.byref(st),
                                           stream or None), "dmrgb200_solve")
        return e.value, st

    def step(self, ket_ptr: int, bra_ptr: int, out_addr: np.ndarray, stream: int = 0) -> None:
        v, arr = _view(out_addr)
        capi.check(capi.lib.dmrgb200_step_execute(self.handle, ket_ptr, bra_ptr, C.byref(v), stream or None),
                   "dmrgb200_step_execute")
        del arr

    def alpha_dm(self, ket_ptr: int, bra_ptr: int, dm_addr: np.ndarray, alpha: float, stream: int = 0) -> None:
        """Density matrix of the split with the perturbation into the blocks at dm_addr
        (dmrgb200_step_alpha_dm; a step plan of the two-site tensor as one site)."""
        v, arr = _view(dm_addr)
        capi.check(capi.lib.dmrgb200_step_alpha_dm(self.handle, ket_ptr, bra_ptr, C.byref(v), float(alpha),
                                                   stream or None), "dmrgb200_step_alpha_dm")
        del arr

    def __del__(self):
        if getattr(self, "handle", None):
            capi.lib.dmrgb200_plan_destroy(self.handle)
            self.handle = None


# ---- device chains ---------------------------------------------------------------

def _torch():
    import torch
    return torch


def to_device(a: np.ndarray, device: int = 0):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(f"cuda:{device}")


def device_left_step(ctx: Context, phys, left, right, mpo: MPOHandle, Lidx: BIndex, Lbuf, ket_rp, bra_lp,
                     symmetric=True, stream: int = 0):
    """overlap_mpo_left_step on the device: returns (new index, new device buffer)."""
    torch = _torch()
    sched, nidx = schedule_left_step(phys, left, right, mpo, Lidx, symmetric)
    plan = DevicePlan(ctx, sched.plan, left_addr=Lidx.cohort_addresses(Lbuf.data_ptr()))
    out = torch.zeros(max(nidx.n_elems, 1), dtype=torch.float64, device=Lbuf.device)
    plan.step(ket_rp.data_ptr(), bra_lp.data_ptr(), nidx.cohort_addresses(out.data_ptr()), stream)
    return nidx, out


def device_right_step(ctx: Context, phys, left, right, mpo: MPOHandle, Ridx: BIndex, Rbuf, ket_rp, bra_rp,
                      symmetric=True, stream: int = 0):
    """overlap_mpo_right_step on the device: returns (new index, new device buffer)."""
    torch = _torch()
    sched, nidx = schedule_right_step(phys, left, right, mpo, Ridx, symmetric)
    plan = DevicePlan(ctx, sched.plan, other_addr=Ridx.cohort_addresses(Rbuf.data_ptr()))
    out = torch.zeros(max(nidx.n_elems, 1), dtype=torch.float64, device=Rbuf.device)
    plan.step(ket_rp.data_ptr(), bra_rp.data_ptr(), nidx.cohort_addresses(out.data_ptr()), stream)
    return nidx, out


class SiteProblem:
    """H·psi at sites (i, i+1) of a chain with device-resident boundaries.

    Boundaries are built by device boundary steps from the chain ends with the
    given site tensors (ket = bra), as the optimizer's boundary caches are
    (optimize.h:134-195)."""

    def __init__(self, ctx: Context, model, tensors, bonds, i: int, symmetric=True, stream: int = 0):
        from . import models as M
        torch = _torch()
        self.ctx, self.model, self.i = ctx, model, i
        dev = ctx.device
        L = len(tensors)
        Lidx = edge_bindex(model.symm, bonds[0])
        Lbuf = to_device(Lidx.edge_values(), dev)
        for p in range(i):
            W = M.MPOHandle(model.mpo[p], model.symm)
            t = tensors[p]
            Lidx, Lbuf = device_left_step(ctx, model.phys, bonds[p], bonds[p + 1], W, Lidx, Lbuf,
                                          to_device(t.data, dev), to_device(t.left_paired(), dev), symmetric, stream)
        Ridx = edge_bindex(model.symm, bonds[L])
        Rbuf = to_device(Ridx.edge_values(), dev)
        for p in range(L - 1, i + 1, -1):
            W = M.MPOHandle(model.mpo[p], model.symm)
            t = tensors[p]
            td = to_device(t.data, dev)
            Ridx, Rbuf = device_right_step(ctx, model.phys, bonds[p], bonds[p + 1], W, Ridx, Rbuf, td, td,
                                           symmetric, stream)
        self.Lidx, self.Lbuf, self.Ridx, self.Rbuf = Lidx, Lbuf, Ridx, Rbuf
        self.p12, _ = M.fuse_phys(model.phys, model.phys)
        self.W12 = M.MPOHandle(M.twosite_for(model, i), model.symm)
        self.left, self.right = bonds[i], bonds[i + 2]
        self.schedule = schedule_hpsi(self.p12, self.left, self.right, self.W12, Lidx, Ridx)
        self.plan = DevicePlan(ctx, self.schedule.plan, left_addr=Lidx.cohort_addresses(Lbuf.data_ptr()),
                               other_addr=Ridx.cohort_addresses(Rbuf.data_ptr()))
        self.size = int(self.schedule.plan["in_size"])
        torch.cuda.synchronize(dev)

    def hpsi(self, x, y, prec: int = capi.PREC_FP64, stream: int = 0):
        self.plan.hpsi(x.data_ptr(), y.data_ptr(), prec, stream)


class BatchedPlan(DevicePlan):
    """Independent H·psi problems merged into one plan (dmrgb200_plan_create_batched).

    `items` is a list of (plan dict, left cohort addresses, right cohort
    addresses); instance i occupies x[in_base[i] : in_base[i] + in_size_i]."""

    def __init__(self, ctx: Context, items):
        n = len(items)
        descs = (capi.PlanDesc * n)()
        lviews = (capi.BoundaryView * n)()
        rviews = (capi.BoundaryView * n)()
        self._keep = []
        for i, (plan, la, ra) in enumerate(items):
            d, k = capi.numpy_to_desc(plan)
            descs[i] = d
            self._keep.append(k)
            lv, larr = _view(la)
            rv, rarr = _view(ra)
            lviews[i], rviews[i] = lv, rv
            self._keep += [larr, rarr]
        base = (C.c_uint64 * n)()
        total = C.c_uint64()
        h = C.c_void_p()
        capi.check(capi.lib.dmrgb200_plan_create_batched(ctx.handle, n, descs, lviews, rviews, base, C.byref(total),
                                                         C.byref(h)), "plan_create_batched")
        self.handle = h
        self.in_base = [int(b) for b in base]
        self.total_size = total.value
        self.sizes = [int(p["in_size"]) for p, _, _ in items]
        f, s = C.c_uint64(), C.c_uint64()
        capi.check(capi.lib.dmrgb200_plan_flops(h, C.byref(f)), "plan_flops")
        capi.check(capi.lib.dmrgb200_plan_scratch_bytes(h, C.byref(s)), "plan_scratch_bytes")
        self.flops, self.scratch_bytes = f.value, s.value
        self.plan = None


def block_svd(blocks, stream=None):
    """Thin SVD of device blocks on the device (dmrgb200_block_svd).

    `blocks` is a list of (rows, cols, a, u, s, vt): a the column-major rows x
    cols input, u (rows x k), s (k) and vt (k x cols) the outputs, k =
    min(rows, cols), all CUDA float64 tensors (plain device buffers; only their
    data pointers are used).  Returns after completion."""
    n = len(blocks)
    rows = np.ascontiguousarray([b[0] for b in blocks], dtype=np.uint32)
    cols = np.ascontiguousarray([b[1] for b in blocks], dtype=np.uint32)
    arr = [(C.c_void_p * max(n, 1))(*[b[j].data_ptr() if b[j] is not None else None for b in blocks])
           for j in range(2, 6)]
    st = capi.lib.dmrgb200_block_svd(n, capi.ptr(rows, C.c_uint32), capi.ptr(cols, C.c_uint32), *arr,
                                     None if stream is None else C.c_void_p(stream))
    capi.check(st, "dmrgb200_block_svd")


def copy_blocks(copies: np.ndarray, src, dst, scale=None, stream=None):
    """Column-major block copies between device buffers (dmrgb200_copy_blocks).
    `copies` is a structured array of capi.BlockCopy records (see copy_records)."""
    n = len(copies)
    if n == 0:
        return
    arr = (capi.BlockCopy * n).from_buffer_copy(np.ascontiguousarray(copies).tobytes())
    st = capi.lib.dmrgb200_copy_blocks(n, arr, src.data_ptr(), dst.data_ptr(),
                                       None if scale is None else scale.data_ptr(),
                                       None if stream is None else C.c_void_p(stream))
    capi.check(st, "dmrgb200_copy_blocks")


COPY_DTYPE = np.dtype([("src_off", np.uint64), ("dst_off", np.uint64), ("scale_off", np.uint64),
                       ("src_ld", np.uint32), ("dst_ld", np.uint32), ("rows", np.uint32), ("cols", np.uint32),
                       ("scale_mode", np.uint32), ("reserved", np.uint32)])


def copy_records(rows):
    """Structured array of block copies from (src_off, src_ld, dst_off, dst_ld,
    nrows, ncols, scale_mode, scale_off) tuples."""
    out = np.zeros(len(rows), dtype=COPY_DTYPE)
    for k, (so, sl, do, dl, r, c, mode, sco) in enumerate(rows):
        out[k] = (so, do, sco, sl, dl, r, c, mode, 0)
    return out


def apply_copies(copies: np.ndarray, src: np.ndarray, dst: np.ndarray, scale: np.ndarray | None = None):
    """The same copies on host arrays (the definition the device copies follow;
    used to check the host-side split logic without a GPU)."""
    for c in copies:
        r, n = int(c["rows"]), int(c["cols"])
        if r == 0 or n == 0:
            continue
        so, sl, do, dl = int(c["src_off"]), int(c["src_ld"]), int(c["dst_off"]), int(c["dst_ld"])
        blk = np.stack([src[so + j * sl: so + j * sl + r] for j in range(n)], axis=1)
        if c["scale_mode"] == capi.SCALE_ROWS:
            blk = blk * scale[int(c["scale_off"]): int(c["scale_off"]) + r, None]
        elif c["scale_mode"] == capi.SCALE_COLS:
            blk = blk * scale[None, int(c["scale_off"]): int(c["scale_off"]) + n]
        for j in range(n):
            dst[do + j * dl: do + j * dl + r] = blk[:, j]
