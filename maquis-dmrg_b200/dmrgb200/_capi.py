"""ctypes binding of libdmrgb200 (include/dmrgb200.h).

The shared library is loaded from this package directory; importing this module
fails loudly when it is missing, so no code path can silently fall back to a
CPU implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libdmrgb200.so"

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python maquis-dmrg_b200/build.py` "
        "(the H·psi path has no CPU fallback)")

lib = C.CDLL(str(LIB_PATH))

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)
f64p = C.POINTER(C.c_double)

OK = 0
INVALID_ARGUMENT, INVALID_PLAN, OUT_OF_MEMORY, DEVICE_ERROR, TIMEOUT, NUMERIC, NOT_SUPPORTED = 1, 2, 3, 4, 5, 6, 7
STATUS = {0: "ok", 1: "invalid argument", 2: "invalid plan", 3: "out of memory", 4: "device error",
          5: "timeout", 6: "numeric error", 7: "not supported"}

PLAN_HPSI, PLAN_LEFT, PLAN_RIGHT = 0, 1, 2
U1, TWOU1, SU2U1 = 1, 2, 3
PREC_FP64, PREC_FP64_EMULATED = 0, 1
SOLVER_GRAPH, SOLVER_STEPWISE = 0, 1


class DmrgError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib.dmrgb200_last_error().decode()
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != OK:
        raise DmrgError(status, where)


class IndexDesc(C.Structure):
    _fields_ = [("n", C.c_uint32), ("charges", i32p), ("sizes", u32p)]


class PlanDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("n_groups", C.c_uint32), ("g_t", u32p), ("g_c", u32p),
        ("n_in_blocks", C.c_uint32), ("in_rows", u32p), ("in_cols", u32p), ("in_off", u64p), ("in_size", C.c_uint64),
        ("n_out_blocks", C.c_uint32), ("out_rows", u32p), ("out_cols", u32p), ("out_off", u64p),
        ("out_size", C.c_uint64),
        ("n_t", C.c_uint32), ("t_lb", u32p), ("t_col", u32p), ("t_ci", u32p), ("t_trans", u8p), ("t_nb", u32p),
        ("t_brows", u32p), ("t_bcols", u32p), ("t_width", u32p),
        ("n_cohorts", C.c_uint32), ("c_lb", u32p), ("c_rb", u32p), ("c_ls", u32p), ("c_rs", u32p), ("c_ci", u32p),
        ("c_trans", u8p), ("c_nsrows", u32p), ("c_stripe", u32p), ("c_out_ci", u32p), ("c_unit", u32p),
        ("n_units", C.c_uint32), ("u_offset", u32p), ("u_ms", u32p), ("u_line", u32p),
        ("n_lines", C.c_uint32), ("l_b1", u32p), ("l_term", u32p),
        ("n_terms", C.c_uint32), ("term_alpha", f64p), ("term_t", u32p), ("term_col", u32p),
    ]


class MpoDesc(C.Structure):
    _fields_ = [
        ("symm", C.c_int), ("row_dim", C.c_uint32), ("col_dim", C.c_uint32),
        ("left_spin", i32p), ("right_spin", i32p), ("left_herm", u32p), ("left_phase", i32p),
        ("right_herm", u32p), ("right_phase", i32p),
        ("n_terms", C.c_uint32), ("term_b1", u32p), ("term_b2", u32p), ("term_op", u32p), ("term_scale", f64p),
        ("n_ops", C.c_uint32), ("op_spin", i32p), ("op_block", u32p), ("blk_in", i32p), ("blk_out", i32p),
        ("blk_entry", u32p), ("e_row", u32p), ("e_col", u32p), ("e_row_spin", i32p), ("e_col_spin", i32p),
        ("e_coeff", f64p),
    ]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("converged", C.c_int32), ("residual", C.c_double),
                ("hpsi_ms", C.c_double), ("solve_ms", C.c_double)]


class BoundaryView(C.Structure):
    _fields_ = [("n_cohorts", C.c_uint32), ("cohort_ptr", C.POINTER(C.c_void_p))]


class BlockCopy(C.Structure):
    """dmrgb200_block_copy: one column-major block copy, optionally scaled per row or column."""
    _fields_ = [("src_off", C.c_uint64), ("dst_off", C.c_uint64), ("scale_off", C.c_uint64),
                ("src_ld", C.c_uint32), ("dst_ld", C.c_uint32), ("rows", C.c_uint32), ("cols", C.c_uint32),
                ("scale_mode", C.c_uint32), ("reserved", C.c_uint32)]


SCALE_NONE, SCALE_ROWS, SCALE_COLS = 0, 1, 2


vp = C.c_void_p
_sigs = {
    "dmrgb200_status_string": ([C.c_int], C.c_char_p),
    "dmrgb200_last_error": ([], C.c_char_p),
    "dmrgb200_abi_version": ([], C.c_int),
    "dmrgb200_plan_check": ([vp, vp], C.c_int),
    "dmrgb200_plan_boundaries_changed": ([vp], C.c_int),
    "dmrgb200_hpsi_per_block": ([vp, vp, vp, vp, u64p], C.c_int),
    "dmrgb200_set_wait_limit": ([C.c_uint64], C.c_int),
    "dmrgb200_plan_set_precision": ([vp, C.c_int], C.c_int),
    "dmrgb200_plan_tune_slices": ([vp, vp, C.c_double, vp, i32p, f64p], C.c_int),
    "dmrgb200_wigner6j": ([C.c_int] * 6, C.c_double),
    "dmrgb200_wigner9j": ([C.c_int] * 9, C.c_double),
    "dmrgb200_set_coupling": ([C.c_int] * 9 + [C.c_double, f64p], None),
    "dmrgb200_context_create": ([C.c_int, C.POINTER(vp)], C.c_int),
    "dmrgb200_context_destroy": ([vp], C.c_int),
    "dmrgb200_plan_create": ([vp, C.POINTER(PlanDesc), C.POINTER(BoundaryView), C.POINTER(BoundaryView),
                              C.POINTER(vp)], C.c_int),
    "dmrgb200_plan_destroy": ([vp], C.c_int),
    "dmrgb200_plan_create_batched": ([vp, C.c_uint32, C.POINTER(PlanDesc), C.POINTER(BoundaryView),
                                      C.POINTER(BoundaryView), u64p, u64p, C.POINTER(vp)], C.c_int),
    "dmrgb200_plan_validate": ([C.POINTER(PlanDesc)], C.c_int),
    "dmrgb200_calibrate": ([C.c_int, f64p], C.c_int),
    "dmrgb200_plan_flops": ([vp, u64p], C.c_int),
    "dmrgb200_plan_scratch_bytes": ([vp, u64p], C.c_int),
    "dmrgb200_hpsi": ([vp, vp, vp, C.c_int, vp], C.c_int),
    "dmrgb200_hpsi_host": ([vp, vp, vp, vp], C.c_int),
    "dmrgb200_hpsi_adjoint": ([vp, vp, vp, vp, vp, vp], C.c_int),
    "dmrgb200_plan_set_timing": ([vp, C.c_int], C.c_int),
    "dmrgb200_plan_set_slices": ([vp, C.c_int], C.c_int),
    "dmrgb200_plan_set_solver": ([vp, C.c_int], C.c_int),
    "dmrgb200_plan_autotune": ([vp, vp, vp, vp, C.POINTER(C.c_int32)], C.c_int),
    "dmrgb200_gemm_variant_name": ([C.c_int], C.c_char_p),
    "dmrgb200_gemm_variant_count": ([], C.c_int),
    "dmrgb200_plan_set_gemm_variants": ([vp, C.c_int32, C.c_int32], C.c_int),
    "dmrgb200_plan_stage_times": ([vp, f64p, u64p, u64p], C.c_int),
    "dmrgb200_dgemm_f64": ([C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp, C.c_uint64, vp, C.c_uint64,
                            C.c_int, vp], C.c_int),
    "dmrgb200_dgemm_emulated": ([C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp, C.c_uint64, vp,
                                 C.c_uint64, C.c_int, vp], C.c_int),
    "dmrgb200_block_svd": ([C.c_uint32, u32p, u32p, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                            vp], C.c_int),
    "dmrgb200_copy_blocks": ([C.c_uint32, C.POINTER(BlockCopy), vp, vp, vp, vp], C.c_int),
    "dmrgb200_solve": ([vp, C.c_uint64, vp, C.POINTER(vp), C.c_uint32, C.c_double, C.c_uint32, f64p, vp,
                        C.POINTER(SolveStats), vp], C.c_int),
    "dmrgb200_hpsi_noalloc": ([C.POINTER(PlanDesc), C.POINTER(BoundaryView), C.POINTER(BoundaryView), vp, vp, vp],
                              C.c_int),
    "dmrgb200_step_execute": ([vp, vp, vp, C.POINTER(BoundaryView), vp], C.c_int),
    "dmrgb200_step_alpha_dm": ([vp, vp, vp, C.POINTER(BoundaryView), C.c_double, vp], C.c_int),
    "dmrgb200_mpo_create": ([C.POINTER(MpoDesc), C.POINTER(vp)], C.c_int),
    "dmrgb200_mpo_destroy": ([vp], C.c_int),
    "dmrgb200_bindex_create_edge": ([C.c_int, C.POINTER(IndexDesc), C.c_uint32, C.POINTER(vp)], C.c_int),
    "dmrgb200_bindex_destroy": ([vp], C.c_int),
    "dmrgb200_bindex_info": ([vp, u32p, u32p, u64p], C.c_int),
    "dmrgb200_bindex_describe": ([vp, u32p, u32p, u8p, u64p, u32p, u32p, u32p, i64p, f64p, u8p], C.c_int),
    "dmrgb200_schedule_hpsi": ([C.POINTER(IndexDesc), C.POINTER(IndexDesc), C.POINTER(IndexDesc), vp, vp, vp,
                                C.POINTER(vp)], C.c_int),
    "dmrgb200_schedule_left_step": ([C.POINTER(IndexDesc), C.POINTER(IndexDesc), C.POINTER(IndexDesc), vp, vp,
                                     C.c_int, C.POINTER(vp), C.POINTER(vp)], C.c_int),
    "dmrgb200_schedule_right_step": ([C.POINTER(IndexDesc), C.POINTER(IndexDesc), C.POINTER(IndexDesc), vp, vp,
                                      C.c_int, C.POINTER(vp), C.POINTER(vp)], C.c_int),
    "dmrgb200_schedule_export": ([vp, C.POINTER(PlanDesc)], C.c_int),
    "dmrgb200_schedule_flops": ([vp, u64p], C.c_int),
    "dmrgb200_schedule_term_sources": ([vp, u32p, f64p], C.c_int),
    "dmrgb200_schedule_destroy": ([vp], C.c_int),
    "dmrgb200_tensor_layout": ([C.POINTER(IndexDesc), C.POINTER(IndexDesc), C.POINTER(IndexDesc), C.c_int, u32p,
                                u32p, u32p, u64p, u64p], C.c_int),
}
EXPORTED = tuple(_sigs)
for _name, (_args, _res) in _sigs.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res


def ptr(a: np.ndarray | None, ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


# ---- plan descriptions <-> numpy --------------------------------------------------

_U32 = ("g_t", "g_c", "in_rows", "in_cols", "out_rows", "out_cols", "t_lb", "t_col", "t_ci", "t_nb", "t_brows",
        "t_bcols", "t_width", "c_lb", "c_rb", "c_ls", "c_rs", "c_ci", "c_nsrows", "c_stripe", "c_out_ci", "c_unit",
        "u_offset", "u_ms", "u_line", "l_b1", "l_term", "term_t", "term_col")
_U64 = ("in_off", "out_off")
_U8 = ("t_trans", "c_trans")
_F64 = ("term_alpha",)


def _lengths(d: PlanDesc) -> dict[str, int]:
    ng, nt, nc, nu, nl, nk = d.n_groups, d.n_t, d.n_cohorts, d.n_units, d.n_lines, d.n_terms
    L = {"g_t": ng + 1, "g_c": ng + 1, "in_rows": d.n_in_blocks, "in_cols": d.n_in_blocks, "in_off": d.n_in_blocks,
         "out_rows": d.n_out_blocks, "out_cols": d.n_out_blocks, "out_off": d.n_out_blocks,
         "c_unit": nc + 1, "u_line": nu + 1, "l_term": nl + 1}
    for k in ("t_lb", "t_col", "t_ci", "t_nb", "t_brows", "t_bcols", "t_width", "t_trans"):
        L[k] = nt
    for k in ("c_lb", "c_rb", "c_ls", "c_rs", "c_ci", "c_nsrows", "c_stripe", "c_out_ci", "c_trans"):
        L[k] = nc
    L.update(u_offset=nu, u_ms=nu, l_b1=nl, term_alpha=nk, term_t=nk, term_col=nk)
    return L


def desc_to_numpy(d: PlanDesc) -> dict:
    """Copy a plan description into numpy arrays (a plain dict)."""
    out = {"kind": int(d.kind), "in_size": int(d.in_size), "out_size": int(d.out_size)}
    L = _lengths(d)
    for name in _U32 + _U64 + _U8 + _F64:
        p = getattr(d, name)
        n = L[name]
        dt = np.uint32 if name in _U32 else np.uint64 if name in _U64 else np.uint8 if name in _U8 else np.float64
        if not p or n == 0:
            out[name] = np.zeros(0 if not (n and name == "t_width") else n, dtype=dt) if not p else np.zeros(n, dt)
            continue
        out[name] = np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True)
    return out


def numpy_to_desc(p: dict) -> tuple[PlanDesc, list]:
    """Build a PlanDesc pointing into the arrays of `p`; the returned list keeps them alive."""
    keep = []
    d = PlanDesc()
    d.kind = p["kind"]
    d.in_size = p["in_size"]
    d.out_size = p["out_size"]
    for name in _U32 + _U64 + _U8 + _F64:
        dt = np.uint32 if name in _U32 else np.uint64 if name in _U64 else np.uint8 if name in _U8 else np.float64
        a = np.ascontiguousarray(p[name], dtype=dt)
        keep.append(a)
        ct = C.c_uint32 if name in _U32 else C.c_uint64 if name in _U64 else C.c_uint8 if name in _U8 else C.c_double
        setattr(d, name, ptr(a, ct) if a.size else C.cast(None, C.POINTER(ct)))
    d.n_groups = len(p["g_t"]) - 1
    d.n_in_blocks = len(p["in_rows"])
    d.n_out_blocks = len(p["out_rows"])
    d.n_t = len(p["t_lb"])
    d.n_cohorts = len(p["c_lb"])
    d.n_units = len(p["u_offset"])
    d.n_lines = len(p["l_b1"])
    d.n_terms = len(p["term_alpha"])
    return d, keep
